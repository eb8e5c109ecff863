// Block-Jacobi / block ILU(k) preconditioner on the nodal-block (BSR) matrix:
// numeric factorisation and the two triangular solves, for the reference's
// iterative option files (-pc_type bjacobi -sub_pc_type ilu
// -sub_pc_factor_levels k, input/petsc_options_gmres.dat:2-5 and
// input/petsc_options_bcgs.dat:2-5, read through SolverPetsc.cpp:101,111).
//
// Factor layout (pattern from build_ilu_pattern): per node row i the blocks
// fptr[i]..fptr[i+1]-1, columns fcol[] sorted, the diagonal at fdiag[i].
// Strictly lower blocks hold the multipliers L_ip (unit block-lower factor),
// the others U_ij; fdinv[i] holds the inverse of U_ii (pivoted Gauss-Jordan).
//
// Scheduling is sync-free: one persistent grid whose warps draw rows from an
// atomic ticket in level-set order (the levels of the factorisation / lower
// solve DAG for the factorisation and the lower solve, of the upper solve DAG
// for the upper solve, computed on the host).  Rows of one level are
// independent, so a row only waits for rows handed out before it: a row whose
// inputs are not ready polls their flags (relaxed loads with back-off, then
// one acquire fence), and a finished row publishes its flag with a release
// store.  The earliest unfinished row always has its inputs, so progress is
// guaranteed; every wait is bounded and records a time-out in the control
// block instead of spinning forever.  Flags hold an epoch number: the last
// warp of a launch resets the ticket and advances the epoch, so no per-launch
// reset kernel is needed and launches can be captured in CUDA graphs.  Every
// row's arithmetic runs in a fixed order, so results do not depend on
// scheduling.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "linalg_kernels.cuh"

namespace cfdgpu {

struct TriCtl {
  unsigned int ticket;    // next chunk to hand out
  unsigned int exited;    // warps of the current launch that finished
  unsigned int epoch;     // launches completed; flags of this launch are set to epoch + 1
  unsigned int error;     // 0, or ILU_ERR_*
  int zero_pivot_row;     // factorisation: first row whose diagonal block is singular
};

constexpr unsigned int ILU_ERR_TIMEOUT = 1u;     // a dependency wait ran out (never expected)
constexpr unsigned int ILU_ERR_ZERO_PIVOT = 2u;  // singular diagonal block in the factorisation
constexpr int ILU_THREADS = 256;
constexpr int ILU_WARPS = ILU_THREADS / 32;
constexpr int ILU_SPIN_LIMIT = 1 << 21;          // ~1-2 s of polling per wait

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p)
{
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_u32(unsigned int *p, unsigned int v)
{
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned int ld_relaxed_u32(const unsigned int *p)
{
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Wait until *f == target (bounded): relaxed polls with exponential back-off.
// The caller completes the acquire with fence_acq_rel_gpu() after the polls
// of all its lanes (one fence per row instead of one acquire per input).
// Returns false after a time-out, or when another warp has already timed out.
__device__ __forceinline__ bool wait_flag(const unsigned int *f, unsigned int target, TriCtl *ctl)
{
  if (ld_relaxed_u32(f) == target) return true;
  unsigned int ns = 32;
  for (int it = 0; it < ILU_SPIN_LIMIT; it++) {
    __nanosleep(ns);
    if (ns < 1024) ns <<= 1;
    if (ld_relaxed_u32(f) == target) return true;
    if (*(volatile unsigned int *)&ctl->error) return false;
  }
  atomicCAS(&ctl->error, 0u, ILU_ERR_TIMEOUT);
  return false;
}

__device__ __forceinline__ int draw_ticket(TriCtl *ctl, int lane)
{
  unsigned int t = 0;
  if (lane == 0) t = atomicAdd(&ctl->ticket, 1u);
  return (int)__shfl_sync(0xffffffffu, t, 0);
}

// Exit accounting: the last warp of the launch resets the ticket and
// advances the epoch.
__device__ __forceinline__ void launch_done(TriCtl *ctl, int lane, unsigned int epoch)
{
  if (lane == 0) {
    __threadfence();
    const unsigned int nw = gridDim.x * (blockDim.x / 32);
    const unsigned int k = atomicAdd(&ctl->exited, 1u);
    if (k == nw - 1) {
      ctl->ticket = 0u;
      ctl->exited = 0u;
      __threadfence();
      *(volatile unsigned int *)&ctl->epoch = epoch + 1u;
      __threadfence();
    }
  }
}

template <typename T>
__device__ __forceinline__ double ld_cg(const T *p)
{
  return (double)__ldcg(p);
}

// Invert an NB x NB block (row-major, FP64) with partial pivoting; returns
// false when a pivot column is zero.
template <int NB>
__device__ __forceinline__ bool invert_block(double (&A)[NB][NB], double (&I)[NB][NB])
{
#pragma unroll
  for (int a = 0; a < NB; a++)
#pragma unroll
    for (int c = 0; c < NB; c++) I[a][c] = (a == c) ? 1.0 : 0.0;
  bool ok = true;
#pragma unroll
  for (int c = 0; c < NB; c++) {
    int piv = c;
#pragma unroll
    for (int r = c + 1; r < NB; r++)
      if (fabs(A[r][c]) > fabs(A[piv][c])) piv = r;
    if (A[piv][c] == 0.0) ok = false;
#pragma unroll
    for (int k = 0; k < NB; k++) {
      if (piv != c) {
        double t = A[c][k]; A[c][k] = A[piv][k]; A[piv][k] = t;
        t = I[c][k]; I[c][k] = I[piv][k]; I[piv][k] = t;
      }
    }
    const double p = A[c][c];
    const double d = (p != 0.0) ? 1.0 / p : 0.0;
#pragma unroll
    for (int k = 0; k < NB; k++) { A[c][k] *= d; I[c][k] *= d; }
#pragma unroll
    for (int r = 0; r < NB; r++) {
      if (r == c) continue;
      const double f = A[r][c];
#pragma unroll
      for (int k = 0; k < NB; k++) { A[r][k] -= f * A[c][k]; I[r][k] -= f * I[c][k]; }
    }
  }
  return ok;
}

// ---------------------------------------------------------------------------
// Numeric block ILU: one warp per node row, rows in ascending order.  For row
// i: W = the row of A on the factor pattern (fill blocks zero); for every
// pivot p < i of the row in increasing column order, L_ip = W_p U_pp^-1 and
// W_j -= L_ip U_pj for the blocks j > p of row p that lie in row i's pattern
// (their positions come from the symbolic phase's update map); then
// U_ii^-1.  AT is the type of the assembled matrix, FT of the factors
// (FP64 arithmetic in both cases).
template <int NB, typename AT, typename FT>
__global__ void __launch_bounds__(ILU_THREADS)
ilu_factor(int n, const int32_t *__restrict__ arow, const int32_t *__restrict__ aslot, const AT *__restrict__ aval,
           const int32_t *__restrict__ fptr, const int32_t *__restrict__ fcol, const int32_t *__restrict__ fdiag,
           const int64_t *__restrict__ uoff, const int32_t *__restrict__ umap, const int32_t *__restrict__ order,
           const int32_t *__restrict__ perm, FT *fval, FT *fdinv, unsigned int *flags, TriCtl *ctl)
{
  constexpr int BB = NB * NB;
  constexpr int G = 32 / BB;          // blocks per warp step
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __shared__ double Lsh[ILU_WARPS][BB];
  const unsigned int epoch = *(volatile unsigned int *)&ctl->epoch;
  const unsigned int target = epoch + 1u;
  const int g = lane / BB, e = lane % BB, er = e / NB, ec = e % NB;
  while (true) {
    const int tk = draw_ticket(ctl, lane);
    if (tk >= n) break;
    const int i = order[tk];
    const int f0 = fptr[i], f1 = fptr[i + 1], fd = fdiag[i];
    for (int64_t x = (int64_t)f0 * BB + lane; x < (int64_t)f1 * BB; x += 32) fval[x] = FT(0);
    __syncwarp();
    {
      const int ai = perm ? perm[i] : i;   // node of factor row i
      const int a0 = arow[ai], a1 = arow[ai + 1];
      for (int64_t x = lane; x < (int64_t)(a1 - a0) * BB; x += 32) {
        const int k = a0 + (int)(x / BB);
        const int s = aslot[k];
        if (s >= 0) fval[(int64_t)s * BB + x % BB] = (FT)aval[(int64_t)k * BB + x % BB];
      }
    }
    __syncwarp();
    for (int q = f0; q < fd; q++) {
      const int p = fcol[q];
      if (lane == 0) wait_flag(flags + p, target, ctl);
      __syncwarp();
      fence_acq_rel_gpu();
      if (lane < BB) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < NB; k++)
          s = fma((double)fval[(int64_t)q * BB + er * NB + k], ld_cg(fdinv + (int64_t)p * BB + k * NB + ec), s);
        Lsh[w][lane] = s;
      }
      __syncwarp();
      if (lane < BB) fval[(int64_t)q * BB + lane] = (FT)Lsh[w][lane];
      const int u0 = fdiag[p] + 1, u1 = fptr[p + 1];
      const int32_t *__restrict__ map = umap + uoff[q] - u0;
      double lrow[NB];
#pragma unroll
      for (int k = 0; k < NB; k++) lrow[k] = Lsh[w][er * NB + k];
      // UNR independent blocks per lane group in flight: all loads first,
      // then the updates (each target block is written by one lane group)
      constexpr int UNR = 4;
      for (int t0 = u0; t0 < u1; t0 += G * UNR) {
        int pos[UNR];
        double ub[UNR][NB];
#pragma unroll
        for (int r = 0; r < UNR; r++) {
          const int t = t0 + r * G + g;
          pos[r] = (g < G && t < u1) ? map[t] : -1;
#pragma unroll
          for (int k = 0; k < NB; k++)
            ub[r][k] = (pos[r] >= 0) ? ld_cg(fval + (int64_t)t * BB + k * NB + ec) : 0.0;
        }
#pragma unroll
        for (int r = 0; r < UNR; r++) {
          if (pos[r] >= 0) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < NB; k++) s = fma(lrow[k], ub[r][k], s);
            fval[(int64_t)pos[r] * BB + e] = (FT)((double)fval[(int64_t)pos[r] * BB + e] - s);
          }
        }
      }
      __syncwarp();
    }
    if (lane == 0) {
      double A[NB][NB], I[NB][NB];
#pragma unroll
      for (int a = 0; a < NB; a++)
#pragma unroll
        for (int c = 0; c < NB; c++) A[a][c] = (double)fval[(int64_t)fd * BB + a * NB + c];
      if (!invert_block<NB>(A, I)) {
        if (atomicCAS(&ctl->error, 0u, ILU_ERR_ZERO_PIVOT) == 0u) ctl->zero_pivot_row = i;
      }
#pragma unroll
      for (int a = 0; a < NB; a++)
#pragma unroll
        for (int c = 0; c < NB; c++) fdinv[(int64_t)i * BB + a * NB + c] = (FT)I[a][c];
    }
    // every lane's writes of the row are visible before the flag
    __threadfence();
    __syncwarp();
    if (lane == 0) st_release_u32(flags + i, target);
  }
  launch_done(ctl, lane, epoch);
}

// ---------------------------------------------------------------------------
// Triangular solves z = (L U)^-1 r.
//
// The values are their own ready flags: the intermediate vector y and the
// output z hold a signalling-NaN sentinel (a bit pattern no arithmetic
// produces) until their row is written, so a row whose inputs are not ready
// polls the input values themselves (relaxed loads with back-off) and needs
// no separate flag, fence or second round trip.  The lower solve writes y_i
// and resets z_i to the sentinel for the upper solve; the upper solve reads
// y_i, writes z_i and resets y_i to the sentinel for the next lower solve.
// y is the handle's own buffer (sentinel-filled at creation); r and z must
// not overlap.
//
// Lower:  y_i = r_i - sum_{p<i} L_ip y_p
// Upper:  z_i = U_ii^-1 (y_i - sum_{p>i} U_ip z_p)
// st/j: inside a GMRES chunk the launch is skipped once the cycle has ended;
// active: inside a BiCGStab chunk, once the solve has ended.
template <typename VT> struct Sentinel;
template <> struct Sentinel<double> {
  using U = unsigned long long;
  static constexpr U bits = 0x7FF4C0FFEE15BAD1ull;   // signalling NaN
  static __device__ __forceinline__ U load(const double *p)
  {
    U v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
  }
  static __device__ __forceinline__ void store(double *p, double x)
  {
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(x) : "memory");
  }
  static __device__ __forceinline__ double value(U v) { return __longlong_as_double((long long)v); }
  static __device__ __forceinline__ double sentinel() { return __longlong_as_double((long long)bits); }
};
template <> struct Sentinel<float> {
  using U = unsigned int;
  static constexpr U bits = 0x7FA0C0DEu;               // signalling NaN
  static __device__ __forceinline__ U load(const float *p)
  {
    U v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
  }
  static __device__ __forceinline__ void store(float *p, float x)
  {
    asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(x) : "memory");
  }
  static __device__ __forceinline__ float value(U v) { return __uint_as_float(v); }
  static __device__ __forceinline__ float sentinel() { return __uint_as_float(bits); }
};

// value at p once it is no longer the sentinel (bounded wait)
template <typename VT>
__device__ __forceinline__ double wait_value(const VT *p, typename Sentinel<VT>::U v, TriCtl *ctl)
{
  using S = Sentinel<VT>;
  if (v != S::bits) return (double)S::value(v);
  unsigned int ns = 32;
  for (int it = 0; it < ILU_SPIN_LIMIT; it++) {
    __nanosleep(ns);
    if (ns < 256) ns <<= 1;
    v = S::load(p);
    if (v != S::bits) return (double)S::value(v);
    if (*(volatile unsigned int *)&ctl->error) break;
  }
  atomicCAS(&ctl->error, 0u, ILU_ERR_TIMEOUT);
  return 0.0;
}

__global__ void fill_sentinel_f64(int64_t n, double *y)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = Sentinel<double>::sentinel();
}

__global__ void fill_sentinel_f32(int64_t n, float *y)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = Sentinel<float>::sentinel();
}

constexpr int TRSV_BATCH = 4;   // input loads in flight per lane
constexpr int TRSV_CHAIN_MAX = 128;

// One warp per chain of rows (see IluPattern::lchain / uchain), chains in
// level order of the chain DAG.  The chain's rows are solved in order; inputs
// from the chain itself come from shared memory, inputs from other chains
// from global memory once they are no longer the sentinel.
//
// Lower:  y_i = r_P(i) - sum_{p<i} L_ip y_p
// Upper:  z_P(i) = U_ii^-1 (y_i - sum_{p>i} U_ip z_P(p))
// with P the factor's row order (perm; NULL: the identity): y is indexed by
// factor row, r and z by node.
template <int NB, bool UPPER, typename FT, typename VT>
__global__ void __launch_bounds__(ILU_THREADS)
ilu_trsv(int nchains, const int32_t *__restrict__ order, const int32_t *__restrict__ chains,
         const int32_t *__restrict__ fptr, const int32_t *__restrict__ fcol, const int32_t *__restrict__ fdiag,
         const FT *__restrict__ fval, const FT *__restrict__ fdinv, const int32_t *__restrict__ perm, const VT *r,
         VT *y, VT *z, TriCtl *ctl, const GmresState *__restrict__ st, int j, const int *__restrict__ active)
{
  if (st && (!st->active || st->it != j)) return;
  if (active && !active[0]) return;
  using S = Sentinel<VT>;
  constexpr int BB = NB * NB;
  constexpr int G = 32 / BB;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __shared__ double red[ILU_WARPS][32];
  __shared__ double sv[ILU_WARPS][NB];
  __shared__ double cache[ILU_WARPS][TRSV_CHAIN_MAX * NB];
  const unsigned int epoch = *(volatile unsigned int *)&ctl->epoch;
  const int g = lane / BB, e = lane % BB, ec = e % NB;
  // the vector the off-diagonal products read: y (lower) or z (upper)
  const VT *src = UPPER ? z : y;
  while (true) {
    const int tk = draw_ticket(ctl, lane);
    if (tk >= nchains) break;
    const int c = order[tk];
    const int lo = chains[2 * c], hi = chains[2 * c + 1];
    for (int step = 0; step < hi - lo; step++) {
      const int i = UPPER ? hi - 1 - step : lo + step;
      const int q0 = UPPER ? fdiag[i] + 1 : fptr[i];
      const int q1 = UPPER ? fptr[i + 1] : fdiag[i];
      // blocks in the order farthest column first, so the chain's own
      // previous row (the input finished last) is consumed last
      double acc = 0.0;
      const int nq = q1 - q0;
      for (int qb = 0; qb < nq; qb += G * TRSV_BATCH) {
        typename S::U v[TRSV_BATCH];
        int p[TRSV_BATCH];
        double a[TRSV_BATCH];
        bool own[TRSV_BATCH];
#pragma unroll
        for (int k = 0; k < TRSV_BATCH; k++) {
          const int qq = qb + k * G + g;
          const bool ok = (g < G && qq < nq);
          const int q = UPPER ? q1 - 1 - qq : q0 + qq;
          p[k] = ok ? fcol[q] : -1;
          a[k] = ok ? (double)fval[(int64_t)q * BB + e] : 0.0;
          own[k] = ok && (UPPER ? p[k] < hi : p[k] >= lo);
        }
        // z is indexed by node, y by factor row
        int64_t at[TRSV_BATCH];
#pragma unroll
        for (int k = 0; k < TRSV_BATCH; k++)
          at[k] = (int64_t)((UPPER && perm && p[k] >= 0) ? perm[p[k]] : p[k]) * NB + ec;
#pragma unroll
        for (int k = 0; k < TRSV_BATCH; k++) v[k] = (p[k] >= 0 && !own[k]) ? S::load(src + at[k]) : 0;
#pragma unroll
        for (int k = 0; k < TRSV_BATCH; k++) {
          if (p[k] < 0) continue;
          const double xv = own[k] ? cache[w][(UPPER ? hi - 1 - p[k] : p[k] - lo) * NB + ec]
                                   : wait_value<VT>(src + at[k], v[k], ctl);
          acc = fma(a[k], xv, acc);
        }
      }
      red[w][lane] = acc;
      __syncwarp();
      const int64_t node = perm ? perm[i] : i;
      if (lane < NB) {
        double s = UPPER ? (double)y[(int64_t)i * NB + lane] : (double)r[node * NB + lane];
#pragma unroll
        for (int gg = 0; gg < G; gg++)
#pragma unroll
          for (int cc = 0; cc < NB; cc++) s -= red[w][gg * BB + lane * NB + cc];
        sv[w][lane] = s;
      }
      __syncwarp();
      if (lane < NB) {
        if (UPPER) {
          double v = 0.0;
#pragma unroll
          for (int cc = 0; cc < NB; cc++) v = fma((double)fdinv[(int64_t)i * BB + lane * NB + cc], sv[w][cc], v);
          const VT vv = (VT)v;
          cache[w][step * NB + lane] = (double)vv;
          S::store(z + node * NB + lane, vv);
          y[(int64_t)i * NB + lane] = S::sentinel();
        } else {
          const VT vv = (VT)sv[w][lane];
          cache[w][step * NB + lane] = (double)vv;
          z[node * NB + lane] = S::sentinel();
          S::store(y + (int64_t)i * NB + lane, vv);
        }
      }
      __syncwarp();
    }
  }
  launch_done(ctl, lane, epoch);
}

}  // namespace cfdgpu
