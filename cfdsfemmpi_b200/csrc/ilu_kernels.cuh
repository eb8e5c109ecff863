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
#ifndef ILU_SPIN_HOT
#define ILU_SPIN_HOT 256
#endif
// polls without sleeping before the back-off starts: an input usually
// arrives within a few L2 round trips, and a sleeping warp wakes late
constexpr int ILU_SPIN_HOT_POLLS = ILU_SPIN_HOT;

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

// Wait until *f == target (bounded): relaxed polls, the first ILU_SPIN_HOT_POLLS
// back to back, then with exponential back-off.
// The caller completes the acquire with fence_acq_rel_gpu() after the polls
// of all its lanes (one fence per row instead of one acquire per input).
// Returns false after a time-out, or when another warp has already timed out.
__device__ __forceinline__ bool wait_flag(const unsigned int *f, unsigned int target, TriCtl *ctl)
{
  if (ld_relaxed_u32(f) == target) return true;
  unsigned int ns = 32;
  for (int it = 0; it < ILU_SPIN_LIMIT; it++) {
    if (it >= ILU_SPIN_HOT_POLLS) {
      __nanosleep(ns);
      if (ns < 1024) ns <<= 1;
    }
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

// value at p once it is no longer the sentinel (bounded wait; polls as in wait_flag)
template <typename VT>
__device__ __forceinline__ double wait_value(const VT *p, typename Sentinel<VT>::U v, TriCtl *ctl)
{
  using S = Sentinel<VT>;
  if (v != S::bits) return (double)S::value(v);
  unsigned int ns = 32;
  for (int it = 0; it < ILU_SPIN_LIMIT; it++) {
    if (it >= ILU_SPIN_HOT_POLLS) {
      __nanosleep(ns);
      if (ns < 256) ns <<= 1;
    }
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

constexpr int TRSV_BATCH = 4;        // input loads in flight per lane for blocks beyond the pipelined ones
constexpr int TRSV_CHAIN_MAX = 128;
constexpr int TRSV_ROW_BLOCKS = 14;  // blocks per row held in the pipeline registers (a 27-point row: 13)

// One warp per chain of rows (see IluPattern::lchain / uchain), chains in
// level order of the chain DAG.  The chain's rows are solved in order; inputs
// from the chain itself come from shared memory, inputs from other chains
// from global memory once they are no longer the sentinel.
//
// The rows of a chain run through a three-stage software pipeline, so that
// the memory latencies of a row overlap the work of the row before it: while
// row s is finished, the warp already holds the matrix values and the other
// chains' input values of row s+1, the column indices of row s+2 are in
// flight, and so is the block range of row s+3.  A lane holds PF blocks of a
// row in registers (G blocks per warp pass, lanes g = lane / (NB*NB));
// further blocks (fill rows of ILU(k), k >= 1) are loaded when their row is
// finished.  Per lane the products are summed in block order, so the result
// does not depend on how far ahead the loads ran.
//
// Lower:  y_i = r_P(i) - sum_{p<i} L_ip y_p
// Upper:  z_P(i) = U_ii^-1 (y_i - sum_{p>i} U_ip z_P(p))
// with P the factor's row order (perm; NULL: the identity): y is indexed by
// factor row, r and z by node.
template <int NB, bool UPPER, typename FT, typename VT>
__global__ void __launch_bounds__(ILU_THREADS, 2)
ilu_trsv(int nchains, const int32_t *__restrict__ order, const int32_t *__restrict__ chains,
         const int32_t *__restrict__ fptr, const int32_t *__restrict__ fcol, const int32_t *__restrict__ fdiag,
         const FT *__restrict__ fval, const FT *__restrict__ fdinv, const int32_t *__restrict__ perm, const VT *r,
         VT *y, VT *z, TriCtl *ctl, const GmresState *__restrict__ st, int j, const int *__restrict__ active)
{
  if (st && (!st->active || st->it != j)) return;
  if (active && !active[0]) return;
  using S = Sentinel<VT>;
  using U = typename S::U;
  constexpr int BB = NB * NB;
  constexpr int G = 32 / BB;
  constexpr int PF = (TRSV_ROW_BLOCKS + G - 1) / G;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __shared__ double red[ILU_WARPS][32];
  __shared__ double sv[ILU_WARPS][NB];
  __shared__ double cache[ILU_WARPS][TRSV_CHAIN_MAX * NB];
  const unsigned int epoch = *(volatile unsigned int *)&ctl->epoch;
  const int g = lane / BB, e = lane % BB, ec = e % NB;
  const bool glane = g < G;
  // the vector the off-diagonal products read: y (lower) or z (upper)
  const VT *src = UPPER ? z : y;
  // position of column p in src: z is indexed by node, y by factor row
  auto at = [&](int p) -> int64_t { return (int64_t)((UPPER && perm) ? perm[p] : p) * NB + ec; };
  while (true) {
    const int tk = draw_ticket(ctl, lane);
    if (tk >= nchains) break;
    const int c = order[tk];
    const int lo = chains[2 * c], hi = chains[2 * c + 1];
    const int len = hi - lo;
    auto row = [&](int s) { return UPPER ? hi - 1 - s : lo + s; };
    auto own = [&](int p) { return UPPER ? p < hi : p >= lo; };
    // strictly lower (upper) blocks [qa, qb) of the chain's s-th row; the
    // qq-th block of a row is the farthest column first, so the chain's own
    // previous row (the input finished last) is consumed last
    auto range = [&](int s, int &qa, int &qb) {
      qa = qb = 0;
      if (s < len) {
        const int i = row(s);
        qa = UPPER ? fdiag[i] + 1 : fptr[i];
        qb = UPPER ? fptr[i + 1] : fdiag[i];
      }
    };
    auto blk = [&](int qa, int qb, int qq) { return UPPER ? qb - 1 - qq : qa + qq; };
    auto cols = [&](int qa, int qb, int (&p)[PF]) {
#pragma unroll
      for (int k = 0; k < PF; k++) {
        const int qq = k * G + g;
        p[k] = (glane && qq < qb - qa) ? fcol[blk(qa, qb, qq)] : -1;
      }
    };
    // matrix values, other chains' inputs and the row's own data (r_P(i) or
    // y_i, and the row of U_ii^-1) of the s-th row
    auto vals = [&](int s, int qa, int qb, const int (&p)[PF], FT (&a)[PF], U (&v)[PF], VT &b, FT (&d)[NB]) {
#pragma unroll
      for (int k = 0; k < PF; k++)
        a[k] = p[k] >= 0 ? fval[(int64_t)blk(qa, qb, k * G + g) * BB + e] : FT(0);
#pragma unroll
      for (int k = 0; k < PF; k++) v[k] = (p[k] >= 0 && !own(p[k])) ? S::load(src + at(p[k])) : U(0);
      b = VT(0);
#pragma unroll
      for (int cc = 0; cc < NB; cc++) d[cc] = FT(0);
      if (s < len) {
        const int i = row(s);
        if constexpr (NB == 4) {
          // every lane: entry er of the row's vector, entry (er, ec) of U_ii^-1
          if (UPPER) {
            b = y[(int64_t)i * NB + e / NB];
            d[0] = fdinv[(int64_t)i * BB + e];
          } else {
            b = r[(int64_t)(perm ? perm[i] : i) * NB + e / NB];
          }
        } else if (lane < NB) {
          if (UPPER) {
            b = y[(int64_t)i * NB + lane];
#pragma unroll
            for (int cc = 0; cc < NB; cc++) d[cc] = fdinv[(int64_t)i * BB + lane * NB + cc];
          } else {
            b = r[(int64_t)(perm ? perm[i] : i) * NB + lane];
          }
        }
      }
    };

    int qa0, qb0, qa1, qb1, qa2, qb2;
    int p0[PF], p1[PF], p2[PF];
    FT a0[PF], a1[PF], d0[NB], d1[NB];
    U v0[PF], v1[PF];
    VT b0, b1;
    range(0, qa0, qb0);
    range(1, qa1, qb1);
    range(2, qa2, qb2);
    cols(qa0, qb0, p0);
    cols(qa1, qb1, p1);
    vals(0, qa0, qb0, p0, a0, v0, b0, d0);
    for (int s = 0; s < len; s++) {
      const int i = row(s);
      // loads for the rows ahead
      vals(s + 1, qa1, qb1, p1, a1, v1, b1, d1);
      cols(qa2, qb2, p2);
      int qa3, qb3;
      range(s + 3, qa3, qb3);

      // row s: products in block order, other chains' inputs once they are
      // no longer the sentinel, the chain's own from shared memory
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < PF; k++) {
        if (p0[k] < 0) continue;
        const double xv = own(p0[k]) ? cache[w][(UPPER ? hi - 1 - p0[k] : p0[k] - lo) * NB + ec]
                                     : wait_value<VT>(src + at(p0[k]), v0[k], ctl);
        acc = fma((double)a0[k], xv, acc);
      }
      const int nq = qb0 - qa0;
      for (int qb = G * PF; qb < nq; qb += G * TRSV_BATCH) {
        U v[TRSV_BATCH];
        int p[TRSV_BATCH];
        double a[TRSV_BATCH];
#pragma unroll
        for (int k = 0; k < TRSV_BATCH; k++) {
          const int qq = qb + k * G + g;
          const bool ok = (glane && qq < nq);
          const int q = blk(qa0, qb0, qq);
          p[k] = ok ? fcol[q] : -1;
          a[k] = ok ? (double)fval[(int64_t)q * BB + e] : 0.0;
        }
#pragma unroll
        for (int k = 0; k < TRSV_BATCH; k++) v[k] = (p[k] >= 0 && !own(p[k])) ? S::load(src + at(p[k])) : U(0);
#pragma unroll
        for (int k = 0; k < TRSV_BATCH; k++) {
          if (p[k] < 0) continue;
          const double xv = own(p[k]) ? cache[w][(UPPER ? hi - 1 - p[k] : p[k] - lo) * NB + ec]
                                      : wait_value<VT>(src + at(p[k]), v[k], ctl);
          acc = fma(a[k], xv, acc);
        }
      }
      const int64_t node = perm ? perm[i] : i;
      if constexpr (NB == 4) {
        // 4x4 blocks, two per warp pass: lane = 16 g + 4 er + ec.  Sum the
        // products of block row er over ec (lane bits 0-1) and g (bit 4)
        // with shuffles; every lane then holds entry er of the row's vector.
        constexpr unsigned FULL = 0xffffffffu;
        double t = acc;
        t += __shfl_xor_sync(FULL, t, 1);
        t += __shfl_xor_sync(FULL, t, 2);
        t += __shfl_xor_sync(FULL, t, 16);
        const double sr = (double)b0 - t;
        const int er = e / NB;
        if (UPPER) {
          // z_i = U_ii^-1 s: lane (er, ec) forms (U_ii^-1)_{er,ec} s_ec, summed over ec
          double x = (double)d0[0] * __shfl_sync(FULL, sr, ec * NB);
          x += __shfl_xor_sync(FULL, x, 1);
          x += __shfl_xor_sync(FULL, x, 2);
          if (lane < BB && ec == 0) {
            const VT vv = (VT)x;
            cache[w][s * NB + er] = (double)vv;
            S::store(z + node * NB + er, vv);
            y[(int64_t)i * NB + er] = S::sentinel();
          }
        } else if (lane < BB && ec == 0) {
          const VT vv = (VT)sr;
          cache[w][s * NB + er] = (double)vv;
          z[node * NB + er] = S::sentinel();
          S::store(y + (int64_t)i * NB + er, vv);
        }
        __syncwarp();
      } else {
      red[w][lane] = acc;
      __syncwarp();
      if (lane < NB) {
        double sum = (double)b0;
#pragma unroll
        for (int gg = 0; gg < G; gg++)
#pragma unroll
          for (int cc = 0; cc < NB; cc++) sum -= red[w][gg * BB + lane * NB + cc];
        sv[w][lane] = sum;
      }
      __syncwarp();
      if (lane < NB) {
        if (UPPER) {
          double x = 0.0;
#pragma unroll
          for (int cc = 0; cc < NB; cc++) x = fma((double)d0[cc], sv[w][cc], x);
          const VT vv = (VT)x;
          cache[w][s * NB + lane] = (double)vv;
          S::store(z + node * NB + lane, vv);
          y[(int64_t)i * NB + lane] = S::sentinel();
        } else {
          const VT vv = (VT)sv[w][lane];
          cache[w][s * NB + lane] = (double)vv;
          z[node * NB + lane] = S::sentinel();
          S::store(y + (int64_t)i * NB + lane, vv);
        }
      }
      __syncwarp();
      }
      // advance the pipeline
      qa0 = qa1; qb0 = qb1; qa1 = qa2; qb1 = qb2; qa2 = qa3; qb2 = qb3;
      b0 = b1;
#pragma unroll
      for (int k = 0; k < PF; k++) {
        p0[k] = p1[k]; p1[k] = p2[k]; a0[k] = a1[k]; v0[k] = v1[k];
      }
#pragma unroll
      for (int cc = 0; cc < NB; cc++) d0[cc] = d1[cc];
    }
  }
  launch_done(ctl, lane, epoch);
}

}  // namespace cfdgpu
