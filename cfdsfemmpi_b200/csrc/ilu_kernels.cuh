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
// Scheduling is sync-free: one persistent grid whose warps draw consecutive
// row chunks from an atomic ticket (ascending rows for the factorisation and
// the lower solve, descending for the upper solve).  A chunk whose rows need
// rows of another chunk waits on that chunk's flag (acquire load), and a
// finished chunk publishes its flag with a release store.  Tickets are drawn
// in dependency order by running warps, so the earliest unfinished chunk
// always has its inputs and progress is guaranteed; every wait is bounded and
// records a time-out in the control block instead of spinning forever.  Flags
// hold an epoch number: the last warp of a launch resets the ticket and
// advances the epoch, so no per-launch reset kernel is needed and launches
// can be captured in CUDA graphs.  Every row's arithmetic runs in a fixed
// order, so results do not depend on scheduling.
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
constexpr int ILU_MAX_CHUNK = 32;
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

// Wait until *f == target (bounded).  Returns false after a time-out, or when
// another warp has already timed out.
__device__ __forceinline__ bool wait_flag(const unsigned int *f, unsigned int target, TriCtl *ctl)
{
  if (ld_acquire_u32(f) == target) return true;
  for (int it = 0; it < ILU_SPIN_LIMIT; it++) {
    __nanosleep(64);
    if (ld_acquire_u32(f) == target) return true;
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

// position of column j in fcol[lo, hi) (sorted), or -1
__device__ __forceinline__ int find_col(const int32_t *__restrict__ fcol, int lo, int hi, int j)
{
  const int end = hi;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (fcol[mid] < j) lo = mid + 1;
    else hi = mid;
  }
  return (lo < end && fcol[lo] == j) ? lo : -1;
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
// W_j -= L_ip U_pj for the blocks j > p of row p that lie in row i's pattern;
// then U_ii^-1.  AT is the type of the assembled matrix, FT of the factors
// (FP64 arithmetic in both cases).
template <int NB, typename AT, typename FT>
__global__ void __launch_bounds__(ILU_THREADS)
ilu_factor(int n, const int32_t *__restrict__ arow, const int32_t *__restrict__ aslot, const AT *__restrict__ aval,
           const int32_t *__restrict__ fptr, const int32_t *__restrict__ fcol, const int32_t *__restrict__ fdiag,
           FT *fval, FT *fdinv, unsigned int *flags, TriCtl *ctl)
{
  constexpr int BB = NB * NB;
  constexpr int G = 32 / BB;          // blocks per warp step
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __shared__ double Lsh[ILU_WARPS][BB];
  const unsigned int epoch = *(volatile unsigned int *)&ctl->epoch;
  const unsigned int target = epoch + 1u;
  const int g = lane / BB, e = lane % BB, er = e / NB, ec = e % NB;
  while (true) {
    const int i = draw_ticket(ctl, lane);
    if (i >= n) break;
    const int f0 = fptr[i], f1 = fptr[i + 1], fd = fdiag[i];
    for (int64_t x = (int64_t)f0 * BB + lane; x < (int64_t)f1 * BB; x += 32) fval[x] = FT(0);
    __syncwarp();
    {
      const int a0 = arow[i], a1 = arow[i + 1];
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
      for (int t0 = u0; t0 < u1; t0 += G) {
        const int t = t0 + g;
        if (g < G && t < u1) {
          const int j = fcol[t];
          const int pos = find_col(fcol, q + 1, f1, j);
          if (pos >= 0) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < NB; k++) s = fma(Lsh[w][er * NB + k], ld_cg(fval + (int64_t)t * BB + k * NB + ec), s);
            fval[(int64_t)pos * BB + e] = (FT)((double)fval[(int64_t)pos * BB + e] - s);
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
    __syncwarp();
    if (lane == 0) {
      __threadfence();
      st_release_u32(flags + i, target);
    }
  }
  launch_done(ctl, lane, epoch);
}

// ---------------------------------------------------------------------------
// Triangular solves z = (L U)^-1 r.  A warp takes a chunk of `chunk`
// consecutive rows (ascending for L, descending for U) and solves them in
// order, keeping the chunk's results in shared memory; rows of other chunks
// are read after their chunk's flag (one flag per chunk).
//
// Lower:  y_i = r_i - sum_{p<i} L_ip y_p              (in place over r allowed)
// Upper:  z_i = U_ii^-1 (y_i - sum_{p>i} U_ip z_p)   (in place over y allowed)
// st/j: inside a GMRES chunk the launch is skipped once the cycle has ended;
// active: inside a BiCGStab chunk, once the solve has ended.
template <int NB, typename FT, typename VT>
__global__ void __launch_bounds__(ILU_THREADS)
ilu_lsolve(int n, int chunk, const int32_t *__restrict__ fptr, const int32_t *__restrict__ fcol,
           const int32_t *__restrict__ fdiag, const FT *__restrict__ fval, const VT *r, VT *y, unsigned int *flags,
           TriCtl *ctl, const GmresState *__restrict__ st, int j, const int *__restrict__ active)
{
  if (st && (!st->active || st->it != j)) return;
  if (active && !active[0]) return;
  constexpr int BB = NB * NB;
  constexpr int G = 32 / BB;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __shared__ double ych[ILU_WARPS][ILU_MAX_CHUNK * NB];
  __shared__ double red[ILU_WARPS][32];
  const unsigned int epoch = *(volatile unsigned int *)&ctl->epoch;
  const unsigned int target = epoch + 1u;
  const int g = lane / BB, e = lane % BB, ec = e % NB;
  const int nchunks = (n + chunk - 1) / chunk;
  while (true) {
    const int t = draw_ticket(ctl, lane);
    if (t >= nchunks) break;
    const int i0 = t * chunk, i1 = min(n, i0 + chunk);
    for (int i = i0; i < i1; i++) {
      const int q0 = fptr[i], q1 = fdiag[i];
      for (int q = q0 + lane; q < q1; q += 32) {
        const int p = fcol[q];
        if (p < i0) wait_flag(flags + p / chunk, target, ctl);
      }
      __syncwarp();
      double acc = 0.0;
      for (int qb = q0; qb < q1; qb += G) {
        const int q = qb + g;
        if (g < G && q < q1) {
          const int p = fcol[q];
          const double yp = (p >= i0) ? ych[w][(p - i0) * NB + ec] : ld_cg(y + (int64_t)p * NB + ec);
          acc = fma((double)fval[(int64_t)q * BB + e], yp, acc);
        }
      }
      red[w][lane] = acc;
      __syncwarp();
      if (lane < NB) {
        double s = (double)r[(int64_t)i * NB + lane];
#pragma unroll
        for (int gg = 0; gg < G; gg++)
#pragma unroll
          for (int c = 0; c < NB; c++) s -= red[w][gg * BB + lane * NB + c];
        ych[w][(i - i0) * NB + lane] = s;
        y[(int64_t)i * NB + lane] = (VT)s;
      }
      __syncwarp();
    }
    if (lane == 0) {
      __threadfence();
      st_release_u32(flags + t, target);
    }
  }
  launch_done(ctl, lane, epoch);
}

template <int NB, typename FT, typename VT>
__global__ void __launch_bounds__(ILU_THREADS)
ilu_usolve(int n, int chunk, const int32_t *__restrict__ fptr, const int32_t *__restrict__ fcol,
           const int32_t *__restrict__ fdiag, const FT *__restrict__ fval, const FT *__restrict__ fdinv, const VT *y,
           VT *z, unsigned int *flags, TriCtl *ctl, const GmresState *__restrict__ st, int j,
           const int *__restrict__ active)
{
  if (st && (!st->active || st->it != j)) return;
  if (active && !active[0]) return;
  constexpr int BB = NB * NB;
  constexpr int G = 32 / BB;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __shared__ double zch[ILU_WARPS][ILU_MAX_CHUNK * NB];
  __shared__ double red[ILU_WARPS][32];
  __shared__ double sv[ILU_WARPS][NB];
  const unsigned int epoch = *(volatile unsigned int *)&ctl->epoch;
  const unsigned int target = epoch + 1u;
  const int g = lane / BB, e = lane % BB, ec = e % NB;
  const int nchunks = (n + chunk - 1) / chunk;
  while (true) {
    const int t = draw_ticket(ctl, lane);
    if (t >= nchunks) break;
    // chunk t covers rows hi, hi-1, ..., lo
    const int hi = n - 1 - t * chunk, lo = max(0, hi - chunk + 1);
    for (int i = hi; i >= lo; i--) {
      const int q0 = fdiag[i] + 1, q1 = fptr[i + 1];
      for (int q = q0 + lane; q < q1; q += 32) {
        const int p = fcol[q];
        if (p > hi) wait_flag(flags + (n - 1 - p) / chunk, target, ctl);
      }
      __syncwarp();
      double acc = 0.0;
      for (int qb = q0; qb < q1; qb += G) {
        const int q = qb + g;
        if (g < G && q < q1) {
          const int p = fcol[q];
          const double zp = (p <= hi) ? zch[w][(hi - p) * NB + ec] : ld_cg(z + (int64_t)p * NB + ec);
          acc = fma((double)fval[(int64_t)q * BB + e], zp, acc);
        }
      }
      red[w][lane] = acc;
      __syncwarp();
      if (lane < NB) {
        double s = ld_cg(y + (int64_t)i * NB + lane);
#pragma unroll
        for (int gg = 0; gg < G; gg++)
#pragma unroll
          for (int c = 0; c < NB; c++) s -= red[w][gg * BB + lane * NB + c];
        sv[w][lane] = s;
      }
      __syncwarp();
      if (lane < NB) {
        double v = 0.0;
#pragma unroll
        for (int c = 0; c < NB; c++) v = fma((double)fdinv[(int64_t)i * BB + lane * NB + c], sv[w][c], v);
        zch[w][(hi - i) * NB + lane] = v;
        z[(int64_t)i * NB + lane] = (VT)v;
      }
      __syncwarp();
    }
    if (lane == 0) {
      __threadfence();
      st_release_u32(flags + t, target);
    }
  }
  launch_done(ctl, lane, epoch);
}

}  // namespace cfdgpu
