// Sparse and dense linear-algebra kernels for the nodal-block (BSR) system:
// SpMV with the preconditioner fused into its epilogue, deterministic
// reductions, and the device-side pieces of restarted GMRES (PETSc 3.10
// KSPGMRES semantics: classical Gram-Schmidt, left preconditioning,
// preconditioned-residual norm, KSPConvergedDefault; the reference calls it
// from src/base/SolverPetsc.cpp:253).
//
// Determinism: every reduction uses a fixed grid, a fixed per-thread stride,
// a fixed in-CTA tree, and a final pass (last CTA, or one warp per output)
// that adds the per-CTA partials in index order, so results do not depend on
// scheduling.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cfdgpu {

constexpr int RED_BLOCKS = 296;     // 2 x 148 SMs
constexpr int RED_THREADS = 256;

// ---------------------------------------------------------------------------
// GMRES control block (device memory).  One thread (the last CTA of a
// reduction kernel) updates it; every other kernel only reads it.
struct GmresState {
  int it;          // Arnoldi columns built in the current cycle
  int its;         // total iterations (KSP iteration count)
  int reason;      // KSPConvergedReason, 0 while iterating
  int active;      // current cycle continues
  int m;           // restart length
  int maxit;
  double rtol, atol, dtol;
  double rnorm0, ttol;
  double res;      // current residual-norm estimate
  double tt;       // norm of the newest Krylov vector
  double v0scale;  // 1/res for V_0 (kept for diagnostics; sigma[0] holds the scale)
  unsigned int counter;
};

struct GmresArrays {
  double *sigma;   // m+1: basis vector k is sigma[k] * V_k (the stored vectors are not normalised)
  double *H;       // (m+1) x m, column-major, see hidx()
  double *cs, *sn; // m
  double *grs;     // m+1
  double *y;       // m
  double *partial; // scratch for reductions: (m+1) * ntiles doubles
  double *coef;    // m+1: H(k, j) * sigma[k], the update coefficients of Arnoldi step j
  unsigned int *kcount;   // m/8+1 arrival counters of the multi-dot's k-groups (zero between launches)
};

__device__ __forceinline__ int ksp_converged(GmresState *s, int n_its, double rnorm)
{
  if (n_its == 0) {
    s->rnorm0 = rnorm;
    s->ttol = fmax(s->rtol * rnorm, s->atol);
  }
  if (isnan(rnorm) || isinf(rnorm)) return -9;            // KSP_DIVERGED_NANORINF
  if (rnorm <= s->ttol) return (rnorm < s->atol) ? 3 : 2; // KSP_CONVERGED_ATOL / RTOL
  if (rnorm >= s->dtol * s->rnorm0) return -4;            // KSP_DIVERGED_DTOL
  return 0;
}

// Block-level sum (fixed tree); result valid in thread 0.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NT / 32; k++) r += sh[k];
  }
  __syncthreads();
  return r;
}

// Returns true in exactly one CTA (the last to arrive), after all CTAs'
// partials are visible.
__device__ __forceinline__ bool last_block(unsigned int *counter, unsigned int nblocks)
{
  __shared__ bool amlast;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int t = atomicAdd(counter, 1u);
    amlast = (t == nblocks - 1);
  }
  __syncthreads();
  if (amlast) {
    __threadfence();
    if (threadIdx.x == 0) *counter = 0u;
  }
  return amlast;
}

// ---------------------------------------------------------------------------
// BSR SpMV, 4x4 blocks, FP64 vectors: one warp per block row; each lane loads
// two entries of a block (row q/2, columns 2(q%2), 2(q%2)+1 of block 'sub'),
// so a warp instruction reads four consecutive blocks (16-byte loads for FP64
// blocks).  MT = float gives the FP64 residual of the FP32 matrix used by the
// mixed-precision refinement.  MODE 0: y = M^-1 (A x), MODE 1: y = M^-1 (b - A x).
// PC: 0 none, 1 jacobi (dinv), 2 point-block (binv, 4x4 per node, row-major).
template <int MODE, int PC, typename MT>
__global__ void __launch_bounds__(256)
bsr4_spmv(int nrows, const int32_t *__restrict__ rowptr, const int32_t *__restrict__ colidx,
              const MT *__restrict__ val, const double *__restrict__ x, const double *__restrict__ b,
              const double *__restrict__ dinv, const double *__restrict__ binv, double *__restrict__ y,
              const GmresState *__restrict__ st, int j, const double *__restrict__ xscale,
              const int *__restrict__ active = nullptr)
{
  if (st && (!st->active || st->it != j)) return;
  if (active && !active[0]) return;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= nrows) return;
  const double xs = xscale ? xscale[0] : 1.0;
  const int sub = lane >> 3, q = lane & 7, row = q >> 1, cp = (q & 1) * 2;
  const int kb0 = rowptr[warp], kb1 = rowptr[warp + 1];
  double acc0 = 0.0, acc1 = 0.0;
  for (int kb = kb0 + sub; kb < kb1; kb += 4) {
    const int c = colidx[kb];
    double a0, a1;
    if constexpr (sizeof(MT) == 8) {
      const double2 a = *reinterpret_cast<const double2 *>(val + (int64_t)kb * 16 + row * 4 + cp);
      a0 = a.x; a1 = a.y;
    } else {
      const float2 a = *reinterpret_cast<const float2 *>(val + (int64_t)kb * 16 + row * 4 + cp);
      a0 = a.x; a1 = a.y;
    }
    const double2 xv = *reinterpret_cast<const double2 *>(x + (int64_t)c * 4 + cp);
    acc0 = fma(a0, xv.x, acc0);
    acc0 = fma(a1, xv.y, acc0);
  }
  double acc = acc0 + acc1;
  acc += __shfl_xor_sync(0xffffffffu, acc, 1);
  acc += __shfl_xor_sync(0xffffffffu, acc, 8);
  acc += __shfl_xor_sync(0xffffffffu, acc, 16);
  acc *= xs;
  // lanes 0,2,4,6 hold rows 0..3
  const int64_t r = (int64_t)warp * 4 + row;
  double v = acc;
  if (MODE == 1) v = b[r] - acc;
  if (PC == 2) {
    const double v0 = __shfl_sync(0xffffffffu, v, 0), v1 = __shfl_sync(0xffffffffu, v, 2);
    const double v2 = __shfl_sync(0xffffffffu, v, 4), v3 = __shfl_sync(0xffffffffu, v, 6);
    if (lane < 8 && (lane & 1) == 0) {
      const double *Bi = binv + (int64_t)warp * 16 + row * 4;
      y[r] = Bi[0] * v0 + Bi[1] * v1 + Bi[2] * v2 + Bi[3] * v3;
    }
  } else if (lane < 8 && (lane & 1) == 0) {
    y[r] = (PC == 1) ? dinv[r] * v : v;
  }
}

// BSR SpMV, 4x4 FP32 blocks and FP32 vectors (inner solve of the mixed
// precision path): one warp per block row, lane = (block sub 0..7, row 0..3),
// each lane loads one 16-byte block row and the matching 16 bytes of x, so a
// warp instruction reads eight consecutive 64-byte blocks.
template <int PC>
__global__ void __launch_bounds__(256)
bsr4_spmv_f32(int nrows, const int32_t *__restrict__ rowptr, const int32_t *__restrict__ colidx,
              const float *__restrict__ val, const float *__restrict__ x, const float *__restrict__ dinv,
              const float *__restrict__ binv, float *__restrict__ y, const GmresState *__restrict__ st, int j,
              const double *__restrict__ xscale, const int *__restrict__ active = nullptr)
{
  if (st && (!st->active || st->it != j)) return;
  if (active && !active[0]) return;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= nrows) return;
  const float xs = xscale ? (float)xscale[0] : 1.f;
  const int sub = lane >> 2, row = lane & 3;
  const int kb0 = rowptr[warp], kb1 = rowptr[warp + 1];
  float acc = 0.f;
  for (int kb = kb0 + sub; kb < kb1; kb += 8) {
    const int c = colidx[kb];
    const float4 a = *reinterpret_cast<const float4 *>(val + (int64_t)kb * 16 + row * 4);
    const float4 xv = *reinterpret_cast<const float4 *>(x + (int64_t)c * 4);
    acc = fmaf(a.x, xv.x, acc);
    acc = fmaf(a.y, xv.y, acc);
    acc = fmaf(a.z, xv.z, acc);
    acc = fmaf(a.w, xv.w, acc);
  }
  acc += __shfl_xor_sync(0xffffffffu, acc, 4);
  acc += __shfl_xor_sync(0xffffffffu, acc, 8);
  acc += __shfl_xor_sync(0xffffffffu, acc, 16);
  acc *= xs;
  const int64_t r = (int64_t)warp * 4 + row;
  if (PC == 2) {
    const float v0 = __shfl_sync(0xffffffffu, acc, 0), v1 = __shfl_sync(0xffffffffu, acc, 1);
    const float v2 = __shfl_sync(0xffffffffu, acc, 2), v3 = __shfl_sync(0xffffffffu, acc, 3);
    if (lane < 4) {
      const float *Bi = binv + (int64_t)warp * 16 + row * 4;
      y[r] = Bi[0] * v0 + Bi[1] * v1 + Bi[2] * v2 + Bi[3] * v3;
    }
  } else if (lane < 4) {
    y[r] = (PC == 1) ? dinv[r] * acc : acc;
  }
}

// Generic BSR SpMV for any block size NB (used for 3x3 blocks): one thread
// per scalar row.
template <int NB, int MODE, int PC, typename VT>
__global__ void bsr_spmv_generic(int nrows, const int32_t *__restrict__ rowptr, const int32_t *__restrict__ colidx,
                                 const VT *__restrict__ val, const double *__restrict__ x, const double *__restrict__ b,
                                 const double *__restrict__ dinv, const double *__restrict__ binv,
                                 double *__restrict__ y, const GmresState *__restrict__ st, int j,
                                 const double *__restrict__ xscale, const int *__restrict__ active = nullptr)
{
  if (st && (!st->active || st->it != j)) return;
  if (active && !active[0]) return;
  const double xs = xscale ? xscale[0] : 1.0;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t node = t / NB;
  const int row = (int)(t % NB);
  if (node >= nrows) return;
  double acc = 0.0;
  for (int kb = rowptr[node]; kb < rowptr[node + 1]; kb++) {
    const int c = colidx[kb];
    const VT *a = val + (int64_t)kb * NB * NB + row * NB;
#pragma unroll
    for (int q = 0; q < NB; q++) acc = fma((double)a[q], x[(int64_t)c * NB + q], acc);
  }
  double v = (MODE == 1) ? b[t] - xs * acc : xs * acc;
  if (PC == 1) v *= dinv[t];
  if (PC == 2) {
    // point block needs the whole node: recompute the node's other rows
    double vv[NB];
#pragma unroll
    for (int rr = 0; rr < NB; rr++) {
      double s = 0.0;
      for (int kb = rowptr[node]; kb < rowptr[node + 1]; kb++) {
        const int c = colidx[kb];
        const VT *a = val + (int64_t)kb * NB * NB + rr * NB;
#pragma unroll
        for (int q = 0; q < NB; q++) s = fma((double)a[q], x[(int64_t)c * NB + q], s);
      }
      vv[rr] = (MODE == 1) ? b[node * NB + rr] - xs * s : xs * s;
    }
    double z = 0.0;
#pragma unroll
    for (int q = 0; q < NB; q++) z += binv[node * NB * NB + row * NB + q] * vv[q];
    v = z;
  }
  y[t] = v;
}

// The same for other block sizes (3x3 in 2D), FP32 blocks and vectors: one
// thread per scalar row, FP32 accumulation as in the 4x4 FP32 kernel.
template <int NB, int PC>
__global__ void bsr_spmv_generic_f32(int nrows, const int32_t *__restrict__ rowptr, const int32_t *__restrict__ colidx,
                                     const float *__restrict__ val, const float *__restrict__ x,
                                     const float *__restrict__ dinv, const float *__restrict__ binv,
                                     float *__restrict__ y, const GmresState *__restrict__ st, int j,
                                     const double *__restrict__ xscale, const int *__restrict__ active = nullptr)
{
  if (st && (!st->active || st->it != j)) return;
  if (active && !active[0]) return;
  const float xs = xscale ? (float)xscale[0] : 1.f;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t node = t / NB;
  const int row = (int)(t % NB);
  if (node >= nrows) return;
  const int kb0 = rowptr[node], kb1 = rowptr[node + 1];
  if (PC == 2) {
    float vv[NB];
#pragma unroll
    for (int rr = 0; rr < NB; rr++) {
      float s = 0.f;
      for (int kb = kb0; kb < kb1; kb++) {
        const int c = colidx[kb];
        const float *a = val + (int64_t)kb * NB * NB + rr * NB;
#pragma unroll
        for (int q = 0; q < NB; q++) s = fmaf(a[q], x[(int64_t)c * NB + q], s);
      }
      vv[rr] = xs * s;
    }
    float z = 0.f;
#pragma unroll
    for (int q = 0; q < NB; q++) z += binv[node * NB * NB + row * NB + q] * vv[q];
    y[t] = z;
    return;
  }
  float acc = 0.f;
  for (int kb = kb0; kb < kb1; kb++) {
    const int c = colidx[kb];
    const float *a = val + (int64_t)kb * NB * NB + row * NB;
#pragma unroll
    for (int q = 0; q < NB; q++) acc = fmaf(a[q], x[(int64_t)c * NB + q], acc);
  }
  acc *= xs;
  y[t] = (PC == 1) ? dinv[t] * acc : acc;
}

// z = M^-1 r (stand-alone preconditioner application)
template <int NB, typename VT, typename PT>
__global__ void pc_apply(int64_t n, int pc, const PT *__restrict__ dinv, const PT *__restrict__ binv,
                         const VT *__restrict__ r, VT *__restrict__ z)
{
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  if (pc == 2) {
    const int64_t node = t / NB;
    const int row = (int)(t % NB);
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < NB; q++) s += (double)binv[node * NB * NB + row * NB + q] * (double)r[node * NB + q];
    z[t] = (VT)s;
  } else if (pc == 1) {
    z[t] = (VT)((double)dinv[t] * (double)r[t]);
  } else {
    z[t] = r[t];
  }
}

// Scalar-diagonal inverse and point-block inverses of the assembled matrix.
template <int NB, typename VT, typename PT>
__global__ void build_jacobi(int nnode, const int32_t *__restrict__ diag_slot, const VT *__restrict__ val,
                             PT *__restrict__ dinv, PT *__restrict__ binv, int pc)
{
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= nnode) return;
  const VT *B = val + (int64_t)diag_slot[node] * NB * NB;
  if (pc == 1) {
#pragma unroll
    for (int a = 0; a < NB; a++) {
      const double d = (double)B[a * NB + a];
      dinv[(int64_t)node * NB + a] = (PT)((d != 0.0) ? 1.0 / d : 1.0);
    }
    return;
  }
  // Gauss-Jordan with partial pivoting on the NB x NB diagonal block
  double A[NB][NB], I[NB][NB];
#pragma unroll
  for (int a = 0; a < NB; a++)
#pragma unroll
    for (int c = 0; c < NB; c++) { A[a][c] = (double)B[a * NB + c]; I[a][c] = (a == c) ? 1.0 : 0.0; }
#pragma unroll
  for (int c = 0; c < NB; c++) {
    int piv = c;
#pragma unroll
    for (int r = c + 1; r < NB; r++)
      if (fabs(A[r][c]) > fabs(A[piv][c])) piv = r;
#pragma unroll
    for (int k = 0; k < NB; k++) {
      if (piv != c) {
        double t = A[c][k]; A[c][k] = A[piv][k]; A[piv][k] = t;
        t = I[c][k]; I[c][k] = I[piv][k]; I[piv][k] = t;
      }
    }
    const double p = A[c][c];
    const double d = (p != 0.0) ? 1.0 / p : 1.0;
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
#pragma unroll
  for (int a = 0; a < NB; a++)
#pragma unroll
    for (int c = 0; c < NB; c++) binv[(int64_t)node * NB * NB + a * NB + c] = (PT)I[a][c];
}

// ---------------------------------------------------------------------------
// deterministic 2-norm: out[0] = ||x||; partials in scratch
__global__ void __launch_bounds__(RED_THREADS)
norm2_kernel(int64_t n, const double *__restrict__ x, double *__restrict__ partial, unsigned int *counter,
             double *__restrict__ out)
{
  __shared__ double sh[RED_THREADS / 32];
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * RED_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * RED_THREADS)
    s = fma(x[i], x[i], s);
  s = block_sum<RED_THREADS>(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  if (last_block(counter, gridDim.x)) {
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (unsigned int k = 0; k < gridDim.x; k++) t += __ldcg(partial + k);
      out[0] = sqrt(t);
    }
  }
}

// 16-byte chunks of a Krylov vector: 2 doubles or 4 floats.  Arithmetic on
// the values is FP64 in every kernel; FP32 vectors only change the storage.
template <typename VT> struct Chunk;
template <> struct Chunk<double> {
  static constexpr int E = 2;
  static __device__ __forceinline__ void load(const double *p, double (&v)[2])
  {
    const double2 t = *reinterpret_cast<const double2 *>(p);
    v[0] = t.x; v[1] = t.y;
  }
  static __device__ __forceinline__ void store(double *p, const double (&v)[2])
  {
    *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
  }
};
template <> struct Chunk<float> {
  static constexpr int E = 4;
  static __device__ __forceinline__ void load(const float *p, double (&v)[4])
  {
    const float4 t = *reinterpret_cast<const float4 *>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  }
  static __device__ __forceinline__ void store(float *p, const double (&v)[4])
  {
    *reinterpret_cast<float4 *>(p) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
  }
};

// out[0] = <a, a - b>, out[1] = ||a - b||^2 (deterministic; partial holds
// 2 * gridDim.x doubles)
__global__ void __launch_bounds__(RED_THREADS)
minres_dots(int64_t n, const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ partial,
            unsigned int *counter, double *__restrict__ out)
{
  __shared__ double sh[RED_THREADS / 32];
  double s0 = 0.0, s1 = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * RED_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * RED_THREADS) {
    const double d = a[i] - b[i];
    s0 = fma(a[i], d, s0);
    s1 = fma(d, d, s1);
  }
  s0 = block_sum<RED_THREADS>(s0, sh);
  s1 = block_sum<RED_THREADS>(s1, sh);
  if (threadIdx.x == 0) { partial[2 * blockIdx.x] = s0; partial[2 * blockIdx.x + 1] = s1; }
  if (last_block(counter, gridDim.x)) {
    if (threadIdx.x == 0) {
      double t0 = 0.0, t1 = 0.0;
      for (unsigned int k = 0; k < gridDim.x; k++) { t0 += __ldcg(partial + 2 * k); t1 += __ldcg(partial + 2 * k + 1); }
      out[0] = t0;
      out[1] = t1;
    }
  }
}

// Gram data of two residual differences k_i = a - b_i (deterministic):
// out = [<a,k1>, <a,k2>, <k1,k1>, <k1,k2>, <k2,k2>]; partial holds 5*gridDim.x
__global__ void __launch_bounds__(RED_THREADS)
minres_dots2(int64_t n, const double *__restrict__ a, const double *__restrict__ b1, const double *__restrict__ b2,
             double *__restrict__ partial, unsigned int *counter, double *__restrict__ out)
{
  __shared__ double sh[RED_THREADS / 32];
  double s[5] = {0, 0, 0, 0, 0};
  for (int64_t i = (int64_t)blockIdx.x * RED_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * RED_THREADS) {
    const double k1 = a[i] - b1[i], k2 = a[i] - b2[i];
    s[0] = fma(a[i], k1, s[0]);
    s[1] = fma(a[i], k2, s[1]);
    s[2] = fma(k1, k1, s[2]);
    s[3] = fma(k1, k2, s[3]);
    s[4] = fma(k2, k2, s[4]);
  }
#pragma unroll
  for (int q = 0; q < 5; q++) {
    const double t = block_sum<RED_THREADS>(s[q], sh);
    if (threadIdx.x == 0) partial[5 * blockIdx.x + q] = t;
  }
  if (last_block(counter, gridDim.x)) {
    if (threadIdx.x < 5) {
      double t = 0.0;
      for (unsigned int k = 0; k < gridDim.x; k++) t += __ldcg(partial + 5 * k + threadIdx.x);
      out[threadIdx.x] = t;
    }
  }
}

// GMRES cycle start: res = ||V0||, convergence test at its, v0scale.
template <typename VT>
__global__ void __launch_bounds__(RED_THREADS)
gmres_start(int64_t n, const VT *__restrict__ v0, GmresState *st, GmresArrays ga)
{
  __shared__ double sh[RED_THREADS / 32];
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * RED_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * RED_THREADS) {
    const double v = (double)v0[i];
    s = fma(v, v, s);
  }
  s = block_sum<RED_THREADS>(s, sh);
  if (threadIdx.x == 0) ga.partial[blockIdx.x] = s;
  if (last_block(&st->counter, gridDim.x)) {
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (unsigned int k = 0; k < gridDim.x; k++) t += __ldcg(ga.partial + k);
      const double res = sqrt(t);
      st->res = res;
      st->it = 0;
      ga.grs[0] = res;
      st->v0scale = (res != 0.0) ? 1.0 / res : 0.0;
      ga.sigma[0] = (res != 0.0) ? 1.0 / res : 1.0;
      if (res == 0.0) {
        if (st->its == 0) { st->rnorm0 = 0.0; st->ttol = st->atol; }
        st->reason = 3;   // KSP_CONVERGED_ATOL: zero residual on entry
        st->active = 0;
      } else {
        st->reason = ksp_converged(st, st->its, res);
        st->active = (st->reason == 0 && st->its < st->maxit && st->m > 0) ? 1 : 0;
      }
    }
  }
}

// Hessenberg storage: column-major, leading dimension m+1: H(r, c) = H[c*(m+1) + r].
__device__ __forceinline__ int64_t hidx(int r, int c, int m) { return (int64_t)c * (m + 1) + r; }

// Krylov vectors are stored with a leading dimension ldv that is a multiple
// of 32 entries; entries n..ldv-1 stay zero, so every kernel below processes
// 16-byte chunks (Chunk<VT>::E entries) over nchunk = ldv / E.
constexpr int ORTHO_THREADS = 256;
constexpr int MDOT_KC = 8;          // basis vectors per CTA in the multi-dot

// Classical Gram-Schmidt dot products <w, V_k> for a group of MDOT_KC
// vectors per grid row: grid (ntiles, ceil((j+1)/KC)).  Every CTA stores its
// tile partial sums; the last CTA to arrive in a grid row adds that row's
// partials (one warp per k, lanes strided over the tiles, then a fixed
// shuffle tree) and stores H(k, j) = sigma_k <w, V_k> and the update
// coefficient H(k, j) sigma_k.
template <typename VT>
__global__ void __launch_bounds__(ORTHO_THREADS)
gmres_mdot(int64_t nchunk, const VT *__restrict__ V, int64_t ldv, int j, const GmresState *__restrict__ st,
           GmresArrays ga)
{
  double *__restrict__ partial = ga.partial;
  if (!st->active || st->it != j) return;
  constexpr int E = Chunk<VT>::E;
  __shared__ double sh[MDOT_KC][ORTHO_THREADS / 32];
  const int k0 = blockIdx.y * MDOT_KC;
  const int nk = min(MDOT_KC, j + 1 - k0);
  const int64_t p = (int64_t)blockIdx.x * ORTHO_THREADS + threadIdx.x;
  const VT *w = V + (int64_t)(j + 1) * ldv;
  double acc[MDOT_KC];
#pragma unroll
  for (int q = 0; q < MDOT_KC; q++) acc[q] = 0.0;
  if (p < nchunk) {
    double wv[E];
    Chunk<VT>::load(w + E * p, wv);
#pragma unroll
    for (int q = 0; q < MDOT_KC; q++) {
      if (q < nk) {
        double v[E];
        Chunk<VT>::load(V + (int64_t)(k0 + q) * ldv + E * p, v);
        double a = wv[0] * v[0];
#pragma unroll
        for (int e = 1; e < E; e++) a = fma(wv[e], v[e], a);
        acc[q] = a;
      }
    }
  }
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < MDOT_KC; q++) {
    double v = acc[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sh[q][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < nk) {
    double t = 0.0;
#pragma unroll
    for (int w2 = 0; w2 < ORTHO_THREADS / 32; w2++) t += sh[threadIdx.x][w2];
    partial[(int64_t)(k0 + threadIdx.x) * gridDim.x + blockIdx.x] = t;
  }
  if (last_block(&ga.kcount[blockIdx.y], gridDim.x)) {
    if (wid < nk) {
      const int k = k0 + wid;
      const double *pp = partial + (int64_t)k * gridDim.x;
      double t = 0.0;
      for (unsigned int b = lane; b < gridDim.x; b += 32) t += __ldcg(pp + b);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (lane == 0) {
        const double hkj = ga.sigma[k] * t;
        ga.H[hidx(k, j, st->m)] = hkj;
        ga.coef[k] = hkj * ga.sigma[k];
      }
    }
  }
}

// w -= sum_k h_k sigma_k V_k, then ||w||^2 partials.  A CTA covers
// 2*MAXPY_CHUNKS 16-byte chunks: each thread owns two chunks (lp and
// lp + MAXPY_CHUNKS, two independent load streams), its quarter of the CTA
// takes the k's congruent to 0..3 mod 4 (consecutive lanes on consecutive
// chunks), and the quarter sums are combined in a fixed order through shared
// memory.  The last CTA finishes the norm, applies the stored Givens rotations
// to column j, forms the new one and runs the convergence test
// (KSPGMRESUpdateHessenberg, KSPConvergedDefault).
constexpr int MAXPY_CHUNKS = 64;
constexpr int MAXPY_SPAN = 2 * MAXPY_CHUNKS;   // chunks per CTA
template <typename VT>
__global__ void __launch_bounds__(ORTHO_THREADS)
gmres_maxpy_norm(int64_t nchunk, VT *__restrict__ V, int64_t ldv, int j, GmresState *st, GmresArrays ga)
{
  if (!st->active || st->it != j) return;
  constexpr int E = Chunk<VT>::E;
  __shared__ double sh[ORTHO_THREADS / 32];
  __shared__ double qs[ORTHO_THREADS / MAXPY_CHUNKS][E][MAXPY_SPAN];
  const int m = st->m;
  // coefficients H(k, j) sigma_k (written by the multi-dot), read as
  // warp-uniform broadcasts inside the loop
  const double *__restrict__ hk = ga.coef;
  VT *w = V + (int64_t)(j + 1) * ldv;
  const int lp = threadIdx.x % MAXPY_CHUNKS;
  const int quarter = threadIdx.x / MAXPY_CHUNKS;
  const int64_t p0 = (int64_t)blockIdx.x * MAXPY_SPAN + lp;
  const int64_t p1 = p0 + MAXPY_CHUNKS;
  // the chunk of w this thread finishes (quarters 0 and 1), loaded early
  const int cfin = lp + (quarter & 1) * MAXPY_CHUNKS;
  const int64_t pfin = (int64_t)blockIdx.x * MAXPY_SPAN + cfin;
  double wfin[E];
  if (quarter < 2 && pfin < nchunk) Chunk<VT>::load(w + E * pfin, wfin);
  double a0[E], a1[E];
#pragma unroll
  for (int e = 0; e < E; e++) { a0[e] = 0.0; a1[e] = 0.0; }
  // nchunk is a multiple of 16 (ldv is a multiple of 32 entries), so a CTA
  // either owns both chunks of a thread or neither past the end
  if (p1 < nchunk) {
    const VT *b0 = V + E * p0;
    const VT *b1 = V + E * p1;
    int k = quarter;
    for (; k + 4 <= j; k += 8) {
      double v0[E], v1[E], u0[E], u1[E];
      const double c0 = __ldg(hk + k), c1 = __ldg(hk + k + 4);
      Chunk<VT>::load(b0 + (int64_t)k * ldv, v0);
      Chunk<VT>::load(b1 + (int64_t)k * ldv, u0);
      Chunk<VT>::load(b0 + (int64_t)(k + 4) * ldv, v1);
      Chunk<VT>::load(b1 + (int64_t)(k + 4) * ldv, u1);
#pragma unroll
      for (int e = 0; e < E; e++) {
        a0[e] = fma(c0, v0[e], a0[e]);
        a1[e] = fma(c0, u0[e], a1[e]);
        a0[e] = fma(c1, v1[e], a0[e]);
        a1[e] = fma(c1, u1[e], a1[e]);
      }
    }
    for (; k <= j; k += 4) {
      double v0[E], u0[E];
      const double c0 = __ldg(hk + k);
      Chunk<VT>::load(b0 + (int64_t)k * ldv, v0);
      Chunk<VT>::load(b1 + (int64_t)k * ldv, u0);
#pragma unroll
      for (int e = 0; e < E; e++) {
        a0[e] = fma(c0, v0[e], a0[e]);
        a1[e] = fma(c0, u0[e], a1[e]);
      }
    }
  }
#pragma unroll
  for (int e = 0; e < E; e++) {
    qs[quarter][e][lp] = a0[e];
    qs[quarter][e][lp + MAXPY_CHUNKS] = a1[e];
  }
  __syncthreads();
  double s = 0.0;
  // quarter q < 2 finishes chunk lp + q*MAXPY_CHUNKS
  if (quarter < 2) {
    const int c = cfin;
    const int64_t p = pfin;
    if (p < nchunk) {
      double a[E];
#pragma unroll
      for (int e = 0; e < E; e++) a[e] = wfin[e];
#pragma unroll
      for (int e = 0; e < E; e++) a[e] -= ((qs[0][e][c] + qs[1][e][c]) + (qs[2][e][c] + qs[3][e][c]));
      Chunk<VT>::store(w + E * p, a);
      // the norm is taken of the stored (possibly rounded) values
#pragma unroll
      for (int e = 0; e < E; e++) {
        const double v = (double)(VT)a[e];
        s = fma(v, v, s);
      }
    }
  }
  s = block_sum<ORTHO_THREADS>(s, sh);
  if (threadIdx.x == 0) ga.partial[blockIdx.x] = s;
  if (last_block(&st->counter, gridDim.x)) {
    double t = 0.0;
    for (unsigned int b = threadIdx.x; b < gridDim.x; b += ORTHO_THREADS) t += __ldcg(ga.partial + b);
    t = block_sum<ORTHO_THREADS>(t, sh);
    // stage column j of H and the stored rotations in shared memory (hk is
    // free again), so the serial rotation chain below runs from registers and
    // shared memory instead of global-memory round trips
    __shared__ double rc[1024], rs[1024], hc[1024];
    const int it = j;
    for (int q = threadIdx.x; q <= it; q += blockDim.x) hc[q] = ga.H[hidx(q, it, m)];
    for (int q = threadIdx.x; q < it; q += blockDim.x) { rc[q] = ga.cs[q]; rs[q] = ga.sn[q]; }
    __syncthreads();
    if (threadIdx.x == 0) {
      const double tt = sqrt(t);
      st->tt = tt;
      ga.sigma[it + 1] = (tt != 0.0) ? 1.0 / tt : 1.0;   // VecNormalize, applied lazily
      hc[it + 1] = tt;
      double hapbnd = fabs(tt / ga.grs[it]);
      if (hapbnd > 1.0e-30) hapbnd = 1.0e-30;
      const bool hapend = tt < hapbnd;
      // apply the previous rotations to the new column
      double a = hc[0];
      for (int q = 1; q <= it; q++) {
        const double bq = hc[q];
        hc[q - 1] = rc[q - 1] * a + rs[q - 1] * bq;
        a = rc[q - 1] * bq - rs[q - 1] * a;
      }
      hc[it] = a;
      double res;
      int reason = 0;
      if (!hapend) {
        const double bq = hc[it + 1];
        const double r = sqrt(a * a + bq * bq);
        if (r == 0.0) {
          reason = -2;   // KSP_DIVERGED_NULL
          res = st->res;
        } else {
          const double c = a / r, sn = bq / r;
          ga.cs[it] = c;
          ga.sn[it] = sn;
          ga.grs[it + 1] = -(sn * ga.grs[it]);
          ga.grs[it] = c * ga.grs[it];
          hc[it] = c * a + sn * bq;
          res = fabs(ga.grs[it + 1]);
        }
      } else {
        res = 0.0;
      }
      if (reason == 0) {
        st->it = it + 1;
        st->its = st->its + 1;
        st->res = res;
        reason = ksp_converged(st, st->its, res);
        if (hapend && reason == 0) reason = -5;   // KSP_DIVERGED_BREAKDOWN
      }
      st->reason = reason;
      st->active = (reason == 0 && st->it < m && st->its < st->maxit) ? 1 : 0;
    }
    __syncthreads();
    for (int q = threadIdx.x; q <= it + 1; q += blockDim.x) ga.H[hidx(q, it, m)] = hc[q];
  }
}

// KSPGMRESBuildSoln back substitution, column-oriented: one CTA; for k from
// the last column down, y_k = r_k / H(k,k), then r_i -= H(i,k) y_k for i < k.
__global__ void __launch_bounds__(1024) gmres_backsub(GmresState *st, GmresArrays ga)
{
  __shared__ double r[1024];
  __shared__ double yk;
  const int last = st->it - 1;
  const int m = st->m;
  if (last < 0) return;
  for (int i = threadIdx.x; i <= last; i += blockDim.x) r[i] = ga.grs[i];
  __syncthreads();
  for (int k = last; k >= 0; k--) {
    if (threadIdx.x == 0) {
      const double d = ga.H[hidx(k, k, m)];
      yk = (d != 0.0) ? r[k] / d : 0.0;
      ga.y[k] = yk;
    }
    __syncthreads();
    const double y = yk;
    for (int i = threadIdx.x; i < k; i += blockDim.x) r[i] -= ga.H[hidx(i, k, m)] * y;
    __syncthreads();
  }
}

// x += scale * sum_{k < it} y_k sigma_k V_k  (x is FP64 whatever the basis type)
template <typename VT>
__global__ void __launch_bounds__(ORTHO_THREADS)
gmres_update_x(int64_t n, double *__restrict__ x, const VT *__restrict__ V, int64_t ldv,
               const GmresState *__restrict__ st, GmresArrays ga, double scale)
{
  __shared__ double yk[1024];
  const int it = st->it;
  if (it <= 0) return;
  for (int k = threadIdx.x; k < it; k += blockDim.x) yk[k] = ga.y[k] * ga.sigma[k];
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < it; k++) s = fma(yk[k], (double)V[(int64_t)k * ldv + i], s);
    x[i] += scale * s;
  }
}

// FP32 copy of an FP64 array of any length
__global__ void k_round_to_f32(int64_t n, const double *__restrict__ a, float *__restrict__ b)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

// b32 = sigma * v (FP32): the normalised Arnoldi vector of a flexible GMRES
// step, the right-hand side of its inner solve; skipped once the cycle ended
__global__ void k_scale_v_to_f32(int64_t n, const double *__restrict__ v, const double *__restrict__ sigma,
                                 float *__restrict__ b32, const GmresState *__restrict__ st, int j)
{
  if (st && (!st->active || st->it != j)) return;
  const double s = sigma[0];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b32[i] = (float)(s * v[i]);
}

// mixed precision helpers: b32 = r64 * s (FP32), x64 += a * d64
__global__ void k_scale_to_f32(int64_t n, const double *__restrict__ r, const double *__restrict__ norm,
                               float *__restrict__ b32)
{
  const double s = (norm[0] != 0.0) ? 1.0 / norm[0] : 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b32[i] = (float)(r[i] * s);
}

__global__ void k_axpy_dev(int64_t n, const double *__restrict__ a, const double *__restrict__ d,
                           double *__restrict__ x)
{
  const double s = a[0];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] += s * d[i];
}

__global__ void gmres_init(GmresState *st, int m, int maxit, double rtol, double atol, double dtol)
{
  if (threadIdx.x || blockIdx.x) return;
  st->it = 0; st->its = 0; st->reason = 0; st->active = 0;
  st->m = m; st->maxit = maxit; st->rtol = rtol; st->atol = atol; st->dtol = dtol;
  st->rnorm0 = 0.0; st->ttol = 0.0; st->res = 0.0; st->tt = 0.0; st->v0scale = 0.0;
  st->counter = 0u;
}

}  // namespace cfdgpu
