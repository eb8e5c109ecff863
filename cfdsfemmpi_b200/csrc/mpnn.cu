// mpnn.cu -- learned Newton initial guess: a message-passing network over the
// mesh's node graph, trained on the GPU with hand-written kernels.
//
// Network (hidden width 64, 3 message-passing layers):
//   features x_i = [u_n / s_u, (u_n - u_{n-1}) / s_d, 2 X_i - 1]   (padded to 16)
//   h0 = relu(x W_e + b_e)
//   h_l = h_{l-1} + relu([h_{l-1}, mean_{j in N(i)} h_{l-1,j}] W_l + b_l),  l = 1..3
//   y  = h_3 W_d + b_d           (the first ndof columns: increment / s_t)
// N(i) is the node's neighbourhood in the BSR pattern (the node itself
// included).  Dense layers run on the tensor cores with mma.sync m16n8k16,
// BF16 operands and FP32 accumulation; activations are kept in FP32 and
// rounded to BF16 where they enter a GEMM.  Backward: the same GEMM for
// dX = dZ W^T, CUDA-core FP32 reductions with fixed per-CTA partials for
// dW = X^T dZ, and the transposed mean-aggregation as a gather (the pattern is
// symmetric).  Adam keeps FP32 master weights.  Every reduction has a fixed
// order, so training is deterministic.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/cfdgpu.h"
#include "internal.h"

namespace {

constexpr int HID = 64;
constexpr int LAYERS = 3;
constexpr int FIN = 16;     // padded input features
constexpr int FOUT = 16;    // padded output columns (first ndof used)
constexpr int ROWS_PER_CTA = 64;   // 4 warps x 16 rows

typedef __nv_bfloat16 bf16;

// parameter blocks (FP32 master), each weight stored K x NO row-major
struct PLayout {
  int We, be, W[LAYERS], b[LAYERS], Wd, bd, total;
  PLayout()
  {
    int o = 0;
    We = o; o += FIN * HID;
    be = o; o += HID;
    for (int l = 0; l < LAYERS; l++) { W[l] = o; o += 2 * HID * HID; b[l] = o; o += HID; }
    Wd = o; o += HID * FOUT;
    bd = o; o += FOUT;
    total = o;
  }
};

}  // namespace

struct cfdgpu_mpnn {
  cfdgpu::GraphView g;
  int N = 0, Npad = 0;
  PLayout L;
  // parameters
  float *P = nullptr, *G = nullptr, *Am = nullptr, *Av = nullptr;
  bf16 *Wb = nullptr;    // per weight: K x NO copy (backward) and NO x K copy (forward)
  int wb_off[2 + 2 * LAYERS + 2];
  int64_t step = 0;
  // activations
  bf16 *X = nullptr;                 // N x FIN
  float *Ze = nullptr;               // N x HID (encoder pre-activation)
  float *Hf[LAYERS + 1];             // N x HID FP32
  bf16 *Cat[LAYERS];                 // N x 2HID: [h_{l-1}, mean]
  float *Z[LAYERS];                  // N x HID pre-activation
  bf16 *H3b = nullptr;               // N x HID (decoder input)
  float *Y = nullptr;                // N x FOUT
  // backward scratch
  float *dH = nullptr, *dZ = nullptr, *dY = nullptr;
  bf16 *dZb = nullptr, *dYb = nullptr, *dMs = nullptr;
  float *dCat = nullptr;             // N x 2HID
  float *partial = nullptr;          // per-CTA weight-gradient partials
  int nchunks = 0;
  float *lossbuf = nullptr;
  // normalisation
  float in_scale[8] = {1, 1, 1, 1, 1, 1, 1, 1}, out_scale[4] = {1, 1, 1, 1};
  double3 xlo = {0.0, 0.0, 0.0}, xinv = {1.0, 1.0, 1.0};   // bounding box of the nodes: lower corner, 1 / extent
  // samples on the device: inputs (bf16 features), targets, masks
  std::vector<bf16 *> sx;
  std::vector<float *> st;
  float *mask = nullptr;             // N x FOUT, 1 on free dofs
  // the mesh graphs samples live on: [0] the graph of the handle the network
  // was created on (the one its predictions serve), then graphs of other
  // handles whose samples train the same weights (at most as many nodes);
  // g, N, mask, xlo, xinv above hold the graph in use
  struct Graph {
    cfdgpu::GraphView g;
    int N;
    float *mask;
    double3 xlo, xinv;
  };
  std::vector<Graph> graphs;
  std::vector<int> sg;               // graph of each sample
  float cond = 0.f;                  // condition input channel (e.g. a scaled Reynolds number)
  std::vector<void *> allocs;
  std::string err;
};

namespace {

template <typename T>
int dalloc(cfdgpu_mpnn *m, T **p, size_t n)
{
  void *q = nullptr;
  if (cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return CFDGPU_ENOMEM;
  cudaMemset(q, 0, std::max<size_t>(n, 1) * sizeof(T));
  m->allocs.push_back(q);
  *p = (T *)q;
  return 0;
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// C[Npad x NO] = A[Npad x K] (bf16, row-major) * W (bf16, given as Wt = NO x K
// row-major, i.e. the "col" operand of mma.sync) + bias (optional), FP32
// accumulation and FP32 output.  One warp computes 16 rows x NO columns
// (NO/8 m16n8k16 tiles per k-step of 16); 4 warps per CTA, each CTA walking
// 64-row tiles with a grid stride.  The weights are staged in shared memory
// once per CTA with rows padded to K + 8 elements, so the eight row groups of
// a fragment read fall in distinct banks (unpadded, a 256-byte row stride put
// them all in one bank: an 8-way conflict that made the kernel bound by
// shared-memory bandwidth).  Each warp copies its 16 rows of A into shared
// memory with 16-byte asynchronous copies (padded the same way) and reads its
// fragments from there: fragment loads straight from global memory touch
// eight rows per instruction and bound the kernel at L1.
template <int K, int NO>
__global__ void __launch_bounds__(128)
gemm_bf16(int Npad, const bf16 *__restrict__ A, const bf16 *__restrict__ Wt, const float *__restrict__ bias,
          float *__restrict__ C)
{
  constexpr int KP = K + 8;
  constexpr int CPR = K / 8;                    // 16-byte chunks per row of A
  static_assert(K % 8 == 0, "rows of A in 16-byte chunks");
  __shared__ __align__(16) bf16 sW[NO * KP];
  __shared__ __align__(16) bf16 sA[4][16 * KP];
  for (int i = threadIdx.x; i < NO * K / 2; i += blockDim.x) {
    const int rr = (2 * i) / K, cc = (2 * i) % K;
    *reinterpret_cast<uint32_t *>(sW + rr * KP + cc) = reinterpret_cast<const uint32_t *>(Wt)[i];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gq = lane >> 2, tq = lane & 3;
  const int ntiles = Npad / ROWS_PER_CTA;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
  const int r0 = tile * ROWS_PER_CTA + warp * 16;
  bf16 *const wa = sA[warp];
  for (int q = lane; q < 16 * CPR; q += 32) {
    const int rr = q / CPR, cc = (q % CPR) * 8;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(wa + rr * KP + cc)),
                 "l"(A + (int64_t)(r0 + rr) * K + cc)
                 : "memory");
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncwarp();
  float acc[NO / 8][4];
#pragma unroll
  for (int t = 0; t < NO / 8; t++) acc[t][0] = acc[t][1] = acc[t][2] = acc[t][3] = 0.f;
#pragma unroll
  for (int k0 = 0; k0 < K; k0 += 16) {
    uint32_t a[4];
    const bf16 *ar0 = wa + gq * KP + k0 + 2 * tq;
    const bf16 *ar1 = wa + (gq + 8) * KP + k0 + 2 * tq;
    a[0] = *reinterpret_cast<const uint32_t *>(ar0);
    a[1] = *reinterpret_cast<const uint32_t *>(ar1);
    a[2] = *reinterpret_cast<const uint32_t *>(ar0 + 8);
    a[3] = *reinterpret_cast<const uint32_t *>(ar1 + 8);
#pragma unroll
    for (int t = 0; t < NO / 8; t++) {
      const bf16 *bp = sW + (t * 8 + gq) * KP + k0 + 2 * tq;
      const uint32_t b0 = *reinterpret_cast<const uint32_t *>(bp);
      const uint32_t b1 = *reinterpret_cast<const uint32_t *>(bp + 8);
      mma_bf16(acc[t], a, b0, b1);
    }
  }
#pragma unroll
  for (int t = 0; t < NO / 8; t++) {
    const int c = t * 8 + 2 * tq;
    const float b0 = bias ? bias[c] : 0.f, b1 = bias ? bias[c + 1] : 0.f;
    float2 v0 = make_float2(acc[t][0] + b0, acc[t][1] + b1);
    float2 v1 = make_float2(acc[t][2] + b0, acc[t][3] + b1);
    *reinterpret_cast<float2 *>(C + (int64_t)(r0 + gq) * NO + c) = v0;
    *reinterpret_cast<float2 *>(C + (int64_t)(r0 + gq + 8) * NO + c) = v1;
  }
  // every lane has read its fragments before the next tile's copy lands
  __syncwarp();
  }
}

// CTAs of gemm_bf16 for Npad rows: one per 64-row tile, at most 8 per SM
inline int gemm_grid(int Npad) { return std::max(1, std::min(Npad / ROWS_PER_CTA, 148 * 8)); }

// h = relu(z) (encoder) or h = hprev + relu(z) (residual layers); writes the
// FP32 result and its BF16 copy into column block [0, HID) of the next
// layer's concatenated input (ld = 2*HID) or into a plain N x HID buffer.
__global__ void k_act(int64_t count, const float *__restrict__ z, const float *__restrict__ hprev,
                      float *__restrict__ hout, bf16 *__restrict__ bout, int ldb)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
    const float v = fmaxf(z[i], 0.f) + (hprev ? hprev[i] : 0.f);
    hout[i] = v;
    if (bout) bout[(i / HID) * ldb + (i % HID)] = __float2bfloat16(v);
  }
}

// mean over the node's neighbourhood: out[i][c] = (1/deg_i) sum_j in[j][c]
// (one warp per node, two channels per lane, neighbours in column order);
// in/out strided (ld in elements); outb receives BF16, outf is accumulated
// (FP32).  With transpose the inputs are divided by their own node's degree
// instead (the transpose of the mean on the symmetric pattern).
__global__ void k_mean_agg(int N, const int32_t *__restrict__ rowptr, const int32_t *__restrict__ colidx,
                           const bf16 *__restrict__ in, int ldi, bf16 *__restrict__ outb, int ldo,
                           const float *__restrict__ inf, float *__restrict__ outf, int transpose)
{
  const int node = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (node >= N) return;
  const int k0 = rowptr[node], k1 = rowptr[node + 1];
  float a0 = 0.f, a1 = 0.f;
  for (int k = k0; k < k1; k++) {
    const int j = colidx[k];
    float v0, v1;
    if (inf) {
      const float2 v = *reinterpret_cast<const float2 *>(inf + (int64_t)j * HID + 2 * lane);
      v0 = v.x; v1 = v.y;
    } else {
      const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162 *>(in + (int64_t)j * ldi + 2 * lane);
      v0 = __bfloat162float(v.x); v1 = __bfloat162float(v.y);
    }
    if (transpose) {
      const float s = 1.f / (float)(rowptr[j + 1] - rowptr[j]);
      v0 *= s; v1 *= s;
    }
    a0 += v0; a1 += v1;
  }
  if (!transpose) {
    const float s = 1.f / (float)(k1 - k0);
    a0 *= s; a1 *= s;
  }
  if (outb) {
    __nv_bfloat162 o;
    o.x = __float2bfloat16(a0); o.y = __float2bfloat16(a1);
    *reinterpret_cast<__nv_bfloat162 *>(outb + (int64_t)node * ldo + 2 * lane) = o;
  }
  if (outf) {
    outf[(int64_t)node * HID + 2 * lane] += a0;
    outf[(int64_t)node * HID + 2 * lane + 1] += a1;
  }
}

// input features of one sample / prediction
__global__ void k_features(int N, int ndof, int ndim, const double *__restrict__ un, const double *__restrict__ unm1,
                           const double *__restrict__ coords, float s0, float s1, float s2, float s3, float d0,
                           float d1, float d2, float d3, double3 xlo, double3 xinv, float cond,
                           bf16 *__restrict__ X)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float su[4] = {s0, s1, s2, s3}, sd[4] = {d0, d1, d2, d3};
  float f[FIN];
#pragma unroll
  for (int c = 0; c < FIN; c++) f[c] = 0.f;
  for (int c = 0; c < ndof; c++) {
    const double u = un[(int64_t)i * ndof + c], um = unm1[(int64_t)i * ndof + c];
    f[c] = (float)(u / su[c]);
    f[ndof + c] = (float)((u - um) / sd[c]);
  }
  // coordinates mapped from the mesh's bounding box to [-1, 1] (2X - 1 on the unit square / cube)
  const double lo[3] = {xlo.x, xlo.y, xlo.z}, inv[3] = {xinv.x, xinv.y, xinv.z};
  for (int c = 0; c < ndim; c++) f[2 * ndof + c] = (float)(2.0 * ((coords[(int64_t)i * ndim + c] - lo[c]) * inv[c]) - 1.0);
  // the condition channel (0 unless set)
  f[2 * ndof + ndim] = cond;
#pragma unroll
  for (int c = 0; c < FIN; c++) X[(int64_t)i * FIN + c] = __float2bfloat16(f[c]);
}

// target: the correction over linear extrapolation, u_{n+1} - 2 u_n + u_{n-1}, scaled
__global__ void k_targets(int N, int ndof, const double *__restrict__ unm1, const double *__restrict__ un,
                          const double *__restrict__ unp1, float t0, float t1, float t2, float t3,
                          float *__restrict__ T)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float ts[4] = {t0, t1, t2, t3};
  for (int c = 0; c < FOUT; c++) {
    float v = 0.f;
    if (c < ndof) {
      const int64_t k = (int64_t)i * ndof + c;
      v = (float)(((unp1[k] - un[k]) - (un[k] - unm1[k])) / ts[c]);
    }
    T[(int64_t)i * FOUT + c] = v;
  }
}

__global__ void k_mask(int N, int ndof, const uint8_t *__restrict__ fixmask, float *__restrict__ mask)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (int c = 0; c < FOUT; c++) mask[(int64_t)i * FOUT + c] = (c < ndof && !((fixmask[i] >> c) & 1u)) ? 1.f : 0.f;
}

// loss = sum mask (y - t)^2 / sum mask ; dY = 2 mask (y - t) / sum mask (BF16 copy
// for the backward GEMM).  Deterministic: per-CTA partials, then one CTA.
__global__ void k_loss(int64_t count, const float *__restrict__ y, const float *__restrict__ t,
                       const float *__restrict__ mask, float inv_cnt, float *__restrict__ dy, bf16 *__restrict__ dyb,
                       float *__restrict__ partial)
{
  __shared__ float sh[256];
  float s = 0.f;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
    const float d = (y[i] - t[i]) * mask[i];
    s += d * d;
    const float g = 2.f * d * inv_cnt;
    dy[i] = g;
    dyb[i] = __float2bfloat16(g);
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0] * inv_cnt;
}

__global__ void k_sum_partials(int n, const float *__restrict__ partial, float *__restrict__ out)
{
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    float s = 0.f;
    for (int i = 0; i < n; i++) s += partial[i];
    out[0] = s;
  }
}

// dZ = dH * (Z > 0) (FP32 and BF16)
__global__ void k_relu_back(int64_t count, const float *__restrict__ dh, const float *__restrict__ z,
                            float *__restrict__ dz, bf16 *__restrict__ dzb)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
    const float v = (z[i] > 0.f) ? dh[i] : 0.f;
    dz[i] = v;
    dzb[i] = __float2bfloat16(v);
  }
}

// weight gradient partials: part[chunk][k][o] = sum_{rows of chunk} A[r][k] dZ[r][o]
// (A bf16 with row stride lda, dZ FP32 N x NO), plus the bias partial in the
// extra row k = K.  Threads own (k, o) pairs; rows are walked in order.
template <int K, int NO>
__global__ void __launch_bounds__(256)
k_wgrad(int Npad, int rows_per_chunk, const bf16 *__restrict__ A, int lda, const float *__restrict__ dZ,
        float *__restrict__ part)
{
  constexpr int PAIRS = (K + 1) * NO;
  __shared__ float sa[32][K + 1];
  __shared__ float sz[32][NO];
  const int r_begin = blockIdx.x * rows_per_chunk;
  const int r_end = min(Npad, r_begin + rows_per_chunk);
  float acc[(PAIRS + 255) / 256];
#pragma unroll
  for (int q = 0; q < (PAIRS + 255) / 256; q++) acc[q] = 0.f;
  for (int r0 = r_begin; r0 < r_end; r0 += 32) {
    const int nr = min(32, r_end - r0);
    for (int i = threadIdx.x; i < 32 * K; i += 256) {
      const int rr = i / K, kk = i % K;
      sa[rr][kk] = (rr < nr) ? __bfloat162float(A[(int64_t)(r0 + rr) * lda + kk]) : 0.f;
    }
    for (int i = threadIdx.x; i < 32; i += 256) sa[i][K] = (i < nr) ? 1.f : 0.f;
    for (int i = threadIdx.x; i < 32 * NO; i += 256) {
      const int rr = i / NO, oo = i % NO;
      sz[rr][oo] = (rr < nr) ? dZ[(int64_t)(r0 + rr) * NO + oo] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < (PAIRS + 255) / 256; q++) {
      const int pidx = q * 256 + threadIdx.x;
      if (pidx < PAIRS) {
        const int kk = pidx / NO, oo = pidx % NO;
        float s = acc[q];
        for (int rr = 0; rr < 32; rr++) s = fmaf(sa[rr][kk], sz[rr][oo], s);
        acc[q] = s;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < (PAIRS + 255) / 256; q++) {
    const int pidx = q * 256 + threadIdx.x;
    if (pidx < PAIRS) part[(int64_t)blockIdx.x * PAIRS + pidx] = acc[q];
  }
}

// sum the chunk partials in order into the gradient blocks (W then bias)
__global__ void k_wgrad_reduce(int nchunks, int K, int NO, const float *__restrict__ part, float *__restrict__ gW,
                               float *__restrict__ gb)
{
  const int pidx = blockIdx.x * blockDim.x + threadIdx.x;
  const int PAIRS = (K + 1) * NO;
  if (pidx >= PAIRS) return;
  float s = 0.f;
  for (int c = 0; c < nchunks; c++) s += part[(int64_t)c * PAIRS + pidx];
  const int kk = pidx / NO, oo = pidx % NO;
  if (kk < K) gW[kk * NO + oo] = s;
  else gb[oo] = s;
}

// dH_prev = dH (residual) + dCat[:, :HID]; dM (mean part) -> scaled BF16 for the transposed aggregation
__global__ void k_split_dcat(int64_t count, const float *__restrict__ dcat, float *__restrict__ dh,
                             bf16 *__restrict__ dm)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / HID, c = i % HID;
    dh[i] += dcat[r * 2 * HID + c];
    dm[i] = __float2bfloat16(dcat[r * 2 * HID + HID + c]);
  }
}

__global__ void k_adam(int n, float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// BF16 copies of a K x NO weight: W (K x NO) and Wt (NO x K)
__global__ void k_wcopy(int K, int NO, const float *__restrict__ W, bf16 *__restrict__ Wb, bf16 *__restrict__ Wtb)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= K * NO) return;
  const int k = i / NO, o = i % NO;
  const bf16 b = __float2bfloat16(W[i]);
  Wb[i] = b;
  Wtb[o * K + k] = b;
}

// predicted increment = extrapolated increment u_n - u_{n-1} + learned correction
__global__ void k_write_delta(int N, int ndof, const float *__restrict__ y, float t0, float t1, float t2, float t3,
                              const double *__restrict__ un, const double *__restrict__ unm1,
                              const uint8_t *__restrict__ fixmask, double *__restrict__ delta)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float ts[4] = {t0, t1, t2, t3};
  for (int c = 0; c < ndof; c++) {
    const int64_t k = (int64_t)i * ndof + c;
    delta[k] = ((fixmask[i] >> c) & 1u) ? 0.0 : (un[k] - unm1[k]) + (double)y[(int64_t)i * FOUT + c] * (double)ts[c];
  }
}

inline int grid1(int64_t n, int bs = 256) { return (int)std::min<int64_t>((n + bs - 1) / bs, 148 * 32); }

// weight index helpers: block order We, W[0..2], Wd
inline void weight_shape(int w, int &K, int &NO)
{
  if (w == 0) { K = FIN; NO = HID; }
  else if (w <= LAYERS) { K = 2 * HID; NO = HID; }
  else { K = HID; NO = FOUT; }
}
inline int weight_off(const PLayout &L, int w) { return w == 0 ? L.We : (w <= LAYERS ? L.W[w - 1] : L.Wd); }
inline int bias_off(const PLayout &L, int w) { return w == 0 ? L.be : (w <= LAYERS ? L.b[w - 1] : L.bd); }

int refresh_bf16(cfdgpu_mpnn *m)
{
  for (int w = 0; w < LAYERS + 2; w++) {
    int K, NO;
    weight_shape(w, K, NO);
    k_wcopy<<<(K * NO + 255) / 256, 256, 0, m->g.stream>>>(K, NO, m->P + weight_off(m->L, w), m->Wb + m->wb_off[2 * w],
                                                             m->Wb + m->wb_off[2 * w + 1]);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : CFDGPU_ECUDA;
}

// forward pass from features X (already in m->X or a sample buffer) to Y
int forward(cfdgpu_mpnn *m, const bf16 *X)
{
  cudaStream_t s = m->g.stream;
  const int Np = m->Npad;
  const int gridg = gemm_grid(Np);
  const PLayout &L = m->L;
  const int64_t cnt = (int64_t)Np * HID;
  gemm_bf16<FIN, HID><<<gridg, 128, 0, s>>>(Np, X, m->Wb + m->wb_off[1], m->P + L.be, m->Ze);
  k_act<<<grid1(cnt), 256, 0, s>>>(cnt, m->Ze, nullptr, m->Hf[0], m->Cat[0], 2 * HID);
  for (int l = 0; l < LAYERS; l++) {
    const int aggGrid = (int)((m->N * 32LL + 255) / 256);
    k_mean_agg<<<aggGrid, 256, 0, s>>>(m->N, m->g.rowptr, m->g.colidx, m->Cat[l], 2 * HID, m->Cat[l] + HID, 2 * HID,
                                       nullptr, nullptr, 0);
    gemm_bf16<2 * HID, HID><<<gridg, 128, 0, s>>>(Np, m->Cat[l], m->Wb + m->wb_off[2 * (l + 1) + 1], m->P + L.b[l], m->Z[l]);
    bf16 *next = (l + 1 < LAYERS) ? m->Cat[l + 1] : m->H3b;
    const int ldn = (l + 1 < LAYERS) ? 2 * HID : HID;
    k_act<<<grid1(cnt), 256, 0, s>>>(cnt, m->Z[l], m->Hf[l], m->Hf[l + 1], next, ldn);
  }
  gemm_bf16<HID, FOUT><<<gridg, 128, 0, s>>>(Np, m->H3b, m->Wb + m->wb_off[2 * (LAYERS + 1) + 1], m->P + L.bd, m->Y);
  return cudaGetLastError() == cudaSuccess ? 0 : CFDGPU_ECUDA;
}

int wgrad(cfdgpu_mpnn *m, int w, const bf16 *A, int lda, const float *dZ)
{
  cudaStream_t s = m->g.stream;
  int K, NO;
  weight_shape(w, K, NO);
  const int rpc = m->Npad / m->nchunks;
  if (w == 0) k_wgrad<FIN, HID><<<m->nchunks, 256, 0, s>>>(m->Npad, rpc, A, lda, dZ, m->partial);
  else if (w <= LAYERS) k_wgrad<2 * HID, HID><<<m->nchunks, 256, 0, s>>>(m->Npad, rpc, A, lda, dZ, m->partial);
  else k_wgrad<HID, FOUT><<<m->nchunks, 256, 0, s>>>(m->Npad, rpc, A, lda, dZ, m->partial);
  const int pairs = (K + 1) * NO;
  k_wgrad_reduce<<<(pairs + 255) / 256, 256, 0, s>>>(m->nchunks, K, NO, m->partial, m->G + weight_off(m->L, w),
                                                     m->G + bias_off(m->L, w));
  return cudaGetLastError() == cudaSuccess ? 0 : CFDGPU_ECUDA;
}

// loss and full backward pass for targets T; gradients into m->G, loss into loss_dev
int backward(cfdgpu_mpnn *m, const bf16 *X, const float *T, float *loss_dev)
{
  cudaStream_t s = m->g.stream;
  const int Np = m->Npad;
  const int gridg = gemm_grid(Np);
  const int64_t cnt = (int64_t)Np * HID;
  const int64_t ycnt = (int64_t)Np * FOUT;
  const float inv_cnt = 1.f / (float)std::max(1, m->g.nfree);
  const int lblocks = 148;
  k_loss<<<lblocks, 256, 0, s>>>(ycnt, m->Y, T, m->mask, inv_cnt, m->dY, m->dYb, m->lossbuf + 1);
  k_sum_partials<<<1, 32, 0, s>>>(lblocks, m->lossbuf + 1, loss_dev);
  int rc;
  if ((rc = wgrad(m, LAYERS + 1, m->H3b, HID, m->dY))) return rc;
  // dH = dY Wd^T  (Wd stored K x NO = 64 x 16 is the NO' x K' operand here)
  gemm_bf16<FOUT, HID><<<gridg, 128, 0, s>>>(Np, m->dYb, m->Wb + m->wb_off[2 * (LAYERS + 1)], nullptr, m->dH);
  for (int l = LAYERS - 1; l >= 0; l--) {
    k_relu_back<<<grid1(cnt), 256, 0, s>>>(cnt, m->dH, m->Z[l], m->dZ, m->dZb);
    if ((rc = wgrad(m, l + 1, m->Cat[l], 2 * HID, m->dZ))) return rc;
    // dCat = dZ W_l^T  (W_l stored K x NO = 128 x 64)
    gemm_bf16<HID, 2 * HID><<<gridg, 128, 0, s>>>(Np, m->dZb, m->Wb + m->wb_off[2 * (l + 1)], nullptr, m->dCat);
    k_split_dcat<<<grid1(cnt), 256, 0, s>>>(cnt, m->dCat, m->dH, m->dMs);
    const int aggGrid = (int)((m->N * 32LL + 255) / 256);
    k_mean_agg<<<aggGrid, 256, 0, s>>>(m->N, m->g.rowptr, m->g.colidx, m->dMs, HID, nullptr, 0, nullptr, m->dH, 1);
  }
  k_relu_back<<<grid1(cnt), 256, 0, s>>>(cnt, m->dH, m->Ze, m->dZ, m->dZb);
  if ((rc = wgrad(m, 0, X, FIN, m->dZ))) return rc;
  return cudaGetLastError() == cudaSuccess ? 0 : CFDGPU_ECUDA;
}

// make graph k the one the kernels use (the creator's stream always)
void use_graph(cfdgpu_mpnn *m, int k)
{
  const cudaStream_t s = m->graphs[0].g.stream;
  const cfdgpu_mpnn::Graph &G = m->graphs[k];
  m->g = G.g;
  m->g.stream = s;
  m->N = G.N;
  m->mask = G.mask;
  m->xlo = G.xlo;
  m->xinv = G.xinv;
}

// bounding box of a graph's nodes (lower corner, 1 / extent per axis)
int graph_box(const cfdgpu::GraphView &g, double3 &xlo, double3 &xinv)
{
  std::vector<double> X((size_t)g.nNode * g.ndim);
  if (cudaMemcpy(X.data(), g.coords, sizeof(double) * X.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
    return CFDGPU_ECUDA;
  double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
  for (int c = 0; c < g.ndim; c++) {
    lo[c] = hi[c] = X[c];
    for (int i = 0; i < g.nNode; i++) {
      lo[c] = std::min(lo[c], X[(size_t)i * g.ndim + c]);
      hi[c] = std::max(hi[c], X[(size_t)i * g.ndim + c]);
    }
    if (!(hi[c] > lo[c])) hi[c] = lo[c] + 1.0;
  }
  xlo = make_double3(lo[0], lo[1], lo[2]);
  xinv = make_double3(1.0 / (hi[0] - lo[0]), 1.0 / (hi[1] - lo[1]), 1.0 / (hi[2] - lo[2]));
  return 0;
}

int sample_features(cfdgpu_mpnn *m, const double *d_unm1, const double *d_un, bf16 *X)
{
  const int N = m->N;
  k_features<<<(N + 255) / 256, 256, 0, m->g.stream>>>(N, m->g.ndof, m->g.ndim, d_un, d_unm1, m->g.coords,
                                                       m->in_scale[0], m->in_scale[1], m->in_scale[2],
                                                       m->in_scale[3], m->in_scale[4], m->in_scale[5],
                                                       m->in_scale[6], m->in_scale[7], m->xlo, m->xinv, m->cond, X);
  return cudaGetLastError() == cudaSuccess ? 0 : CFDGPU_ECUDA;
}

}  // namespace

namespace cfdgpu {

int mpnn_predict_increment(cfdgpu_mpnn *m, const double *u_n, const double *u_nm1, double *delta, cudaStream_t s)
{
  (void)s;
  const int N = m->N;
  int rc = sample_features(m, u_nm1, u_n, m->X);
  if (rc) return rc;
  rc = forward(m, m->X);
  if (rc) return rc;
  k_write_delta<<<(N + 255) / 256, 256, 0, m->g.stream>>>(N, m->g.ndof, m->Y, m->out_scale[0], m->out_scale[1],
                                                          m->out_scale[2], m->out_scale[3], u_n, u_nm1,
                                                          m->g.fixmask, delta);
  return cudaGetLastError() == cudaSuccess ? 0 : CFDGPU_ECUDA;
}

}  // namespace cfdgpu

// ---------------------------------------------------------------------------
// C ABI

extern "C" {

int cfdgpu_mpnn_create(cfdgpu_handle *h, uint64_t seed, cfdgpu_mpnn **out)
{
  if (!h || !out) return CFDGPU_EINVAL;
  cfdgpu_mpnn *m = new cfdgpu_mpnn();
  *out = m;
  int rc = cfdgpu::handle_graph(h, &m->g);
  if (rc) { m->err = "handle has no device graph"; return rc; }
  if (m->g.ndof > 4 || 2 * m->g.ndof + m->g.ndim > FIN) { m->err = "unsupported dofs"; return CFDGPU_EINVAL; }
  m->N = m->g.nNode;
  m->Npad = (m->N + ROWS_PER_CTA - 1) / ROWS_PER_CTA * ROWS_PER_CTA;
  const int Np = m->Npad;
  // parameters: FP32 master, gradients, Adam moments, BF16 copies
  if ((rc = dalloc(m, &m->P, m->L.total)) || (rc = dalloc(m, &m->G, m->L.total)) || (rc = dalloc(m, &m->Am, m->L.total)) ||
      (rc = dalloc(m, &m->Av, m->L.total)))
    return rc;
  int woff = 0;
  for (int w = 0; w < LAYERS + 2; w++) {
    int K, NO;
    weight_shape(w, K, NO);
    m->wb_off[2 * w] = woff; woff += K * NO;
    m->wb_off[2 * w + 1] = woff; woff += K * NO;
  }
  if ((rc = dalloc(m, &m->Wb, woff))) return rc;
  // deterministic initialisation: uniform(-a, a), a = gain * sqrt(3 / K)
  std::vector<float> p(m->L.total, 0.f);
  std::mt19937_64 gen(seed);
  std::uniform_real_distribution<float> uni(-1.f, 1.f);
  for (int w = 0; w < LAYERS + 2; w++) {
    int K, NO;
    weight_shape(w, K, NO);
    const float gain = (w == 0) ? 1.0f : (w <= LAYERS ? 0.5f : 0.05f);
    const float a = gain * std::sqrt(3.0f / K);
    for (int i = 0; i < K * NO; i++) p[weight_off(m->L, w) + i] = a * uni(gen);
  }
  cudaMemcpy(m->P, p.data(), sizeof(float) * p.size(), cudaMemcpyHostToDevice);
  if ((rc = graph_box(m->g, m->xlo, m->xinv))) {
    m->err = "coordinate copy failed";
    return rc;
  }
  // activations
  if ((rc = dalloc(m, &m->X, (size_t)Np * FIN)) || (rc = dalloc(m, &m->Ze, (size_t)Np * HID)) ||
      (rc = dalloc(m, &m->H3b, (size_t)Np * HID)) || (rc = dalloc(m, &m->Y, (size_t)Np * FOUT)))
    return rc;
  for (int l = 0; l <= LAYERS; l++)
    if ((rc = dalloc(m, &m->Hf[l], (size_t)Np * HID))) return rc;
  for (int l = 0; l < LAYERS; l++)
    if ((rc = dalloc(m, &m->Cat[l], (size_t)Np * 2 * HID)) || (rc = dalloc(m, &m->Z[l], (size_t)Np * HID))) return rc;
  if ((rc = dalloc(m, &m->dH, (size_t)Np * HID)) || (rc = dalloc(m, &m->dZ, (size_t)Np * HID)) ||
      (rc = dalloc(m, &m->dY, (size_t)Np * FOUT)) || (rc = dalloc(m, &m->dZb, (size_t)Np * HID)) ||
      (rc = dalloc(m, &m->dYb, (size_t)Np * FOUT)) || (rc = dalloc(m, &m->dMs, (size_t)Np * HID)) ||
      (rc = dalloc(m, &m->dCat, (size_t)Np * 2 * HID)) || (rc = dalloc(m, &m->mask, (size_t)Np * FOUT)) ||
      (rc = dalloc(m, &m->lossbuf, 256)))
    return rc;
  m->nchunks = std::max(1, std::min(512, Np / 256));
  while (Np % m->nchunks) m->nchunks--;
  if ((rc = dalloc(m, &m->partial, (size_t)m->nchunks * (2 * HID + 1) * HID))) return rc;
  k_mask<<<(m->N + 255) / 256, 256, 0, m->g.stream>>>(m->N, m->g.ndof, m->g.fixmask, m->mask);
  m->graphs.push_back({m->g, m->N, m->mask, m->xlo, m->xinv});
  if ((rc = refresh_bf16(m))) return rc;
  if (cudaStreamSynchronize(m->g.stream) != cudaSuccess) return CFDGPU_ECUDA;
  return 0;
}

int cfdgpu_mpnn_destroy(cfdgpu_mpnn *m)
{
  if (!m) return 0;
  if (m->g.stream) cudaStreamSynchronize(m->g.stream);
  for (void *p : m->allocs) cudaFree(p);
  delete m;
  return 0;
}

int cfdgpu_mpnn_num_params(cfdgpu_mpnn *m) { return m ? m->L.total : CFDGPU_EINVAL; }

int cfdgpu_mpnn_get_params(cfdgpu_mpnn *m, float *p)
{
  if (!m || !p) return CFDGPU_EINVAL;
  if (cudaMemcpyAsync(p, m->P, sizeof(float) * m->L.total, cudaMemcpyDeviceToHost, m->g.stream) != cudaSuccess)
    return CFDGPU_ECUDA;
  return cudaStreamSynchronize(m->g.stream) == cudaSuccess ? 0 : CFDGPU_ECUDA;
}

int cfdgpu_mpnn_set_params(cfdgpu_mpnn *m, const float *p)
{
  if (!m || !p) return CFDGPU_EINVAL;
  if (cudaMemcpyAsync(m->P, p, sizeof(float) * m->L.total, cudaMemcpyHostToDevice, m->g.stream) != cudaSuccess)
    return CFDGPU_ECUDA;
  int rc = refresh_bf16(m);
  if (rc) return rc;
  return cudaStreamSynchronize(m->g.stream) == cudaSuccess ? 0 : CFDGPU_ECUDA;
}

int cfdgpu_mpnn_set_scales(cfdgpu_mpnn *m, const float *in_scale, const float *out_scale)
{
  if (!m || !in_scale || !out_scale) return CFDGPU_EINVAL;
  const int nd = m->g.ndof;
  for (int c = 0; c < 4; c++) {
    m->in_scale[c] = (c < nd && in_scale[c] > 0.f) ? in_scale[c] : 1.f;
    m->in_scale[4 + c] = (c < nd && in_scale[nd + c] > 0.f) ? in_scale[nd + c] : 1.f;
    m->out_scale[c] = (c < nd && out_scale[c] > 0.f) ? out_scale[c] : 1.f;
  }
  return 0;
}

int cfdgpu_mpnn_add_sample(cfdgpu_mpnn *m, const double *u_nm1, const double *u_n, const double *u_np1)
{
  if (!m || !u_nm1 || !u_n || !u_np1) return CFDGPU_EINVAL;
  const int64_t n = (int64_t)m->N * m->g.ndof;
  bf16 *X = nullptr;
  float *T = nullptr;
  double *tmp = nullptr;
  int rc;
  if ((rc = dalloc(m, &X, (size_t)m->Npad * FIN)) || (rc = dalloc(m, &T, (size_t)m->Npad * FOUT))) return rc;
  if (cudaMalloc(&tmp, sizeof(double) * 3 * n) != cudaSuccess) return CFDGPU_ENOMEM;
  cudaMemcpyAsync(tmp, u_nm1, sizeof(double) * n, cudaMemcpyHostToDevice, m->g.stream);
  cudaMemcpyAsync(tmp + n, u_n, sizeof(double) * n, cudaMemcpyHostToDevice, m->g.stream);
  cudaMemcpyAsync(tmp + 2 * n, u_np1, sizeof(double) * n, cudaMemcpyHostToDevice, m->g.stream);
  rc = sample_features(m, tmp, tmp + n, X);
  k_targets<<<(m->N + 255) / 256, 256, 0, m->g.stream>>>(m->N, m->g.ndof, tmp, tmp + n, tmp + 2 * n,
                                                         m->out_scale[0], m->out_scale[1], m->out_scale[2],
                                                         m->out_scale[3], T);
  cudaStreamSynchronize(m->g.stream);
  cudaFree(tmp);
  if (rc || cudaGetLastError() != cudaSuccess) return CFDGPU_ECUDA;
  m->sx.push_back(X);
  m->st.push_back(T);
  m->sg.push_back(0);
  return 0;
}

int cfdgpu_mpnn_set_condition(cfdgpu_mpnn *m, double cond)
{
  if (!m || !std::isfinite(cond)) return CFDGPU_EINVAL;
  m->cond = (float)cond;
  return 0;
}

int cfdgpu_mpnn_add_sample_on(cfdgpu_mpnn *m, cfdgpu_handle *h, double cond, const double *u_nm1, const double *u_n,
                              const double *u_np1)
{
  if (!m || !h || !u_nm1 || !u_n || !u_np1 || !std::isfinite(cond)) return CFDGPU_EINVAL;
  cfdgpu::GraphView gv;
  int rc = cfdgpu::handle_graph(h, &gv);
  if (rc) return rc;
  const cfdgpu_mpnn::Graph &G0 = m->graphs[0];
  if (gv.ndof != G0.g.ndof || gv.ndim != G0.g.ndim || gv.nNode > G0.N) {
    m->err = "sample graph: other dof count, dimension, or more nodes than the network's own graph";
    return CFDGPU_EINVAL;
  }
  int k = -1;
  for (size_t q = 0; q < m->graphs.size(); q++)
    if (m->graphs[q].g.rowptr == gv.rowptr) k = (int)q;
  if (k < 0) {
    cfdgpu_mpnn::Graph G{gv, gv.nNode, nullptr, {}, {}};
    if ((rc = graph_box(gv, G.xlo, G.xinv))) return rc;
    if ((rc = dalloc(m, &G.mask, (size_t)m->Npad * FOUT))) return rc;
    k_mask<<<(G.N + 255) / 256, 256, 0, G0.g.stream>>>(G.N, gv.ndof, gv.fixmask, G.mask);
    m->graphs.push_back(G);
    k = (int)m->graphs.size() - 1;
  }
  // the other handle's stream may still be writing what it returns: finish it
  if (cudaStreamSynchronize(gv.stream) != cudaSuccess) return CFDGPU_ECUDA;
  const float keep = m->cond;
  use_graph(m, k);
  m->cond = (float)cond;
  rc = cfdgpu_mpnn_add_sample(m, u_nm1, u_n, u_np1);
  m->cond = keep;
  if (!rc) m->sg.back() = k;
  use_graph(m, 0);
  return rc;
}

int cfdgpu_mpnn_num_samples(cfdgpu_mpnn *m) { return m ? (int)m->sx.size() : CFDGPU_EINVAL; }

int cfdgpu_mpnn_loss_grad(cfdgpu_mpnn *m, int sample, float *loss, float *grad)
{
  if (!m || sample < 0 || sample >= (int)m->sx.size()) return CFDGPU_EINVAL;
  use_graph(m, m->sg[sample]);
  int rc = forward(m, m->sx[sample]);
  if (!rc) rc = backward(m, m->sx[sample], m->st[sample], m->lossbuf);
  use_graph(m, 0);
  if (rc) return rc;
  if (loss) cudaMemcpyAsync(loss, m->lossbuf, sizeof(float), cudaMemcpyDeviceToHost, m->g.stream);
  if (grad) cudaMemcpyAsync(grad, m->G, sizeof(float) * m->L.total, cudaMemcpyDeviceToHost, m->g.stream);
  return cudaStreamSynchronize(m->g.stream) == cudaSuccess ? 0 : CFDGPU_ECUDA;
}

int cfdgpu_mpnn_train(cfdgpu_mpnn *m, int iters, float lr, float *loss_out)
{
  if (!m || iters < 0 || m->sx.empty()) return CFDGPU_EINVAL;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const int S = (int)m->sx.size();
  for (int it = 0; it < iters; it++) {
    const int smp = (int)(m->step % S);
    use_graph(m, m->sg[smp]);
    int rc = forward(m, m->sx[smp]);
    if (!rc) rc = backward(m, m->sx[smp], m->st[smp], m->lossbuf);
    if (rc) {
      use_graph(m, 0);
      return rc;
    }
    m->step++;
    const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
    k_adam<<<(m->L.total + 255) / 256, 256, 0, m->g.stream>>>(m->L.total, m->P, m->G, m->Am, m->Av, lr, b1, b2, eps, c1, c2);
    if ((rc = refresh_bf16(m))) return rc;
  }
  use_graph(m, 0);
  if (loss_out) cudaMemcpyAsync(loss_out, m->lossbuf, sizeof(float), cudaMemcpyDeviceToHost, m->g.stream);
  return cudaStreamSynchronize(m->g.stream) == cudaSuccess ? 0 : CFDGPU_ECUDA;
}

int cfdgpu_mpnn_predict(cfdgpu_mpnn *m, const double *u_nm1, const double *u_n, double *delta)
{
  if (!m || !u_nm1 || !u_n || !delta) return CFDGPU_EINVAL;
  const int64_t n = (int64_t)m->N * m->g.ndof;
  double *tmp = nullptr;
  if (cudaMalloc(&tmp, sizeof(double) * 3 * n) != cudaSuccess) return CFDGPU_ENOMEM;
  cudaMemcpyAsync(tmp, u_nm1, sizeof(double) * n, cudaMemcpyHostToDevice, m->g.stream);
  cudaMemcpyAsync(tmp + n, u_n, sizeof(double) * n, cudaMemcpyHostToDevice, m->g.stream);
  int rc = cfdgpu::mpnn_predict_increment(m, tmp + n, tmp, tmp + 2 * n, m->g.stream);
  if (!rc) cudaMemcpyAsync(delta, tmp + 2 * n, sizeof(double) * n, cudaMemcpyDeviceToHost, m->g.stream);
  cudaStreamSynchronize(m->g.stream);
  cudaFree(tmp);
  return rc ? rc : (cudaGetLastError() == cudaSuccess ? 0 : CFDGPU_ECUDA);
}

}  // extern "C"
