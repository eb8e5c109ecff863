// cfdgpu.cu -- host side of the C ABI declared in include/cfdgpu.h.
//
// Device layout (all resident in HBM for the handle's lifetime):
//   coords   nNode*ndim FP64, conn nElem*npe int32 (element-major)
//   nodal vectors (nNode*ndof FP64, reference layout node*ndof+dof):
//     soln, solnPrev, solnPrev2..4, solnCur, solnDot, solnDotPrev, solnDotCur,
//     solnApplied, rhs, dx
//   BSR: rowptr (nNode+1), colidx (nnzb), values nnzb*ndof*ndof (row-major
//     blocks, FP64; FP32 copy in mixed mode), diag_slot per node
//   element->block slot map nElem*npe*npe int32, colour-ordered element list
//   Krylov basis (m+1) vectors, Hessenberg/Givens arrays, reduction scratch
//   block ILU(k) factors (own BSR pattern), BiCGStab work vectors
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cfdgpu.h"
#include "bcgs_kernels.cuh"
#include "element_kernels.cuh"
#include "ilu_kernels.cuh"
#include "internal.h"
#include "linalg_kernels.cuh"
#include "setup.h"

using namespace cfdgpu;

namespace {

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

}  // namespace

struct cfdgpu_handle {
  std::string err;
  int ndim = 0, npe = 0, ndof = 0, nNode = 0, nElem = 0, et = 0;
  int64_t n = 0;  // nNode*ndof
  cfdgpu_control ctrl{};
  cfdgpu_solver_opts opts{};
  Topology topo;
  double td[16] = {0};
  bool td_set = false;
  cudaStream_t stream = nullptr;
  std::vector<void *> allocs;
  int64_t launches = 0;
  double timers[5] = {0, 0, 0, 0, 0};

  // device arrays
  double *coords = nullptr;
  int32_t *conn = nullptr;
  int32_t *rowptr = nullptr, *colidx = nullptr, *slot = nullptr, *color_elems = nullptr, *diag_slot = nullptr;
  uint8_t *fixmask = nullptr;
  int32_t *dbc_index = nullptr, *fixed_dofs = nullptr, *dbc_mult = nullptr;
  double *dbc_value = nullptr;
  double *soln = nullptr, *prev = nullptr, *prev2 = nullptr, *prev3 = nullptr, *prev4 = nullptr;
  double *cur = nullptr, *dot = nullptr, *dotPrev = nullptr, *dotCur = nullptr, *applied = nullptr;
  double *rhs = nullptr, *dx = nullptr;
  double *bsr = nullptr;
  double *dinv = nullptr, *binv = nullptr;
  int m = 0;
  int64_t ldv = 0;     // Krylov vector stride (multiple of 32 entries, zero padded)
  // mixed precision: FP64 flexible GMRES outer solve on the FP64 matrix, FP32
  // BiCGStab inner solves on an FP32 copy with an FP32 preconditioner
  bool mixed = false;
  float *bsr32 = nullptr, *dinv32 = nullptr, *binv32 = nullptr, *b32 = nullptr;
  float *fval32 = nullptr, *fdinv32 = nullptr, *ptmp32 = nullptr;
  float *iR = nullptr, *iRP = nullptr, *iP = nullptr, *iV = nullptr, *iS = nullptr, *iT = nullptr;
  BcgsState *ist = nullptr;
  double *Zb = nullptr, *ones = nullptr;   // flexible GMRES: preconditioned directions, unit scales
  int inner_its = 20;
  double inner_rtol = 1e-2, refine_rtol = 1e-10;
  // Arnoldi chunks captured as CUDA graphs (per Krylov space, per chunk start)
  bool use_graphs = true;
  std::vector<cudaGraphExec_t> graphs64, graphs32;   // graphs32: flexible GMRES steps (mixed mode)
  std::vector<int64_t> glaunch64, glaunch32;
  double *V = nullptr;
  GmresState *gst = nullptr;
  GmresArrays ga{};
  double *red_partial = nullptr, *red_partial2 = nullptr;
  unsigned int *red_counter = nullptr;
  double *scalar = nullptr;          // device scalar slots
  int *negjac = nullptr;
  double *h_scalar = nullptr;        // pinned host mirror
  GmresState *h_gst = nullptr;       // pinned
  bool assembled_K = false;
  static constexpr int MAX_DEPTH = 8;
  cudaEvent_t evq[MAX_DEPTH + 1] = {};   // one per chunk in flight
  cudaEvent_t evw = nullptr;
  bool blocking = false;   // host waits sleep (cudaEventBlockingSync) instead of spinning
  int chunk = 8;           // Arnoldi steps enqueued (and replayed as one graph) between host polls
  int depth = 1;           // chunks enqueued beyond the one whose state the host waits for
  double newton_target = 1e-8;   // this step's Newton stopping residual (absolute, and relative when asked)
  // learned initial guess
  cfdgpu_mpnn *guess = nullptr;
  int guess_mode = 0;
  double *guess_delta = nullptr, *rhs_plain = nullptr, *guess_dir2 = nullptr, *guess_res1 = nullptr,
         *guess_res2 = nullptr;
  // per-kernel event timing
  bool prof = false;
  std::vector<cudaEvent_t> pev;          // pool of 2*PROF_POOL events
  std::vector<int> pkind;                // kind of each recorded pair
  std::vector<double> pbytes;            // algorithmic bytes of each recorded launch
  int pused = 0;
  int64_t prof_launches[CFDGPU_KIND_COUNT] = {};
  double prof_ms[CFDGPU_KIND_COUNT] = {};
  double prof_bytes[CFDGPU_KIND_COUNT] = {};
  // block-Jacobi ILU(k) preconditioner (pc_type CFDGPU_PC_BJACOBI_ILU)
  IluPattern ilu;
  int32_t *frow = nullptr, *fcol = nullptr, *fdiag = nullptr, *faslot = nullptr, *fumap = nullptr;
  int32_t *florder = nullptr, *fuorder = nullptr;
  int32_t *flchain = nullptr, *fuchain = nullptr, *flchord = nullptr, *fuchord = nullptr, *fperm = nullptr;
  int64_t *fuoff = nullptr;
  double *fval = nullptr, *fdinv = nullptr;
  unsigned int *iflags = nullptr;
  TriCtl *tctl = nullptr, *h_tctl = nullptr;
  double *ptmp = nullptr;          // A x before the triangular solves
  double *ybuf = nullptr;          // intermediate vector of the triangular solves (sentinel between solves)
  float *ybuf32 = nullptr;
  // BiCGStab (ksp_type CFDGPU_KSP_BCGS)
  BcgsState *bst = nullptr, *h_bst = nullptr;
  double *bR = nullptr, *bRP = nullptr, *bP = nullptr, *bV = nullptr, *bS = nullptr, *bT = nullptr;
  std::vector<cudaGraphExec_t> graphs_bcgs;
};

static const int PROF_POOL = 32768;

// flush recorded event pairs into the per-kind totals
static void prof_collect(cfdgpu_handle *h)
{
  if (!h->pused) return;
  cudaEventSynchronize(h->pev[2 * (h->pused - 1) + 1]);
  for (int i = 0; i < h->pused; i++) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, h->pev[2 * i], h->pev[2 * i + 1]) == cudaSuccess) {
      h->prof_ms[h->pkind[i]] += ms;
      h->prof_launches[h->pkind[i]] += 1;
      h->prof_bytes[h->pkind[i]] += h->pbytes[i];
    }
  }
  h->pused = 0;
}

static int prof_begin(cfdgpu_handle *h, int kind, double bytes)
{
  if (!h->prof) return -1;
  if (h->pused >= PROF_POOL) prof_collect(h);
  const int i = h->pused++;
  h->pkind[i] = kind;
  h->pbytes[i] = bytes;
  cudaEventRecord(h->pev[2 * i], h->stream);
  return i;
}

static void prof_end(cfdgpu_handle *h, int i)
{
  if (i >= 0) cudaEventRecord(h->pev[2 * i + 1], h->stream);
}

#define CK(call)                                                                   \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      h->err = std::string(#call) + ": " + cudaGetErrorString(e_);                 \
      return CFDGPU_ECUDA;                                                         \
    }                                                                              \
  } while (0)

#define LAUNCHED(h) ((h)->launches++)

static int check_launch(cfdgpu_handle *h, const char *what)
{
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    h->err = std::string(what) + ": " + cudaGetErrorString(e);
    return CFDGPU_ECUDA;
  }
  return 0;
}

template <typename T>
static int dalloc(cfdgpu_handle *h, T **p, size_t count)
{
  void *q = nullptr;
  size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess) {
    h->err = std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e);
    return CFDGPU_ENOMEM;
  }
  h->allocs.push_back(q);
  *p = (T *)q;
  return 0;
}

template <typename T>
static int upload(cfdgpu_handle *h, T **p, const T *src, size_t count)
{
  int rc = dalloc(h, p, count);
  if (rc) return rc;
  if (count) CK(cudaMemcpy(*p, src, count * sizeof(T), cudaMemcpyHostToDevice));
  return 0;
}

// SetTimeParametersFluid (src/base/UtilitiesGeneral.cpp:5-205)
static void time_params(int tis, double rho, double dt, double *td)
{
  for (int i = 0; i < 16; i++) td[i] = 0.0;
  td[0] = dt;
  double alpf, alpm, gamm;
  switch (tis) {
    case 0:
      td[1] = 1.0; td[2] = 1.0; td[3] = 1.0; td[4] = 1.0;
      break;
    case 1:
      alpf = 1.0 / (1.0 + rho); alpm = 1.0; gamm = 1.0;
      td[1] = alpm; td[2] = alpf; td[3] = alpm; td[4] = gamm;
      td[5] = alpf * dt; td[6] = alpm / gamm; td[7] = 1.0 - alpm / gamm; td[8] = 0.0;
      td[9] = 1.0 / dt; td[10] = -td[9];
      break;
    case 2:
    case 4:
      alpf = 1.0 / (1.0 + rho); alpm = 0.5 * (3.0 - rho) / (1.0 + rho); gamm = 0.5 + alpm - alpf;
      td[1] = alpm; td[2] = alpf; td[3] = alpm; td[4] = gamm;
      td[5] = alpf * dt; td[6] = alpm / gamm; td[7] = 1.0 - alpm / gamm; td[8] = alpm / gamm / dt;
      td[9] = 1.0 / gamm / dt; td[10] = -td[9]; td[15] = 1.0 - 1.0 / gamm;
      break;
    case 3:
    case 5:
    case 6:
    case 7: {
      td[1] = 1.0; td[2] = 1.0; td[3] = 1.0; td[4] = 1.0;
      td[5] = dt; td[6] = 1.0; td[7] = 0.0; td[8] = 1.0 / dt;
      if (tis == 3) { td[9] = 1.0 / dt; td[10] = -1.0 / dt; }
      if (tis == 5) { td[9] = 1.5 / dt; td[10] = -2.0 / dt; td[11] = 0.5 / dt; }
      if (tis == 6) { td[9] = (11.0 / 6.0) / dt; td[10] = -3.0 / dt; td[11] = 1.5 / dt; td[12] = -(1.0 / 3.0) / dt; }
      if (tis == 7) {
        td[9] = (25.0 / 12.0) / dt; td[10] = -4.0 / dt; td[11] = 3.0 / dt; td[12] = -(4.0 / 3.0) / dt;
        td[13] = (1.0 / 4.0) / dt;
      }
    } break;
    default:
      break;
  }
}

// ---------------------------------------------------------------------------
// small elementwise kernels

struct TdCoef {
  double c9, c10, c11, c12, c13, c15, af, am;
};

// SolutionData::updateIterStep (src/base/SolutionData.cpp:83-91)
__global__ void k_update_iter_step(int64_t n, TdCoef c, const double *__restrict__ soln,
                                   const double *__restrict__ prev, const double *__restrict__ prev2,
                                   const double *__restrict__ prev3, const double *__restrict__ prev4,
                                   const double *__restrict__ dotPrev, double *__restrict__ dot,
                                   double *__restrict__ cur, double *__restrict__ dotCur)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double s = soln[i], p = prev[i], dp = dotPrev[i];
    const double d = c.c9 * s + c.c10 * p + c.c11 * prev2[i] + c.c12 * prev3[i] + c.c13 * prev4[i] + c.c15 * dp;
    dot[i] = d;
    cur[i] = c.af * s + (1.0 - c.af) * p;
    dotCur[i] = c.am * d + (1.0 - c.am) * dp;
  }
}

// StabFEM::assignBoundaryConditions (src/base/StabFEM.cpp:391-410)
__global__ void k_apply_bc(int nDBC, const int32_t *__restrict__ idx, const double *__restrict__ val,
                           double timeFact, const double *__restrict__ soln, double *__restrict__ applied)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nDBC) applied[idx[k]] = val[k] * timeFact - soln[idx[k]];
}

// soln[d] += solnApplied[d], once per Dirichlet entry naming d (StabFEM2.cpp:719-730)
__global__ void k_dirichlet_update(int nfix, const int32_t *__restrict__ fixed, const int32_t *__restrict__ mult,
                                   const double *__restrict__ applied, double *__restrict__ soln)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nfix) return;
  const int32_t g = fixed[k];
  double s = soln[g];
  const double a = applied[g];
  for (int r = 0; r < mult[k]; r++) s += a;
  soln[g] = s;
}

// identity on the diagonal of prescribed dofs
template <typename VT>
__global__ void k_dirichlet_diag(int nfix, int ndof, const int32_t *__restrict__ fixed,
                                 const int32_t *__restrict__ diag_slot, VT *__restrict__ bsr)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nfix) return;
  const int32_t g = fixed[k];
  const int node = g / ndof, d = g % ndof;
  bsr[(int64_t)diag_slot[node] * ndof * ndof + d * ndof + d] = VT(1);
}

// FP32 copy of an FP64 array, 4 entries per thread (n4 = count / 4)
__global__ void k_round_f32(int64_t n4, const double *__restrict__ a, float *__restrict__ b)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
    const double2 u = reinterpret_cast<const double2 *>(a)[2 * i];
    const double2 v = reinterpret_cast<const double2 *>(a)[2 * i + 1];
    reinterpret_cast<float4 *>(b)[i] = make_float4((float)u.x, (float)u.y, (float)v.x, (float)v.y);
  }
}

// zero dof d of every node
__global__ void k_zero_dof(int nNode, int ndof, int d, double *__restrict__ v)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nNode; i += (int64_t)gridDim.x * blockDim.x)
    v[i * ndof + d] = 0.0;
}

// d = a - b on free dofs, 0 on prescribed ones
__global__ void k_diff_free(int nNode, int ndof, const double *__restrict__ a, const double *__restrict__ b,
                            const uint8_t *__restrict__ fixmask, double *__restrict__ d)
{
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < (int64_t)nNode * ndof;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t node = t / ndof;
    const int dof = (int)(t % ndof);
    d[t] = ((fixmask[node] >> dof) & 1u) ? 0.0 : a[t] - b[t];
  }
}

// y = a*x + b*y
__global__ void k_lincomb(int64_t n, double a, const double *__restrict__ x, double b, double *__restrict__ y)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = a * x[i] + b * y[i];
}

__global__ void k_axpy(int64_t n, double a, const double *__restrict__ x, double *__restrict__ y)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] += a * x[i];
}

// Blocks for an elementwise kernel over n entries, at most `cap`: every
// kernel launched with it loops over its range with a grid stride.
static inline int grid_for(int64_t n, int bs = 256, int cap = 148 * 16)
{
  int64_t g = (n + bs - 1) / bs;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

// ---------------------------------------------------------------------------
// element launches

template <int ET, int MODE, bool LIFT, int FORM>
static int launch_elements(cfdgpu_handle *h, const int32_t *elems, int nel, double *outK, double *outF)
{
  constexpr int GS = ElemTraits<ET>::GS;
  constexpr int GROUPS = (GS == 32) ? 4 : 8;
  const int grid = (nel + GROUPS - 1) / GROUPS;
  if (grid <= 0) return 0;
  // algorithmic bytes of one assembly (BSR written once, RHS, coordinates,
  // connectivity, three state vectors), shared evenly by the colour launches
  const double Vb = 8.0 * h->n;
  const double asm_bytes = ((MODE == MODE_RESIDUAL) ? 0.0 : 8.0 * h->topo.nnzb() * h->ndof * h->ndof) + Vb +
                           8.0 * h->nNode * h->ndim + 4.0 * h->nElem * h->npe + 3.0 * Vb;
  const int pi = prof_begin(h, MODE == MODE_RESIDUAL ? CFDGPU_KIND_ELEM_F : CFDGPU_KIND_ELEM_K,
                            asm_bytes / std::max(1, h->topo.ncolors));
  ElemParams P;
  P.rho = h->ctrl.rho; P.mu = h->ctrl.mu; P.af = h->td[2]; P.am = h->td[1]; P.acceFact = h->td[8];
  P.stab0 = h->ctrl.stab[0]; P.stab1 = h->ctrl.stab[1]; P.stab2 = h->ctrl.stab[2];
  element_kernel<ET, double, double, MODE, LIFT, GROUPS, FORM><<<grid, GS * GROUPS, 0, h->stream>>>(
      elems, nel, h->conn, h->coords, h->prev, h->cur, h->dotCur, h->applied, h->fixmask, P, h->slot, h->bsr,
      h->rhs, outK, outF, h->negjac);
  prof_end(h, pi);
  LAUNCHED(h);
  return check_launch(h, "element_kernel");
}

template <int MODE, bool LIFT, int FORM>
static int launch_elements_form(cfdgpu_handle *h, const int32_t *elems, int nel, double *outK, double *outF)
{
  switch (h->et) {
    case CFDGPU_HEX8: return launch_elements<CFDGPU_HEX8, MODE, LIFT, FORM>(h, elems, nel, outK, outF);
    case CFDGPU_TET4: return launch_elements<CFDGPU_TET4, MODE, LIFT, FORM>(h, elems, nel, outK, outF);
    case CFDGPU_QUAD4: return launch_elements<CFDGPU_QUAD4, MODE, LIFT, FORM>(h, elems, nel, outK, outF);
    default: return launch_elements<CFDGPU_TRI3, MODE, LIFT, FORM>(h, elems, nel, outK, outF);
  }
}

template <int MODE, bool LIFT>
static int launch_elements_et(cfdgpu_handle *h, const int32_t *elems, int nel, double *outK, double *outF)
{
  if (h->opts.formulation == CFDGPU_FORM_FULLY_IMPLICIT)
    return launch_elements_form<MODE, LIFT, FORM_FULLY_IMPLICIT>(h, elems, nel, outK, outF);
  return launch_elements_form<MODE, LIFT, FORM_SEMI_IMPLICIT>(h, elems, nel, outK, outF);
}

// Assembly of one Newton iteration: rhs (and the tangent when want_K),
// colour by colour (StabFEM2.cpp:658-738).
static int assemble(cfdgpu_handle *h, int iter, bool want_K)
{
  CK(cudaMemsetAsync(h->rhs, 0, sizeof(double) * h->n, h->stream));
  const Topology &t = h->topo;
  for (int c = 0; c < t.ncolors; c++) {
    const int32_t *el = h->color_elems + t.color_ptr[c];
    const int nel = t.color_ptr[c + 1] - t.color_ptr[c];
    int rc;
    if (want_K) {
      rc = (iter == 0) ? launch_elements_et<MODE_ASSEMBLE, true>(h, el, nel, nullptr, nullptr)
                       : launch_elements_et<MODE_ASSEMBLE, false>(h, el, nel, nullptr, nullptr);
    } else {
      rc = (iter == 0) ? launch_elements_et<MODE_RESIDUAL, true>(h, el, nel, nullptr, nullptr)
                       : launch_elements_et<MODE_RESIDUAL, false>(h, el, nel, nullptr, nullptr);
    }
    if (rc) return rc;
  }
  if (want_K && !t.fixed_dofs.empty()) {
    const int nfix = (int)t.fixed_dofs.size();
    k_dirichlet_diag<double><<<(nfix + 255) / 256, 256, 0, h->stream>>>(nfix, h->ndof, h->fixed_dofs, h->diag_slot, h->bsr);
    LAUNCHED(h);
    int rc = check_launch(h, "dirichlet_diag");
    if (rc) return rc;
  }
  if (want_K) {
    h->assembled_K = true;
    if (h->mixed) {
      // FP32 copy of the tangent for the inner solves
      const int64_t cnt = h->topo.nnzb() * h->ndof * h->ndof;
      k_round_to_f32<<<grid_for(cnt), 256, 0, h->stream>>>(cnt, h->bsr, h->bsr32);
      LAUNCHED(h);
      int rc = check_launch(h, "round_to_f32");
      if (rc) return rc;
    }
  }


  return 0;
}

// Persistent grid of the sync-free ILU kernels: warps in flight for `tasks`
// rows whose widest dependency level holds `width` rows.  Warps beyond what
// the levels can feed only add polling traffic: on the 115^3 cavity the
// triangular-solve pair takes 5.4 ms with 2 CTAs of 8 warps per SM against
// 9.5 ms with 4 and 14 ms with 8, and a chain of single-row levels (the
// complete factorisation of a band) needs a few dozen warps, not thousands.
static inline int ilu_grid(int64_t tasks, int64_t width)
{
  const int64_t warps = std::min<int64_t>(tasks, std::max<int64_t>(256, 2 * width));
  const int64_t ctas = (warps + ILU_WARPS - 1) / ILU_WARPS;
  return (int)std::max<int64_t>(1, std::min<int64_t>(ctas, 148 * 2));
}

static double ilu_factor_bytes(cfdgpu_handle *h)
{
  // read A and the update map once, write the factors and the inverted diagonals once
  const double bb = (double)h->ndof * h->ndof * 8.0;
  return (double)h->topo.nnzb() * bb + (double)h->ilu.nnzb() * bb + (double)h->nNode * bb +
         4.0 * (double)h->ilu.umap.size();
}

static double trsv_bytes(cfdgpu_handle *h)
{
  // both factors once (blocks + column indices), the inverted diagonals, and
  // the vector in, intermediate (written and read) and out
  const double bb = (double)h->ndof * h->ndof * 8.0, V = 8.0 * h->n;
  return (double)h->ilu.nnzb() * (bb + 4.0) + (double)h->nNode * bb + 4.0 * V;
}

// numeric block ILU of the FP32 copy (mixed mode: FP64 arithmetic, FP32 factors)
static int ilu_factor_run32(cfdgpu_handle *h)
{
  const int pi = prof_begin(h, CFDGPU_KIND_ILU, 0.5 * ilu_factor_bytes(h));
  const int grid = ilu_grid(h->nNode, h->ilu.maxw_l);
  if (h->ndof == 4)
    ilu_factor<4, float, float><<<grid, ILU_THREADS, 0, h->stream>>>(h->nNode, h->rowptr, h->faslot, h->bsr32, h->frow,
                                                                    h->fcol, h->fdiag, h->fuoff, h->fumap, h->florder, h->fperm,
                                                                    h->fval32, h->fdinv32, h->iflags, h->tctl);
  else
    ilu_factor<3, float, float><<<grid, ILU_THREADS, 0, h->stream>>>(h->nNode, h->rowptr, h->faslot, h->bsr32, h->frow,
                                                                    h->fcol, h->fdiag, h->fuoff, h->fumap, h->florder, h->fperm,
                                                                    h->fval32, h->fdinv32, h->iflags, h->tctl);
  prof_end(h, pi);
  LAUNCHED(h);
  return check_launch(h, "ilu_factor32");
}

// z = (L U)^-1 r with the FP32 factors on FP32 vectors
static int ilu_apply32(cfdgpu_handle *h, const float *r, float *z, const GmresState *st, int j, const int *active)
{
  if ((const void *)r == (const void *)z) { h->err = "ILU apply: input and output overlap"; return CFDGPU_EINVAL; }
  const int pi = prof_begin(h, CFDGPU_KIND_TRSV, 0.5 * trsv_bytes(h));
  const int nl = (int)h->ilu.lchain_order.size(), nu = (int)h->ilu.uchain_order.size();
  // every chain of a wavefront band is in flight at once: up to one warp per chain
  const int gl = ilu_grid(nl, nl), gu = ilu_grid(nu, nu);
#define TRSV32(NB)                                                                                              \
  ilu_trsv<NB, false, float, float><<<gl, ILU_THREADS, 0, h->stream>>>(nl, h->flchord, h->flchain, h->frow,       \
      h->fcol, h->fdiag, h->fval32, h->fdinv32, h->fperm, r, h->ybuf32, z, h->tctl, st, j, active);                      \
  ilu_trsv<NB, true, float, float><<<gu, ILU_THREADS, 0, h->stream>>>(nu, h->fuchord, h->fuchain, h->frow,        \
      h->fcol, h->fdiag, h->fval32, h->fdinv32, h->fperm, nullptr, h->ybuf32, z, h->tctl, st, j, active);
  if (h->ndof == 4) { TRSV32(4); } else { TRSV32(3); }
#undef TRSV32
  prof_end(h, pi);
  h->launches += 2;
  return check_launch(h, "ilu_solve32");
}

// numeric block ILU of the assembled FP64 matrix
static int ilu_factor_run(cfdgpu_handle *h)
{
  const int pi = prof_begin(h, CFDGPU_KIND_ILU, ilu_factor_bytes(h));
  const int grid = ilu_grid(h->nNode, h->ilu.maxw_l);
  if (h->ndof == 4)
    ilu_factor<4, double, double><<<grid, ILU_THREADS, 0, h->stream>>>(h->nNode, h->rowptr, h->faslot, h->bsr, h->frow,
                                                                      h->fcol, h->fdiag, h->fuoff, h->fumap, h->florder, h->fperm,
                                                                      h->fval, h->fdinv, h->iflags, h->tctl);
  else
    ilu_factor<3, double, double><<<grid, ILU_THREADS, 0, h->stream>>>(h->nNode, h->rowptr, h->faslot, h->bsr, h->frow,
                                                                      h->fcol, h->fdiag, h->fuoff, h->fumap, h->florder, h->fperm,
                                                                      h->fval, h->fdinv, h->iflags, h->tctl);
  prof_end(h, pi);
  LAUNCHED(h);
  return check_launch(h, "ilu_factor");
}

// z = (L U)^-1 r: lower solve r -> y (the handle's buffer), upper solve y -> z
static int ilu_apply(cfdgpu_handle *h, const double *r, double *z, const GmresState *st, int j, const int *active)
{
  if ((const void *)r == (const void *)z) { h->err = "ILU apply: input and output overlap"; return CFDGPU_EINVAL; }
  const int pi = prof_begin(h, CFDGPU_KIND_TRSV, trsv_bytes(h));
  const int nl = (int)h->ilu.lchain_order.size(), nu = (int)h->ilu.uchain_order.size();
  // every chain of a wavefront band is in flight at once: up to one warp per chain
  const int gl = ilu_grid(nl, nl), gu = ilu_grid(nu, nu);
#define TRSV64(NB)                                                                                                \
  ilu_trsv<NB, false, double, double><<<gl, ILU_THREADS, 0, h->stream>>>(nl, h->flchord, h->flchain, h->frow,       \
      h->fcol, h->fdiag, h->fval, h->fdinv, h->fperm, r, h->ybuf, z, h->tctl, st, j, active);                              \
  ilu_trsv<NB, true, double, double><<<gu, ILU_THREADS, 0, h->stream>>>(nu, h->fuchord, h->fuchain, h->frow,        \
      h->fcol, h->fdiag, h->fval, h->fdinv, h->fperm, nullptr, h->ybuf, z, h->tctl, st, j, active);
  if (h->ndof == 4) { TRSV64(4); } else { TRSV64(3); }
#undef TRSV64
  prof_end(h, pi);
  h->launches += 2;
  return check_launch(h, "ilu_solve");
}

// errors recorded by the ILU kernels since the last check (zero pivot in the
// factorisation, a dependency wait that ran out); clears them
static int ilu_check(cfdgpu_handle *h)
{
  if (!h->tctl) return 0;
  CK(cudaMemcpyAsync(h->h_tctl, h->tctl, sizeof(TriCtl), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  const TriCtl c = *h->h_tctl;
  if (c.error == 0) return 0;
  CK(cudaMemsetAsync(&h->tctl->error, 0, sizeof(unsigned int), h->stream));
  // a solve that stopped early leaves rows of the intermediate vector set:
  // restore the sentinel before the next solve
  if (h->ybuf) fill_sentinel_f64<<<grid_for(h->n), 256, 0, h->stream>>>(h->n, h->ybuf);
  if (h->ybuf32) fill_sentinel_f32<<<grid_for(h->n), 256, 0, h->stream>>>(h->n, h->ybuf32);
  if (c.error == ILU_ERR_ZERO_PIVOT) {
    h->err = "Zero pivot in the ILU factorisation (singular diagonal block at node " +
             std::to_string(c.zero_pivot_row) + ")";
    return CFDGPU_EKSP;
  }
  h->err = "ILU triangular solve: a dependency wait timed out";
  return CFDGPU_ECUDA;
}

static int build_pc(cfdgpu_handle *h)
{
  const int pc = h->opts.pc_type;
  if (pc == CFDGPU_PC_NONE) return 0;
  if (pc == CFDGPU_PC_BJACOBI_ILU) return h->mixed ? ilu_factor_run32(h) : ilu_factor_run(h);
  const int g = (h->nNode + 127) / 128;
  if (h->mixed && h->ndof == 4) {
    build_jacobi<4, float, float><<<g, 128, 0, h->stream>>>(h->nNode, h->diag_slot, h->bsr32, h->dinv32, h->binv32, pc);
  } else if (h->mixed) {
    build_jacobi<3, float, float><<<g, 128, 0, h->stream>>>(h->nNode, h->diag_slot, h->bsr32, h->dinv32, h->binv32, pc);
  } else if (h->ndof == 4) {
    build_jacobi<4, double, double><<<g, 128, 0, h->stream>>>(h->nNode, h->diag_slot, h->bsr, h->dinv, h->binv, pc);
  } else {
    build_jacobi<3, double, double><<<g, 128, 0, h->stream>>>(h->nNode, h->diag_slot, h->bsr, h->dinv, h->binv, pc);
  }
  LAUNCHED(h);
  return check_launch(h, "build_jacobi");
}

static double spmv_bytes(cfdgpu_handle *h, int mode, int vbytes, int mbytes, int pc)
{
  // algorithmic bytes: blocks + column indices + row pointers + x + y (+ b)
  // + the preconditioner's data
  const double V = (double)vbytes * h->n, B = (double)h->topo.nnzb(), bb = (double)h->ndof * h->ndof;
  const double pcb = (pc == 1) ? V : (pc == 2) ? (double)vbytes * bb * h->nNode : 0.0;
  return B * bb * mbytes + 4.0 * B + 4.0 * (h->nNode + 1) + 2.0 * V + (mode == 1 ? V : 0.0) + pcb;
}

// y = M^-1 (A x) (mode 0) or y = M^-1 (b - A x) (mode 1), FP64 vectors
static int spmv_pc(cfdgpu_handle *h, int mode, const double *x, const double *b, double *y, const GmresState *st, int j,
                   const double *xscale = nullptr, const int *active = nullptr)
{
  const int pc = h->opts.pc_type;
  if (pc == CFDGPU_PC_BJACOBI_ILU) {
    // y = (LU)^-1 (A x) or (LU)^-1 (b - A x): SpMV into the scratch vector, then the two solves
    h->opts.pc_type = CFDGPU_PC_NONE;
    int rc = spmv_pc(h, mode, x, b, h->ptmp, st, j, xscale, active);
    h->opts.pc_type = CFDGPU_PC_BJACOBI_ILU;
    if (rc) return rc;
    return ilu_apply(h, h->ptmp, y, st, j, active);
  }
  const int pi = prof_begin(h, CFDGPU_KIND_SPMV, spmv_bytes(h, mode, 8, 8, pc));
  if (h->ndof == 4) {
    const int grid = (int)((h->nNode * 32LL + 255) / 256);
#define SPMV4(MO, PCV)                                                                                          \
  bsr4_spmv<MO, PCV, double><<<grid, 256, 0, h->stream>>>(h->nNode, h->rowptr, h->colidx, h->bsr, x, b, h->dinv, \
                                                           h->binv, y, st, j, xscale, active)
    if (mode == 0) {
      if (pc == 0) SPMV4(0, 0); else if (pc == 1) SPMV4(0, 1); else SPMV4(0, 2);
    } else {
      if (pc == 0) SPMV4(1, 0); else if (pc == 1) SPMV4(1, 1); else SPMV4(1, 2);
    }
#undef SPMV4
  } else {
    const int grid = (int)((h->n + 255) / 256);
#define SPMV3(MO, PCV)                                                                                        \
  bsr_spmv_generic<3, MO, PCV, double><<<grid, 256, 0, h->stream>>>(h->nNode, h->rowptr, h->colidx, h->bsr, x, b, \
                                                                     h->dinv, h->binv, y, st, j, xscale, active)
    if (mode == 0) {
      if (pc == 0) SPMV3(0, 0); else if (pc == 1) SPMV3(0, 1); else SPMV3(0, 2);
    } else {
      if (pc == 0) SPMV3(1, 0); else if (pc == 1) SPMV3(1, 1); else SPMV3(1, 2);
    }
#undef SPMV3
  }
  prof_end(h, pi);
  LAUNCHED(h);
  return check_launch(h, "bsr_spmv");
}

// y = M32^-1 (A32 x), FP32 vectors (mixed-precision inner solve)
static int spmv32_pc(cfdgpu_handle *h, const float *x, float *y, const GmresState *st, int j, const double *xscale,
                     const int *active = nullptr)
{
  const int pc = h->opts.pc_type;
  if (pc == CFDGPU_PC_BJACOBI_ILU) {
    h->opts.pc_type = CFDGPU_PC_NONE;
    int rc = spmv32_pc(h, x, h->ptmp32, st, j, xscale, active);
    h->opts.pc_type = CFDGPU_PC_BJACOBI_ILU;
    if (rc) return rc;
    return ilu_apply32(h, h->ptmp32, y, st, j, active);
  }
  const int pi = prof_begin(h, CFDGPU_KIND_SPMV, spmv_bytes(h, 0, 4, 4, pc));
  if (h->ndof == 4) {
    const int grid = (int)((h->nNode * 32LL + 255) / 256);
    if (pc == 0)
      bsr4_spmv_f32<0><<<grid, 256, 0, h->stream>>>(h->nNode, h->rowptr, h->colidx, h->bsr32, x, h->dinv32, h->binv32, y, st, j, xscale, active);
    else if (pc == 1)
      bsr4_spmv_f32<1><<<grid, 256, 0, h->stream>>>(h->nNode, h->rowptr, h->colidx, h->bsr32, x, h->dinv32, h->binv32, y, st, j, xscale, active);
    else
      bsr4_spmv_f32<2><<<grid, 256, 0, h->stream>>>(h->nNode, h->rowptr, h->colidx, h->bsr32, x, h->dinv32, h->binv32, y, st, j, xscale, active);
  } else {
    const int grid = (int)((h->n + 255) / 256);
    if (pc == 0)
      bsr_spmv_generic_f32<3, 0><<<grid, 256, 0, h->stream>>>(h->nNode, h->rowptr, h->colidx, h->bsr32, x, h->dinv32, h->binv32, y, st, j, xscale, active);
    else if (pc == 1)
      bsr_spmv_generic_f32<3, 1><<<grid, 256, 0, h->stream>>>(h->nNode, h->rowptr, h->colidx, h->bsr32, x, h->dinv32, h->binv32, y, st, j, xscale, active);
    else
      bsr_spmv_generic_f32<3, 2><<<grid, 256, 0, h->stream>>>(h->nNode, h->rowptr, h->colidx, h->bsr32, x, h->dinv32, h->binv32, y, st, j, xscale, active);
  }
  prof_end(h, pi);
  LAUNCHED(h);
  return check_launch(h, "bsr_spmv_f32");
}

static int norm2_dev(cfdgpu_handle *h, const double *x, double *d_out)
{
  norm2_kernel<<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(h->n, x, h->red_partial, h->red_counter, d_out);
  LAUNCHED(h);
  return check_launch(h, "norm2");
}

// Wait on the host for everything enqueued on the handle's stream.  A handle
// driven by one of many host threads (cfdgpu_batch_*) sleeps in the wait
// instead of spinning, so that dozens of such threads can share a few cores.
static int host_wait(cfdgpu_handle *h)
{
  if (!h->blocking) {
    CK(cudaStreamSynchronize(h->stream));
    return 0;
  }
  CK(cudaEventRecord(h->evw, h->stream));
  CK(cudaEventSynchronize(h->evw));
  return 0;
}

static int norm2(cfdgpu_handle *h, const double *x, double *out_host)
{
  int rc = norm2_dev(h, x, h->scalar);
  if (rc) return rc;
  CK(cudaMemcpyAsync(h->h_scalar, h->scalar, sizeof(double) * 1, cudaMemcpyDeviceToHost, h->stream));
  if ((rc = host_wait(h))) return rc;
  *out_host = h->h_scalar[0];
  return 0;
}

// One Krylov space: basis, control block and Hessenberg arrays.
template <typename VT>
struct Krylov {
  VT *V = nullptr;
  int m = 0;
  int64_t ldv = 0;
  GmresState *st = nullptr;
  GmresArrays ga{};
  double *Z = nullptr;   // flexible GMRES: x += sum_k y_k Z_k (with gaz.sigma = 1)
  GmresArrays gaz{};
  std::vector<cudaGraphExec_t> &graphs;
  std::vector<int64_t> &graph_launches;   // kernel launches inside each cached graph
  Krylov(std::vector<cudaGraphExec_t> &g, std::vector<int64_t> &gl) : graphs(g), graph_launches(gl) {}
};

// Restarted GMRES with PETSc semantics on a Krylov space.  The caller has
// already enqueued V_0 = M^-1 b.  arnoldi(j) enqueues V_{j+1} = M^-1 A V_j;
// restart() enqueues V_0 = M^-1 (b - A x) (not called when single_cycle).
// x (FP64) is zeroed here and receives xscale * (the Krylov correction).
template <typename VT, typename Arn, typename Res>
static int gmres_run(cfdgpu_handle *h, Krylov<VT> &K, double *x, int max_it, double rtol, double atol, double dtol,
                     bool single_cycle, Arn arnoldi, Res restart, int *its_out, int *reason_out)
{
  constexpr int E = Chunk<VT>::E;
  const int64_t n = h->n;
  const int m = K.m;
  const int64_t ldv = K.ldv;
  const int64_t nchunk = ldv / E;
  const int ntiles = (int)((nchunk + ORTHO_THREADS - 1) / ORTHO_THREADS);
  const int mtiles = (int)(nchunk / MAXPY_SPAN);
  VT *V = K.V;
  GmresState *st = K.st;
  int rc;
  gmres_init<<<1, 1, 0, h->stream>>>(st, m, max_it, rtol, atol, dtol);
  LAUNCHED(h);
  CK(cudaMemsetAsync(x, 0, sizeof(double) * n, h->stream));
  const int vgrid = grid_for(n);
  // Arnoldi steps j0..j0+CH-1 enqueued as one unit: directly, or (without
  // per-kernel profiling) as a CUDA graph captured once per chunk and reused
  const int CH = h->chunk;
  auto enqueue_chunk = [&](int j0) -> int {
    for (int j = j0; j < std::min(m, j0 + CH); j++) {
      int r;
      if ((r = arnoldi(j))) return r;
      const int pi = prof_begin(h, CFDGPU_KIND_ORTHO, (2.0 * j + 3.0) * (double)sizeof(VT) * n);
      dim3 g2(ntiles, (j + 1 + MDOT_KC - 1) / MDOT_KC);
      gmres_mdot<VT><<<g2, ORTHO_THREADS, 0, h->stream>>>(nchunk, V, ldv, j, st, K.ga);
      gmres_maxpy_norm<VT><<<mtiles, ORTHO_THREADS, 0, h->stream>>>(nchunk, V, ldv, j, st, K.ga);
      prof_end(h, pi);
    }
    return check_launch(h, "gmres_arnoldi");
  };
  while (true) {
    gmres_start<VT><<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(n, V, st, K.ga);
    h->launches += 1;
    if ((rc = check_launch(h, "gmres_start"))) return rc;
    // poll the device flag `depth` chunks behind so the GPU stays fed; the
    // chunks enqueued past convergence run as no-ops
    bool stop = false;
    const int D = h->depth, R = D + 1;
    int c = 0;
    for (int j0 = 0; j0 < m && !stop; j0 += CH, c++) {
      const int nk = std::min(m, j0 + CH) - j0;
      if (h->use_graphs && !h->prof) {
        std::vector<cudaGraphExec_t> &cache = K.graphs;
        if (cache.size() < (size_t)((m + CH - 1) / CH)) {
          cache.resize((m + CH - 1) / CH, nullptr);
          K.graph_launches.resize(cache.size(), 0);
        }
        cudaGraphExec_t &ex = cache[j0 / CH];
        if (!ex) {
          cudaGraph_t g = nullptr;
          CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
          const int64_t before = h->launches;
          const int r = enqueue_chunk(j0);
          const cudaError_t ec = cudaStreamEndCapture(h->stream, &g);
          if (r) return r;
          if (ec != cudaSuccess) { h->err = std::string("graph capture: ") + cudaGetErrorString(ec); return CFDGPU_ECUDA; }
          CK(cudaGraphInstantiate(&ex, g, 0));
          CK(cudaGraphDestroy(g));
          K.graph_launches[j0 / CH] = h->launches - before + 2 * nk;
          h->launches = before;   // counted when the graph runs
        }
        CK(cudaGraphLaunch(ex, h->stream));
        h->launches += K.graph_launches[j0 / CH];
      } else {
        if ((rc = enqueue_chunk(j0))) return rc;
        h->launches += 2 * nk;
      }
      const int cidx = c % R;
      CK(cudaMemcpyAsync(&h->h_gst[cidx], st, sizeof(GmresState), cudaMemcpyDeviceToHost, h->stream));
      CK(cudaEventRecord(h->evq[cidx], h->stream));
      // wait for the snapshot taken `depth` chunks ago
      if (c >= D) {
        const int pidx = (c - D) % R;
        CK(cudaEventSynchronize(h->evq[pidx]));
        if (!h->h_gst[pidx].active) stop = true;
      }
    }
    gmres_backsub<<<1, 1024, 0, h->stream>>>(st, K.ga);
    h->launches += 1;
    if (K.Z)
      gmres_update_x<double><<<vgrid, ORTHO_THREADS, 0, h->stream>>>(n, x, K.Z, ldv, st, K.gaz, 1.0);
    else
      gmres_update_x<VT><<<vgrid, ORTHO_THREADS, 0, h->stream>>>(n, x, V, ldv, st, K.ga, 1.0);
    h->launches += 1;
    if ((rc = check_launch(h, "gmres_build_soln"))) return rc;
    GmresState *fin = h->h_gst + cfdgpu_handle::MAX_DEPTH + 1;
    CK(cudaMemcpyAsync(fin, st, sizeof(GmresState), cudaMemcpyDeviceToHost, h->stream));
    if ((rc = host_wait(h))) return rc;
    GmresState s = *fin;
    int reason = s.reason;
    if (reason == 0 && s.its >= max_it) reason = -3;   // KSP_DIVERGED_ITS
    if (reason != 0 || single_cycle) {
      if (its_out) *its_out = s.its;
      if (reason_out) *reason_out = reason;
      return 0;
    }
    rc = restart();
    if (rc != 0) return rc;
  }
}

// Restarted GMRES on the assembled FP64 BSR: x = A^-1 b, x0 = 0.
// z = M^-1 r with the handle's FP64 preconditioner
static int pc_apply_vec(cfdgpu_handle *h, const double *r, double *z, const int *active = nullptr)
{
  const int64_t n = h->n;
  if (h->opts.pc_type == CFDGPU_PC_BJACOBI_ILU) return ilu_apply(h, r, z, nullptr, 0, active);
  if (h->ndof == 4)
    pc_apply<4, double, double><<<grid_for(n, 256, 1 << 30), 256, 0, h->stream>>>(n, h->opts.pc_type, h->dinv, h->binv, r, z);
  else
    pc_apply<3, double, double><<<grid_for(n, 256, 1 << 30), 256, 0, h->stream>>>(n, h->opts.pc_type, h->dinv, h->binv, r, z);
  LAUNCHED(h);
  return check_launch(h, "pc_apply");
}

static int gmres(cfdgpu_handle *h, const double *b, double *x, int *its_out, int *reason_out)
{
  int rc0 = pc_apply_vec(h, b, h->V);
  if (rc0) return rc0;
  Krylov<double> K(h->graphs64, h->glaunch64);
  K.V = h->V; K.m = h->m; K.ldv = h->ldv; K.st = h->gst; K.ga = h->ga;
  auto arn = [&](int j) {
    return spmv_pc(h, 0, h->V + (int64_t)j * h->ldv, nullptr, h->V + (int64_t)(j + 1) * h->ldv, h->gst, j, h->ga.sigma + j);
  };
  auto res = [&]() { return spmv_pc(h, 1, x, b, h->V, nullptr, 0, nullptr); };
  return gmres_run<double>(h, K, x, h->opts.max_it, h->opts.rtol, h->opts.atol, h->opts.dtol, false, arn, res,
                           its_out, reason_out);
}

// BiCGStab (PETSc KSPBCGS semantics, left preconditioning, x0 = 0) on the
// assembled FP64 BSR: x = A^-1 b.  Iterations are enqueued in chunks of
// h->chunk / 2 (captured once as a CUDA graph and replayed: every iteration
// runs the same kernels on the same buffers), and the host polls the device
// control block `depth` chunks behind; iterations after the solve has ended
// return at once.
static int bcgs(cfdgpu_handle *h, const double *b, double *x, int *its_out, int *reason_out)
{
  const int64_t n = h->n;
  int rc;
  BcgsState *st = h->bst;
  const int *act = &st->active;
  bcgs_setup<<<1, 1, 0, h->stream>>>(st, h->opts.max_it, h->opts.rtol, h->opts.atol, h->opts.dtol);
  LAUNCHED(h);
  CK(cudaMemsetAsync(x, 0, sizeof(double) * n, h->stream));
  if ((rc = pc_apply_vec(h, b, h->bR))) return rc;
  bcgs_init<double><<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(n, h->bR, h->bRP, h->bP, h->bV, st, h->red_partial2);
  LAUNCHED(h);
  if ((rc = check_launch(h, "bcgs_init"))) return rc;
  const int vgrid = grid_for(n);
  const double V = 8.0 * n;
  auto iteration = [&]() -> int {
    int r;
    int pi = prof_begin(h, CFDGPU_KIND_BCGS, 4.0 * V);
    bcgs_p<double><<<vgrid, 256, 0, h->stream>>>(n, h->bR, h->bV, h->bP, st);
    prof_end(h, pi);
    if ((r = spmv_pc(h, 0, h->bP, nullptr, h->bV, nullptr, 0, nullptr, act))) return r;
    pi = prof_begin(h, CFDGPU_KIND_BCGS, 5.0 * V);
    bcgs_alpha<double><<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(n, h->bV, h->bRP, st, h->red_partial2);
    bcgs_s<double><<<vgrid, 256, 0, h->stream>>>(n, h->bR, h->bV, h->bS, st);
    prof_end(h, pi);
    if ((r = spmv_pc(h, 0, h->bS, nullptr, h->bT, nullptr, 0, nullptr, act))) return r;
    pi = prof_begin(h, CFDGPU_KIND_BCGS, 10.0 * V);
    bcgs_omega<double><<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(n, h->bS, h->bT, st, h->red_partial2);
    bcgs_xr<double><<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(n, x, h->bP, h->bS, h->bT, h->bR, h->bRP, st,
                                                              h->red_partial2);
    prof_end(h, pi);
    h->launches += 5;
    return check_launch(h, "bcgs_iteration");
  };
  const int CH = std::max(1, h->chunk / 2);
  const int D = h->depth, R = D + 1;
  const int64_t max_chunks = (int64_t)h->opts.max_it / CH + D + 2;
  bool stop = false;
  for (int64_t c = 0; c < max_chunks && !stop; c++) {
    if (h->use_graphs && !h->prof) {
      if (h->graphs_bcgs.empty()) h->graphs_bcgs.resize(1, nullptr);
      cudaGraphExec_t &ex = h->graphs_bcgs[0];
      if (!ex) {
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        const int64_t before = h->launches;
        int r = 0;
        for (int k = 0; k < CH && !r; k++) r = iteration();
        const cudaError_t ec = cudaStreamEndCapture(h->stream, &g);
        if (r) return r;
        if (ec != cudaSuccess) { h->err = std::string("graph capture: ") + cudaGetErrorString(ec); return CFDGPU_ECUDA; }
        CK(cudaGraphInstantiate(&ex, g, 0));
        CK(cudaGraphDestroy(g));
        h->launches = before;
      }
      CK(cudaGraphLaunch(ex, h->stream));
      const int per_it = (h->opts.pc_type == CFDGPU_PC_BJACOBI_ILU) ? 11 : 7;
      h->launches += (int64_t)CH * per_it;
    } else {
      for (int k = 0; k < CH; k++)
        if ((rc = iteration())) return rc;
    }
    const int cidx = (int)(c % R);
    CK(cudaMemcpyAsync(&h->h_bst[cidx], st, sizeof(BcgsState), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaEventRecord(h->evq[cidx], h->stream));
    if (c >= D) {
      const int pidx = (int)((c - D) % R);
      CK(cudaEventSynchronize(h->evq[pidx]));
      if (!h->h_bst[pidx].active) stop = true;
    }
  }
  BcgsState *fin = h->h_bst + cfdgpu_handle::MAX_DEPTH + 1;
  CK(cudaMemcpyAsync(fin, st, sizeof(BcgsState), cudaMemcpyDeviceToHost, h->stream));
  if ((rc = host_wait(h))) return rc;
  if ((rc = ilu_check(h))) return rc;
  int reason = fin->reason;
  if (reason == 0) reason = -3;   // the chunk cap ended the loop (maxit normally ends the solve first)
  if (its_out) *its_out = fin->its;
  if (reason_out) *reason_out = reason;
  return 0;
}

// Linear solve of the FP64 system with the handle's Krylov method
static int krylov_solve(cfdgpu_handle *h, const double *b, double *x, int *its, int *reason)
{
  int rc;
  if (h->opts.ksp_type == CFDGPU_KSP_BCGS) {
    rc = bcgs(h, b, x, its, reason);
  } else if (h->opts.ksp_type == CFDGPU_KSP_PREONLY) {
    // KSPSolve_PREONLY: one application of the preconditioner
    rc = pc_apply_vec(h, b, x);
    if (!rc) rc = host_wait(h);
    if (!rc) rc = ilu_check(h);
    if (its) *its = 1;
    if (reason) *reason = 4;   // KSP_CONVERGED_ITS
  } else {
    rc = gmres(h, b, x, its, reason);
    if (!rc) rc = ilu_check(h);
  }
  return rc;
}

// z32 = M32^-1 r32 (FP32 preconditioner of the inner solves)
static int pc32_apply_vec(cfdgpu_handle *h, const float *r, float *z, const GmresState *st, int j)
{
  const int64_t n = h->n;
  if (h->opts.pc_type == CFDGPU_PC_BJACOBI_ILU) return ilu_apply32(h, r, z, st, j, nullptr);
  if (h->ndof == 4)
    pc_apply<4, float, float><<<grid_for(n, 256, 1 << 30), 256, 0, h->stream>>>(n, h->opts.pc_type, h->dinv32, h->binv32, r, z);
  else
    pc_apply<3, float, float><<<grid_for(n, 256, 1 << 30), 256, 0, h->stream>>>(n, h->opts.pc_type, h->dinv32, h->binv32, r, z);
  LAUNCHED(h);
  return check_launch(h, "pc32_apply");
}

// Inner solve of flexible GMRES step j (mixed mode): z = (FP32 BiCGStab with
// the FP32 preconditioner, at most inner_its iterations or inner_rtol) applied
// to the normalised Arnoldi vector sigma_j V_j; z accumulates in FP64.  Every
// kernel is skipped once the outer cycle has ended, so whole outer steps can
// be enqueued (and captured) without host round trips.
static int inner_bcgs32(cfdgpu_handle *h, const double *vj, const double *sigma_j, double *z, const GmresState *ost,
                        int j)
{
  const int64_t n = h->n;
  int rc;
  BcgsState *st = h->ist;
  const int *act = &st->active;
  k_scale_v_to_f32<<<grid_for(n), 256, 0, h->stream>>>(n, vj, sigma_j, h->b32, ost, j);
  bcgs_setup<<<1, 1, 0, h->stream>>>(st, h->inner_its, h->inner_rtol, 1e-50, 1e30, ost, j);
  h->launches += 2;
  CK(cudaMemsetAsync(z, 0, sizeof(double) * n, h->stream));
  if ((rc = pc32_apply_vec(h, h->b32, h->iR, ost, j))) return rc;
  bcgs_init<float><<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(n, h->iR, h->iRP, h->iP, h->iV, st, h->red_partial2);
  LAUNCHED(h);
  const int vgrid = grid_for(n);
  for (int k = 0; k < h->inner_its; k++) {
    bcgs_p<float><<<vgrid, 256, 0, h->stream>>>(n, h->iR, h->iV, h->iP, st);
    if ((rc = spmv32_pc(h, h->iP, h->iV, nullptr, 0, nullptr, act))) return rc;
    bcgs_alpha<float><<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(n, h->iV, h->iRP, st, h->red_partial2);
    bcgs_s<float><<<vgrid, 256, 0, h->stream>>>(n, h->iR, h->iV, h->iS, st);
    if ((rc = spmv32_pc(h, h->iS, h->iT, nullptr, 0, nullptr, act))) return rc;
    bcgs_omega<float><<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(n, h->iS, h->iT, st, h->red_partial2);
    bcgs_xr<float><<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(n, z, h->iP, h->iS, h->iT, h->iR, h->iRP, st,
                                                             h->red_partial2);
    h->launches += 5;
  }
  return check_launch(h, "inner_bcgs32");
}

// y = A x (mode 0) or b - A x (mode 1) with the FP64 matrix, no preconditioner
static int spmv64_plain(cfdgpu_handle *h, int mode, const double *x, const double *b, double *y,
                        const GmresState *st, int j)
{
  const int saved = h->opts.pc_type;
  h->opts.pc_type = CFDGPU_PC_NONE;
  const int rc = spmv_pc(h, mode, x, b, y, st, j, nullptr, nullptr);
  h->opts.pc_type = saved;
  return rc;
}

// Mixed precision linear solve: flexible GMRES (right preconditioning, FP64
// basis, Hessenberg, Givens rotations and residual on the FP64 matrix) whose
// preconditioner is the FP32 inner solve above, x0 = 0.  The residual
// estimate is the true residual ||b - A x||; the solve stops at
// max(refine_rtol ||b||, F), F = refine_atol when set (none when negative),
// else T/10 with T the step's Newton stopping residual.  The Newton loop's
// FP64 residual test (element kernels in FP64) decides whether the step has
// converged.
static int fgmres_mixed(cfdgpu_handle *h, const double *b, double *x, int *its_out, int *reason_out)
{
  const int64_t n = h->n;
  CK(cudaMemcpyAsync(h->V, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream));
  Krylov<double> K(h->graphs32, h->glaunch32);
  K.V = h->V; K.m = h->m; K.ldv = h->ldv; K.st = h->gst; K.ga = h->ga;
  K.Z = h->Zb;
  K.gaz = h->ga;
  K.gaz.sigma = h->ones;
  auto arn = [&](int j) {
    int rc = inner_bcgs32(h, h->V + (int64_t)j * h->ldv, h->ga.sigma + j, h->Zb + (int64_t)j * h->ldv, h->gst, j);
    if (rc) return rc;
    return spmv64_plain(h, 0, h->Zb + (int64_t)j * h->ldv, nullptr, h->V + (int64_t)(j + 1) * h->ldv, h->gst, j);
  };
  auto res = [&]() { return spmv64_plain(h, 1, x, b, h->V, nullptr, 0); };
  const double floor = (h->opts.refine_atol > 0.0) ? h->opts.refine_atol
                       : (h->opts.refine_atol < 0.0) ? 0.0 : 0.1 * h->newton_target;
  return gmres_run<double>(h, K, x, h->opts.max_it, h->refine_rtol, floor, h->opts.dtol, false, arn, res, its_out,
                           reason_out);
}

static int upload_td(cfdgpu_handle *h)
{
  time_params(h->ctrl.tis, h->ctrl.rhoInf, h->ctrl.dt, h->td);
  h->td_set = true;
  return 0;
}

static int update_iter_step(cfdgpu_handle *h)
{
  TdCoef c{h->td[9], h->td[10], h->td[11], h->td[12], h->td[13], h->td[15], h->td[2], h->td[1]};
  k_update_iter_step<<<grid_for(h->n), 256, 0, h->stream>>>(h->n, c, h->soln, h->prev, h->prev2, h->prev3, h->prev4,
                                                            h->dotPrev, h->dot, h->cur, h->dotCur);
  LAUNCHED(h);
  return check_launch(h, "update_iter_step");
}

static int check_negjac(cfdgpu_handle *h)
{
  int v = 0;
  CK(cudaMemcpyAsync(&v, h->negjac, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  if (int rc = host_wait(h)) return rc;
  if (v) {
    h->err = "Negative Jacobian in the element routine";
    return CFDGPU_ENEGJAC;
  }
  return 0;
}

namespace cfdgpu {

int set_host_schedule(cfdgpu_handle *h, bool blocking, int chunk, int depth)
{
  if (!h || chunk < 1 || chunk > 64 || depth < 1 || depth > cfdgpu_handle::MAX_DEPTH) return CFDGPU_EINVAL;
  if (blocking != h->blocking) {
    constexpr int NE = cfdgpu_handle::MAX_DEPTH + 2;
    cudaEvent_t e[NE] = {};
    const unsigned flags = cudaEventDisableTiming | (blocking ? cudaEventBlockingSync : 0u);
    for (auto &x : e) CK(cudaEventCreateWithFlags(&x, flags));
    CK(cudaStreamSynchronize(h->stream));
    for (auto &x : h->evq) cudaEventDestroy(x);
    cudaEventDestroy(h->evw);
    for (int i = 0; i < NE - 1; i++) h->evq[i] = e[i];
    h->evw = e[NE - 1];
    h->blocking = blocking;
  }
  h->depth = depth;
  if (chunk != h->chunk) {
    // the cached Arnoldi graphs hold chunk-length pieces of the cycle
    CK(cudaStreamSynchronize(h->stream));
    for (auto &g : h->graphs64) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    for (auto &g : h->graphs32) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    for (auto &g : h->graphs_bcgs) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    h->chunk = chunk;
  }
  return 0;
}

int set_stream_priority(cfdgpu_handle *h, int priority)
{
  if (!h) return CFDGPU_EINVAL;
  cudaStream_t s2 = nullptr;
  CK(cudaStreamCreateWithPriority(&s2, cudaStreamNonBlocking, priority));
  CK(cudaStreamSynchronize(h->stream));
  cudaStreamDestroy(h->stream);
  h->stream = s2;
  return 0;
}

int handle_work(cfdgpu_handle *h, double *dofs, double *blocks)
{
  if (!h) return CFDGPU_EINVAL;
  if (dofs) *dofs = (double)h->n;
  if (blocks) *blocks = (double)h->topo.nnzb();
  return 0;
}

}  // namespace cfdgpu

namespace cfdgpu {
int handle_graph(cfdgpu_handle *h, GraphView *out)
{
  if (!h || !out) return CFDGPU_EINVAL;
  out->nNode = h->nNode; out->ndof = h->ndof; out->ndim = h->ndim; out->nfree = h->topo.nfree;
  out->rowptr = h->rowptr; out->colidx = h->colidx; out->coords = h->coords; out->fixmask = h->fixmask;
  out->stream = h->stream;
  return 0;
}
}  // namespace cfdgpu

extern "C" {

int cfdgpu_create(const cfdgpu_mesh *mesh, const cfdgpu_control *ctrl, const cfdgpu_solver_opts *opts,
                  cfdgpu_handle **out)
{
  if (!out) return CFDGPU_EINVAL;
  *out = nullptr;
  cfdgpu_handle *h = new cfdgpu_handle();
  *out = h;
  if (!mesh || !ctrl || !opts || !mesh->coords || !mesh->conn) { h->err = "null argument"; return CFDGPU_EINVAL; }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { h->err = "no CUDA device"; return CFDGPU_ENODEV; }
  h->ndim = mesh->ndim; h->npe = mesh->npElem; h->ndof = mesh->ndim + 1;
  h->nNode = mesh->nNode; h->nElem = mesh->nElem;
  if (h->ndim == 2 && h->npe == 3) h->et = CFDGPU_TRI3;
  else if (h->ndim == 2 && h->npe == 4) h->et = CFDGPU_QUAD4;
  else if (h->ndim == 3 && h->npe == 4) h->et = CFDGPU_TET4;
  else if (h->ndim == 3 && h->npe == 8) h->et = CFDGPU_HEX8;
  else { h->err = " Invalid npElem " + std::to_string(h->npe); return CFDGPU_EINVAL; }
  h->n = (int64_t)h->nNode * h->ndof;
  h->ctrl = *ctrl;
  h->opts = *opts;
  if (h->opts.restart <= 0) h->opts.restart = 30;
  if (h->opts.restart > 1000) { h->err = "restart > 1000 is not supported"; return CFDGPU_EINVAL; }
  if (h->opts.max_it <= 0) h->opts.max_it = 10000;
  if (h->opts.formulation != CFDGPU_FORM_SEMI_IMPLICIT && h->opts.formulation != CFDGPU_FORM_FULLY_IMPLICIT) {
    h->err = "unknown element formulation";
    return CFDGPU_EINVAL;
  }
  if (h->opts.ksp_type != CFDGPU_KSP_GMRES && h->opts.ksp_type != CFDGPU_KSP_BCGS &&
      h->opts.ksp_type != CFDGPU_KSP_PREONLY) {
    h->err = "unknown Krylov method";
    return CFDGPU_EINVAL;
  }
  if (h->opts.pc_type < CFDGPU_PC_NONE || h->opts.pc_type > CFDGPU_PC_BJACOBI_ILU) {
    h->err = "unknown preconditioner";
    return CFDGPU_EINVAL;
  }
  if (h->opts.ksp_type != CFDGPU_KSP_GMRES && h->opts.precision != CFDGPU_PREC_FP64) {
    h->err = "mixed precision solves with flexible GMRES (ksp_type CFDGPU_KSP_GMRES) around FP32 BiCGStab";
    return CFDGPU_EINVAL;
  }
  if (h->ctrl.newton_max_iter <= 0) h->ctrl.newton_max_iter = 10;
  if (h->ctrl.newton_max_iter > CFDGPU_MAX_NEWTON) h->ctrl.newton_max_iter = CFDGPU_MAX_NEWTON;
  h->m = h->opts.restart;

  auto t0 = std::chrono::steady_clock::now();
  std::string msg = build_topology(h->nNode, h->nElem, h->npe, h->ndof, mesh->conn, mesh->nDBC, mesh->dbc_node,
                                   mesh->dbc_dof, mesh->dbc_value, h->topo);
  if (!msg.empty()) { h->err = msg; return CFDGPU_EINVAL; }
  const Topology &t = h->topo;
  CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  for (auto &e : h->evq) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&h->evw, cudaEventDisableTiming));
  int rc = 0;
  const int64_t n = h->n;
  std::vector<int32_t> diag(h->nNode);
  for (int v = 0; v < h->nNode; v++) {
    const int32_t *b = t.colidx.data() + t.rowptr[v], *e = t.colidx.data() + t.rowptr[v + 1];
    diag[v] = (int32_t)(std::lower_bound(b, e, v) - t.colidx.data());
  }
  if ((rc = upload(h, &h->coords, mesh->coords, (size_t)h->nNode * h->ndim))) return rc;
  if ((rc = upload(h, &h->conn, mesh->conn, (size_t)h->nElem * h->npe))) return rc;
  if ((rc = upload(h, &h->rowptr, t.rowptr.data(), t.rowptr.size()))) return rc;
  if ((rc = upload(h, &h->colidx, t.colidx.data(), t.colidx.size()))) return rc;
  if ((rc = upload(h, &h->slot, t.slot.data(), t.slot.size()))) return rc;
  if ((rc = upload(h, &h->color_elems, t.color_elems.data(), t.color_elems.size()))) return rc;
  if ((rc = upload(h, &h->diag_slot, diag.data(), diag.size()))) return rc;
  if ((rc = upload(h, &h->fixmask, t.fixmask.data(), t.fixmask.size()))) return rc;
  if ((rc = upload(h, &h->dbc_index, t.dbc_index.data(), t.dbc_index.size()))) return rc;
  if ((rc = upload(h, &h->dbc_value, t.dbc_value.data(), t.dbc_value.size()))) return rc;
  if ((rc = upload(h, &h->fixed_dofs, t.fixed_dofs.data(), t.fixed_dofs.size()))) return rc;
  if ((rc = upload(h, &h->dbc_mult, t.dbc_mult.data(), t.dbc_mult.size()))) return rc;
  double **vecs[] = {&h->soln, &h->prev, &h->prev2, &h->prev3, &h->prev4, &h->cur, &h->dot,
                     &h->dotPrev, &h->dotCur, &h->applied, &h->rhs, &h->dx};
  for (double **v : vecs) {
    if ((rc = dalloc(h, v, (size_t)n))) return rc;
    CK(cudaMemset(*v, 0, sizeof(double) * n));
  }
  const size_t bb = (size_t)h->ndof * h->ndof;
  if (h->opts.precision != CFDGPU_PREC_FP64 && h->opts.precision != CFDGPU_PREC_MIXED) {
    h->err = "unknown precision mode";
    return CFDGPU_EINVAL;
  }
  h->mixed = (h->opts.precision == CFDGPU_PREC_MIXED);
  // Krylov stride: a multiple of 512 entries, so every update CTA covers whole chunks
  h->ldv = (n + 511) / 512 * 512;
  if ((rc = dalloc(h, &h->bsr, (size_t)t.nnzb() * bb))) return rc;
  CK(cudaMemset(h->bsr, 0, sizeof(double) * t.nnzb() * bb));
  if (h->mixed) {
    // FP32 copy of the tangent, FP32 preconditioner and FP32 inner BiCGStab
    // vectors; FP64 outer flexible GMRES (V and Z bases)
    h->inner_its = (h->opts.inner_restart > 0) ? h->opts.inner_restart : 20;
    if (h->inner_its > 1000) { h->err = "inner iterations > 1000 are not supported"; return CFDGPU_EINVAL; }
    h->inner_rtol = (h->opts.inner_rtol > 0.0) ? h->opts.inner_rtol : 1e-2;
    h->refine_rtol = (h->opts.refine_rtol > 0.0) ? h->opts.refine_rtol : 1e-10;
    if ((rc = dalloc(h, &h->bsr32, (size_t)t.nnzb() * bb))) return rc;
    CK(cudaMemset(h->bsr32, 0, sizeof(float) * t.nnzb() * bb));
    if ((rc = dalloc(h, &h->dinv32, (size_t)n))) return rc;
    if ((rc = dalloc(h, &h->binv32, (size_t)h->nNode * bb))) return rc;
    if ((rc = dalloc(h, &h->b32, (size_t)n))) return rc;
    CK(cudaMemset(h->b32, 0, sizeof(float) * n));
    float **iv[] = {&h->iR, &h->iRP, &h->iP, &h->iV, &h->iS, &h->iT, &h->ptmp32};
    for (float **v : iv) {
      if ((rc = dalloc(h, v, (size_t)n))) return rc;
      CK(cudaMemset(*v, 0, sizeof(float) * n));
    }
    if ((rc = dalloc(h, &h->ist, 1))) return rc;
    CK(cudaMemset(h->ist, 0, sizeof(BcgsState)));
    if ((rc = dalloc(h, &h->Zb, (size_t)h->ldv * h->m))) return rc;
    CK(cudaMemset(h->Zb, 0, sizeof(double) * h->ldv * h->m));
    std::vector<double> ones(h->m + 1, 1.0);
    if ((rc = upload(h, &h->ones, ones.data(), ones.size()))) return rc;
  } else {
    if ((rc = dalloc(h, &h->dinv, (size_t)n))) return rc;
    if ((rc = dalloc(h, &h->binv, (size_t)h->nNode * bb))) return rc;
  }
  if ((rc = dalloc(h, &h->V, (size_t)h->ldv * (h->m + 1)))) return rc;
  CK(cudaMemset(h->V, 0, sizeof(double) * h->ldv * (h->m + 1)));
  if ((rc = dalloc(h, &h->gst, 1))) return rc;
  if ((rc = dalloc(h, &h->ga.H, (size_t)(h->m + 1) * h->m))) return rc;
  if ((rc = dalloc(h, &h->ga.sigma, (size_t)h->m + 1))) return rc;
  if ((rc = dalloc(h, &h->ga.cs, (size_t)h->m))) return rc;
  if ((rc = dalloc(h, &h->ga.sn, (size_t)h->m))) return rc;
  if ((rc = dalloc(h, &h->ga.grs, (size_t)h->m + 1))) return rc;
  if ((rc = dalloc(h, &h->ga.y, (size_t)h->m))) return rc;
  {
    const int64_t ntiles = (h->ldv / 2 + ORTHO_THREADS - 1) / ORTHO_THREADS + h->ldv / 2 / MAXPY_SPAN + 1;
    if ((rc = dalloc(h, &h->ga.partial, (size_t)(h->m + 1) * std::max<int64_t>(ntiles, RED_BLOCKS)))) return rc;
  }
  if ((rc = dalloc(h, &h->ga.coef, (size_t)h->m + 1))) return rc;
  if ((rc = dalloc(h, &h->ga.kcount, (size_t)h->m / MDOT_KC + 2))) return rc;
  CK(cudaMemset(h->ga.kcount, 0, sizeof(unsigned int) * (h->m / MDOT_KC + 2)));
  if ((rc = dalloc(h, &h->red_partial, (size_t)RED_BLOCKS))) return rc;
  if ((rc = dalloc(h, &h->red_partial2, (size_t)5 * RED_BLOCKS))) return rc;
  if ((rc = dalloc(h, &h->red_counter, 1))) return rc;
  CK(cudaMemset(h->red_counter, 0, sizeof(unsigned int)));
  if ((rc = dalloc(h, &h->scalar, 8))) return rc;
  if ((rc = dalloc(h, &h->negjac, 1))) return rc;
  CK(cudaMemset(h->negjac, 0, sizeof(int)));
  CK(cudaMemset(h->gst, 0, sizeof(GmresState)));
  CK(cudaMallocHost(&h->h_scalar, 8 * sizeof(double)));
  CK(cudaMallocHost(&h->h_gst, (cfdgpu_handle::MAX_DEPTH + 2) * sizeof(GmresState)));
  if (h->opts.pc_type == CFDGPU_PC_BJACOBI_ILU) {
    const int nblk = (h->opts.bjacobi_blocks > 0) ? h->opts.bjacobi_blocks : 1;
    std::string m2 = build_ilu_pattern(t, h->opts.ilu_levels, nblk, h->ilu);
    if (!m2.empty()) { h->err = m2; return CFDGPU_EINVAL; }
    const IluPattern &f = h->ilu;
    if ((rc = upload(h, &h->frow, f.rowptr.data(), f.rowptr.size()))) return rc;
    if ((rc = upload(h, &h->fcol, f.colidx.data(), f.colidx.size()))) return rc;
    if ((rc = upload(h, &h->fdiag, f.diag.data(), f.diag.size()))) return rc;
    if ((rc = upload(h, &h->faslot, f.aslot.data(), f.aslot.size()))) return rc;
    if ((rc = upload(h, &h->fuoff, f.uoff.data(), f.uoff.size()))) return rc;
    if ((rc = upload(h, &h->fumap, f.umap.data(), f.umap.size()))) return rc;
    if ((rc = upload(h, &h->florder, f.lorder.data(), f.lorder.size()))) return rc;
    if ((rc = upload(h, &h->fuorder, f.uorder.data(), f.uorder.size()))) return rc;
    if ((rc = upload(h, &h->flchain, f.lchain.data(), f.lchain.size()))) return rc;
    if ((rc = upload(h, &h->fuchain, f.uchain.data(), f.uchain.size()))) return rc;
    if ((rc = upload(h, &h->flchord, f.lchain_order.data(), f.lchain_order.size()))) return rc;
    if ((rc = upload(h, &h->fuchord, f.uchain_order.data(), f.uchain_order.size()))) return rc;
    if (!f.perm.empty() && (rc = upload(h, &h->fperm, f.perm.data(), f.perm.size()))) return rc;
    if (h->mixed) {
      if ((rc = dalloc(h, &h->fval32, (size_t)f.nnzb() * bb))) return rc;
      CK(cudaMemset(h->fval32, 0, sizeof(float) * f.nnzb() * bb));
      if ((rc = dalloc(h, &h->fdinv32, (size_t)h->nNode * bb))) return rc;
      CK(cudaMemset(h->fdinv32, 0, sizeof(float) * h->nNode * bb));
    } else {
      if ((rc = dalloc(h, &h->fval, (size_t)f.nnzb() * bb))) return rc;
      CK(cudaMemset(h->fval, 0, sizeof(double) * f.nnzb() * bb));
      if ((rc = dalloc(h, &h->fdinv, (size_t)h->nNode * bb))) return rc;
      CK(cudaMemset(h->fdinv, 0, sizeof(double) * h->nNode * bb));
    }
    if ((rc = dalloc(h, &h->iflags, (size_t)h->nNode))) return rc;
    CK(cudaMemset(h->iflags, 0, sizeof(unsigned int) * h->nNode));
    if ((rc = dalloc(h, &h->tctl, 1))) return rc;
    CK(cudaMemset(h->tctl, 0, sizeof(TriCtl)));
    if ((rc = dalloc(h, &h->ptmp, (size_t)n))) return rc;
    CK(cudaMemset(h->ptmp, 0, sizeof(double) * n));
    if (h->mixed) {
      if ((rc = dalloc(h, &h->ybuf32, (size_t)n))) return rc;
      fill_sentinel_f32<<<grid_for(n), 256, 0, h->stream>>>(n, h->ybuf32);
    } else {
      if ((rc = dalloc(h, &h->ybuf, (size_t)n))) return rc;
      fill_sentinel_f64<<<grid_for(n), 256, 0, h->stream>>>(n, h->ybuf);
    }
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMallocHost(&h->h_tctl, sizeof(TriCtl)));
  }
  if (h->opts.ksp_type == CFDGPU_KSP_BCGS) {
    double **bv[] = {&h->bR, &h->bRP, &h->bP, &h->bV, &h->bS, &h->bT};
    for (double **v : bv) {
      if ((rc = dalloc(h, v, (size_t)n))) return rc;
      CK(cudaMemset(*v, 0, sizeof(double) * n));
    }
    if ((rc = dalloc(h, &h->bst, 1))) return rc;
    CK(cudaMemset(h->bst, 0, sizeof(BcgsState)));
    CK(cudaMallocHost(&h->h_bst, (cfdgpu_handle::MAX_DEPTH + 2) * sizeof(BcgsState)));
  }
  CK(cudaDeviceSynchronize());
  h->timers[0] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return 0;
}

int cfdgpu_destroy(cfdgpu_handle *h)
{
  if (!h) return 0;
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (void *p : h->allocs) cudaFree(p);
  if (h->h_scalar) cudaFreeHost(h->h_scalar);
  if (h->h_gst) cudaFreeHost(h->h_gst);
  for (auto &e : h->pev) cudaEventDestroy(e);
  for (auto g : h->graphs64) if (g) cudaGraphExecDestroy(g);
  for (auto g : h->graphs32) if (g) cudaGraphExecDestroy(g);
  for (auto g : h->graphs_bcgs) if (g) cudaGraphExecDestroy(g);
  if (h->h_tctl) cudaFreeHost(h->h_tctl);
  if (h->h_bst) cudaFreeHost(h->h_bst);
  for (auto &e : h->evq)
    if (e) cudaEventDestroy(e);
  if (h->evw) cudaEventDestroy(h->evw);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return 0;
}

const char *cfdgpu_last_error(const cfdgpu_handle *h) { return h ? h->err.c_str() : "null handle"; }

int cfdgpu_step(cfdgpu_handle *h, double timeNow, double timeFact, cfdgpu_step_stats *stats)
{
  (void)timeNow;
  if (!h || !stats) return CFDGPU_EINVAL;
  memset(stats, 0, sizeof(*stats));
  auto tstart = std::chrono::steady_clock::now();
  int rc;
  upload_td(h);
  // SolutionData::timeUpdate (SolutionData.cpp:64-78): rotate history
  double *old4 = h->prev4;
  h->prev4 = h->prev3; h->prev3 = h->prev2; h->prev2 = h->prev; h->prev = old4;
  CK(cudaMemcpyAsync(h->prev, h->soln, sizeof(double) * h->n, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaMemcpyAsync(h->dotPrev, h->dot, sizeof(double) * h->n, cudaMemcpyDeviceToDevice, h->stream));
  const int nDBC = (int)h->topo.dbc_index.size();
  if (nDBC) {
    k_apply_bc<<<(nDBC + 255) / 256, 256, 0, h->stream>>>(nDBC, h->dbc_index, h->dbc_value, timeFact, h->soln, h->applied);
    LAUNCHED(h);
    if ((rc = check_launch(h, "apply_bc"))) return rc;
  }
  const int nfix = (int)h->topo.fixed_dofs.size();
  // the semi-implicit tangent depends only on solnPrev: one assembly per step;
  // the fully-implicit tangent depends on the iterate: one per iteration
  const bool reuse = h->opts.reuse_tangent != 0 && h->opts.formulation == CFDGPU_FORM_SEMI_IMPLICIT;
  double ms_asm = 0.0, ms_sol = 0.0;
  for (int iter = 0; iter < h->ctrl.newton_max_iter; iter++) {
    auto ta = std::chrono::steady_clock::now();
    if ((rc = update_iter_step(h))) return rc;
    const bool want_K = !reuse || iter == 0;
    if ((rc = assemble(h, iter, want_K))) return rc;
    if (iter == 0 && (h->guess || (h->guess_mode & CFDGPU_GUESS_EXTRAPOLATION))) {
      // Initial guess u_n + a1*d1 + a2*d2 on the free dofs, d1 the network's
      // predicted increment (optionally velocity only), d2 the extrapolated
      // increment u_n - u_{n-1}.  The iteration-0 residual is affine in the
      // state, F(u_n + d) = F_A - K d, and K d_i = F_A - F(u_n + d_i), so the
      // coefficients minimising ||F|| come from a 2x2 least-squares problem on
      // the two residual differences.  No decrease keeps the constant
      // predictor (the reference's guess) unchanged.
      double nplain = 0.0;
      if ((rc = norm2(h, h->rhs, &nplain))) return rc;
      CK(cudaMemcpyAsync(h->rhs_plain, h->rhs, sizeof(double) * h->n, cudaMemcpyDeviceToDevice, h->stream));
      const bool use_net = h->guess && (h->guess_mode & (CFDGPU_GUESS_NETWORK | CFDGPU_GUESS_NETWORK_VELOCITY));
      const bool use_ext = (h->guess_mode & CFDGPU_GUESS_EXTRAPOLATION) != 0;
      double *dir[2] = {h->guess_delta, h->guess_dir2};
      double *res[2] = {h->guess_res1, h->guess_res2};
      int nd = 0;
      if (use_net) {
        if ((rc = cfdgpu::mpnn_predict_increment(h->guess, h->prev, h->prev2, h->guess_delta, h->stream))) {
          h->err = "guess network failed";
          return rc;
        }
        if (!(h->guess_mode & CFDGPU_GUESS_NETWORK)) {
          k_zero_dof<<<grid_for(h->nNode), 256, 0, h->stream>>>(h->nNode, h->ndof, h->ndof - 1, h->guess_delta);
          LAUNCHED(h);
        }
        dir[nd++] = h->guess_delta;
      }
      if (use_ext) {
        double *d2 = (nd == 0) ? h->guess_delta : h->guess_dir2;
        k_diff_free<<<grid_for(h->n), 256, 0, h->stream>>>(h->nNode, h->ndof, h->prev, h->prev2, h->fixmask, d2);
        LAUNCHED(h);
        dir[nd++] = d2;
      }
      for (int q = 0; q < nd; q++) {
        CK(cudaMemcpyAsync(h->soln, h->prev, sizeof(double) * h->n, cudaMemcpyDeviceToDevice, h->stream));
        k_axpy<<<grid_for(h->n), 256, 0, h->stream>>>(h->n, 1.0, dir[q], h->soln);
        LAUNCHED(h);
        if ((rc = update_iter_step(h))) return rc;
        if ((rc = assemble(h, 0, false))) return rc;
        CK(cudaMemcpyAsync(res[q], h->rhs, sizeof(double) * h->n, cudaMemcpyDeviceToDevice, h->stream));
      }
      minres_dots2<<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(h->n, h->rhs_plain, res[0], nd > 1 ? res[1] : res[0],
                                                             h->red_partial2, h->red_counter, h->scalar + 2);
      LAUNCHED(h);
      CK(cudaMemcpyAsync(h->h_scalar + 2, h->scalar + 2, 5 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
      if ((rc = host_wait(h))) return rc;
      const double r1 = h->h_scalar[2], r2 = h->h_scalar[3], g11 = h->h_scalar[4], g12 = h->h_scalar[5],
                   g22 = h->h_scalar[6];
      double a1 = 0.0, a2 = 0.0;
      const double det = g11 * g22 - g12 * g12;
      if (nd > 1 && det > 1e-12 * g11 * g22) {
        a1 = (r1 * g22 - r2 * g12) / det;
        a2 = (g11 * r2 - g12 * r1) / det;
      } else if (g11 > 0.0) {
        a1 = r1 / g11;
      }
      const double decrease = a1 * r1 + (nd > 1 ? a2 * r2 : 0.0);   // ||F_A||^2 - ||F||^2
      const double nguess = std::sqrt(std::max(nplain * nplain - decrease, 0.0));
      stats->plain_norm = nplain;
      stats->guess_norm = nplain;
      CK(cudaMemcpyAsync(h->soln, h->prev, sizeof(double) * h->n, cudaMemcpyDeviceToDevice, h->stream));
      if (decrease > 0.0 && nguess < nplain) {
        stats->guess_used = 1;
        stats->guess_alpha = a1;
        stats->guess_alpha2 = (nd > 1) ? a2 : 0.0;
        stats->guess_norm = nguess;
        // soln = u_n + a1 d1 + a2 d2 ; rhs = (1 - a1 - a2) F_A + a1 F_1 + a2 F_2
        k_axpy<<<grid_for(h->n), 256, 0, h->stream>>>(h->n, a1, dir[0], h->soln);
        k_lincomb<<<grid_for(h->n), 256, 0, h->stream>>>(h->n, a1, res[0], 0.0, h->rhs);
        h->launches += 2;
        if (nd > 1) {
          k_axpy<<<grid_for(h->n), 256, 0, h->stream>>>(h->n, a2, dir[1], h->soln);
          k_axpy<<<grid_for(h->n), 256, 0, h->stream>>>(h->n, a2, res[1], h->rhs);
          h->launches += 2;
        }
        k_axpy<<<grid_for(h->n), 256, 0, h->stream>>>(h->n, 1.0 - a1 - (nd > 1 ? a2 : 0.0), h->rhs_plain, h->rhs);
        LAUNCHED(h);
      } else {
        CK(cudaMemcpyAsync(h->rhs, h->rhs_plain, sizeof(double) * h->n, cudaMemcpyDeviceToDevice, h->stream));
      }
      if ((rc = update_iter_step(h))) return rc;
      if (!reuse && stats->guess_used) {
        // fully implicit: the residual is not affine and the tangent moves
        // with the state, so the chosen guess is re-assembled and kept only
        // if its true residual is lower
        if ((rc = assemble(h, 0, true))) return rc;
        double ntrue = 0.0;
        if ((rc = norm2(h, h->rhs, &ntrue))) return rc;
        stats->guess_norm = ntrue;
        if (!(ntrue < nplain)) {
          stats->guess_used = 0;
          stats->guess_alpha = stats->guess_alpha2 = 0.0;
          stats->guess_norm = nplain;
          CK(cudaMemcpyAsync(h->soln, h->prev, sizeof(double) * h->n, cudaMemcpyDeviceToDevice, h->stream));
          if ((rc = update_iter_step(h))) return rc;
          if ((rc = assemble(h, 0, true))) return rc;
        }
      }
    }
    if (iter == 0 && nfix) {
      k_dirichlet_update<<<(nfix + 255) / 256, 256, 0, h->stream>>>(nfix, h->fixed_dofs, h->dbc_mult, h->applied, h->soln);
      LAUNCHED(h);
      if ((rc = check_launch(h, "dirichlet_update"))) return rc;
    }
    double norm = 0.0;
    if ((rc = norm2(h, h->rhs, &norm))) return rc;
    if ((rc = check_negjac(h))) return rc;
    ms_asm += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ta).count();
    stats->norms[iter] = norm;
    stats->newton_iters = iter + 1;
    // the reference's absolute test (StabFEM2.cpp:749); with newton_rtol > 0
    // the residual must also have dropped by that factor from the
    // iteration-0 residual of the constant predictor (the reference's start,
    // so that a better initial guess does not tighten the test)
    if (iter == 0) {
      const double fref = (stats->plain_norm > 0.0) ? stats->plain_norm : norm;
      h->newton_target = (h->opts.newton_rtol > 0.0) ? std::min(h->ctrl.newton_tol, h->opts.newton_rtol * fref)
                                                      : h->ctrl.newton_tol;
    }
    if (norm < h->ctrl.newton_tol && norm <= h->newton_target) {
      stats->converged = 1;
      break;
    }
    auto ts = std::chrono::steady_clock::now();
    if (want_K && (rc = build_pc(h))) return rc;
    int its = 0, reason = 0, passes = 0;
    if (h->mixed) {
      if ((rc = fgmres_mixed(h, h->rhs, h->dx, &its, &reason))) return rc;
      if ((rc = ilu_check(h))) return rc;
      passes = its;
    } else {
      if ((rc = krylov_solve(h, h->rhs, h->dx, &its, &reason))) return rc;
    }
    stats->ksp_its[iter] = its;
    stats->ksp_reason[iter] = reason;
    stats->refinements[iter] = passes;
    if (reason < 0) {
      h->err = "KSP diverged, reason " + std::to_string(reason) + " after " + std::to_string(its) + " iterations";
      return CFDGPU_EKSP;
    }
    k_axpy<<<grid_for(h->n), 256, 0, h->stream>>>(h->n, 1.0, h->dx, h->soln);
    LAUNCHED(h);
    if ((rc = check_launch(h, "axpy"))) return rc;
    if ((rc = host_wait(h))) return rc;
    ms_sol += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ts).count();
  }
  if ((rc = host_wait(h))) return rc;
  stats->ms_assembly = ms_asm;
  stats->ms_solver = ms_sol;
  stats->ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tstart).count();
  h->timers[1] += ms_asm * 1e-3;
  h->timers[2] += ms_sol * 1e-3;
  h->timers[4] += stats->ms_total * 1e-3;
  return 0;
}

int cfdgpu_set_guess(cfdgpu_handle *h, cfdgpu_mpnn *m)
{
  return cfdgpu_set_guess_mode(h, m, m ? (CFDGPU_GUESS_NETWORK | CFDGPU_GUESS_EXTRAPOLATION) : 0);
}

int cfdgpu_set_guess_mode(cfdgpu_handle *h, cfdgpu_mpnn *m, int mode)
{
  if (!h) return CFDGPU_EINVAL;
  if (mode && !h->guess_delta) {
    int rc;
    if ((rc = dalloc(h, &h->guess_delta, (size_t)h->n))) return rc;
    if ((rc = dalloc(h, &h->rhs_plain, (size_t)h->n))) return rc;
    if ((rc = dalloc(h, &h->guess_dir2, (size_t)h->n))) return rc;
    if ((rc = dalloc(h, &h->guess_res1, (size_t)h->n))) return rc;
    if ((rc = dalloc(h, &h->guess_res2, (size_t)h->n))) return rc;
  }
  if (!m) mode &= ~(CFDGPU_GUESS_NETWORK | CFDGPU_GUESS_NETWORK_VELOCITY);
  h->guess = m;
  h->guess_mode = mode;
  return 0;
}

int cfdgpu_get_solution(cfdgpu_handle *h, double *soln)
{
  if (!h || !soln) return CFDGPU_EINVAL;
  CK(cudaMemcpyAsync(soln, h->soln, sizeof(double) * h->n, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

int cfdgpu_set_solution(cfdgpu_handle *h, const double *soln)
{
  if (!h || !soln) return CFDGPU_EINVAL;
  CK(cudaMemcpyAsync(h->soln, soln, sizeof(double) * h->n, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

int cfdgpu_device_solution(cfdgpu_handle *h, double **dptr)
{
  if (!h || !dptr) return CFDGPU_EINVAL;
  *dptr = h->soln;
  return 0;
}

int cfdgpu_stream(cfdgpu_handle *h, void **stream)
{
  if (!h || !stream) return CFDGPU_EINVAL;
  *stream = (void *)h->stream;
  return 0;
}

int cfdgpu_set_history(cfdgpu_handle *h, const double *solnPrev, const double *solnDot)
{
  if (!h) return CFDGPU_EINVAL;
  if (solnPrev) CK(cudaMemcpyAsync(h->prev, solnPrev, sizeof(double) * h->n, cudaMemcpyHostToDevice, h->stream));
  if (solnDot) CK(cudaMemcpyAsync(h->dot, solnDot, sizeof(double) * h->n, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

int cfdgpu_get_history(cfdgpu_handle *h, double *solnPrev, double *solnDot)
{
  if (!h) return CFDGPU_EINVAL;
  if (solnPrev) CK(cudaMemcpyAsync(solnPrev, h->prev, sizeof(double) * h->n, cudaMemcpyDeviceToHost, h->stream));
  if (solnDot) CK(cudaMemcpyAsync(solnDot, h->dot, sizeof(double) * h->n, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

int cfdgpu_set_element_state(cfdgpu_handle *h, const double *solnPrev, const double *solnCur, const double *solnDotCur)
{
  if (!h) return CFDGPU_EINVAL;
  upload_td(h);
  if (solnPrev) CK(cudaMemcpyAsync(h->prev, solnPrev, sizeof(double) * h->n, cudaMemcpyHostToDevice, h->stream));
  if (solnCur) CK(cudaMemcpyAsync(h->cur, solnCur, sizeof(double) * h->n, cudaMemcpyHostToDevice, h->stream));
  if (solnDotCur) CK(cudaMemcpyAsync(h->dotCur, solnDotCur, sizeof(double) * h->n, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

int cfdgpu_element_matrices(cfdgpu_handle *h, const int32_t *elem_ids, int n, double *K, double *F)
{
  if (!h || !elem_ids || n < 0 || !K || !F) return CFDGPU_EINVAL;
  if (n == 0) return 0;
  for (int i = 0; i < n; i++)
    if (elem_ids[i] < 0 || elem_ids[i] >= h->nElem) { h->err = "element id out of range"; return CFDGPU_EINVAL; }
  if (!h->td_set) upload_td(h);
  const int nsize = h->npe * h->ndof;
  int32_t *d_ids = nullptr;
  double *dK = nullptr, *dF = nullptr;
  CK(cudaMalloc(&d_ids, sizeof(int32_t) * n));
  CK(cudaMalloc(&dK, sizeof(double) * (size_t)n * nsize * nsize));
  CK(cudaMalloc(&dF, sizeof(double) * (size_t)n * nsize));
  CK(cudaMemcpyAsync(d_ids, elem_ids, sizeof(int32_t) * n, cudaMemcpyHostToDevice, h->stream));
  int rc = launch_elements_et<MODE_EXPORT, false>(h, d_ids, n, dK, dF);
  if (!rc) {
    CK(cudaMemcpyAsync(K, dK, sizeof(double) * (size_t)n * nsize * nsize, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(F, dF, sizeof(double) * (size_t)n * nsize, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  }
  cudaFree(d_ids); cudaFree(dK); cudaFree(dF);
  if (!rc) rc = check_negjac(h);
  return rc;
}

int cfdgpu_pattern_info_get(cfdgpu_handle *h, cfdgpu_pattern_info *info)
{
  if (!h || !info) return CFDGPU_EINVAL;
  info->nNode = h->nNode; info->nElem = h->nElem; info->npElem = h->npe; info->ndof = h->ndof;
  info->nnzb = h->topo.nnzb(); info->ncolors = h->topo.ncolors;
  info->nfixed = (int)h->topo.fixed_dofs.size(); info->nfree = h->topo.nfree;
  return 0;
}

int cfdgpu_export_pattern(cfdgpu_handle *h, int32_t *rowptr, int32_t *colidx, int32_t *slot, int32_t *color,
                          int32_t *color_ptr, int32_t *color_elems, int32_t *fixed_dofs, int32_t *dofmap)
{
  if (!h) return CFDGPU_EINVAL;
  const Topology &t = h->topo;
  auto cp = [](int32_t *dst, const std::vector<int32_t> &v) { if (dst && !v.empty()) memcpy(dst, v.data(), v.size() * 4); };
  cp(rowptr, t.rowptr); cp(colidx, t.colidx); cp(slot, t.slot); cp(color, t.color); cp(color_ptr, t.color_ptr);
  cp(color_elems, t.color_elems); cp(fixed_dofs, t.fixed_dofs); cp(dofmap, t.dofmap);
  return 0;
}

int cfdgpu_pattern_build(const cfdgpu_mesh *mesh, cfdgpu_pattern_info *info, int32_t *rowptr, int32_t *colidx,
                         int32_t *slot, int32_t *color, int32_t *color_ptr, int32_t *color_elems,
                         int32_t *fixed_dofs, int32_t *dofmap)
{
  if (!mesh || !info || !mesh->conn) return CFDGPU_EINVAL;
  Topology t;
  std::string msg = build_topology(mesh->nNode, mesh->nElem, mesh->npElem, mesh->ndim + 1, mesh->conn, mesh->nDBC,
                                   mesh->dbc_node, mesh->dbc_dof, mesh->dbc_value, t);
  if (!msg.empty()) return CFDGPU_EINVAL;
  info->nNode = mesh->nNode; info->nElem = mesh->nElem; info->npElem = mesh->npElem; info->ndof = mesh->ndim + 1;
  info->nnzb = t.nnzb(); info->ncolors = t.ncolors;
  info->nfixed = (int)t.fixed_dofs.size(); info->nfree = t.nfree;
  auto cp = [](int32_t *dst, const std::vector<int32_t> &v) { if (dst && !v.empty()) memcpy(dst, v.data(), v.size() * 4); };
  cp(rowptr, t.rowptr); cp(colidx, t.colidx); cp(slot, t.slot); cp(color, t.color); cp(color_ptr, t.color_ptr);
  cp(color_elems, t.color_elems); cp(fixed_dofs, t.fixed_dofs); cp(dofmap, t.dofmap);
  return 0;
}

int cfdgpu_ilu_pattern_build(const cfdgpu_mesh *mesh, int levels, int nblocks, cfdgpu_ilu_info *info,
                             int32_t *rowptr, int32_t *colidx, int32_t *perm, int32_t *lorder, int32_t *uorder,
                             int32_t *lchain, int32_t *uchain, int32_t *lchain_order, int32_t *uchain_order)
{
  if (!mesh || !info || !mesh->conn) return CFDGPU_EINVAL;
  Topology t;
  std::string msg = build_topology(mesh->nNode, mesh->nElem, mesh->npElem, mesh->ndim + 1, mesh->conn, mesh->nDBC,
                                   mesh->dbc_node, mesh->dbc_dof, mesh->dbc_value, t);
  if (!msg.empty()) return CFDGPU_EINVAL;
  IluPattern f;
  msg = build_ilu_pattern(t, levels, nblocks, f);
  if (!msg.empty()) return CFDGPU_EINVAL;
  info->nNode = mesh->nNode;
  info->nnzb = f.nnzb();
  info->nchains_l = (int)f.lchain_order.size();
  info->nchains_u = (int)f.uchain_order.size();
  info->nlev_l = f.nlev_l;
  info->nlev_u = f.nlev_u;
  info->chain_levels_l = f.lchain_levels;
  info->chain_levels_u = f.uchain_levels;
  auto cp = [](int32_t *dst, const std::vector<int32_t> &v) { if (dst && !v.empty()) memcpy(dst, v.data(), v.size() * 4); };
  cp(rowptr, f.rowptr); cp(colidx, f.colidx); cp(lorder, f.lorder); cp(uorder, f.uorder);
  cp(lchain, f.lchain); cp(uchain, f.uchain); cp(lchain_order, f.lchain_order); cp(uchain_order, f.uchain_order);
  if (perm) {
    if (f.perm.empty())
      for (int i = 0; i < mesh->nNode; i++) perm[i] = i;
    else
      cp(perm, f.perm);
  }
  return 0;
}

int cfdgpu_assemble_export(cfdgpu_handle *h, int iter, double *bsr_vals, double *rhs)
{
  if (!h) return CFDGPU_EINVAL;

  if (!h->td_set) upload_td(h);
  int rc = assemble(h, iter, true);
  if (rc) return rc;
  const size_t bb = (size_t)h->ndof * h->ndof;
  if (bsr_vals) CK(cudaMemcpyAsync(bsr_vals, h->bsr, sizeof(double) * h->topo.nnzb() * bb, cudaMemcpyDeviceToHost, h->stream));
  if (rhs) CK(cudaMemcpyAsync(rhs, h->rhs, sizeof(double) * h->n, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return check_negjac(h);
}

int cfdgpu_solve_export(cfdgpu_handle *h, const double *b, double *x, int *its, int *reason)
{
  if (!h || !b || !x) return CFDGPU_EINVAL;
  if (h->mixed) { h->err = "cfdgpu_solve_export solves the FP64 system"; return CFDGPU_EINVAL; }
  if (!h->assembled_K) { h->err = "assemble the matrix first"; return CFDGPU_EINVAL; }
  CK(cudaMemcpyAsync(h->rhs, b, sizeof(double) * h->n, cudaMemcpyHostToDevice, h->stream));
  int rc = build_pc(h);
  if (rc) return rc;
  int i = 0, r = 0;
  rc = krylov_solve(h, h->rhs, h->dx, &i, &r);
  if (rc) return rc;
  CK(cudaMemcpyAsync(x, h->dx, sizeof(double) * h->n, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (its) *its = i;
  if (reason) *reason = r;
  return 0;
}

int cfdgpu_ilu_export(cfdgpu_handle *h, int64_t *nnzb, int32_t *rowptr, int32_t *colidx, int32_t *diag, double *vals,
                      double *dinv)
{
  if (!h) return CFDGPU_EINVAL;
  if (h->opts.pc_type != CFDGPU_PC_BJACOBI_ILU) { h->err = "the handle has no ILU preconditioner"; return CFDGPU_EINVAL; }
  if (h->mixed && (vals || dinv)) { h->err = "mixed precision keeps FP32 factors"; return CFDGPU_EINVAL; }
  const IluPattern &f = h->ilu;
  if (nnzb) *nnzb = f.nnzb();
  auto cp = [](int32_t *dst, const std::vector<int32_t> &v) { if (dst && !v.empty()) memcpy(dst, v.data(), v.size() * 4); };
  cp(rowptr, f.rowptr); cp(colidx, f.colidx); cp(diag, f.diag);
  if (!vals && !dinv) return 0;
  if (!h->assembled_K) { h->err = "assemble the matrix first"; return CFDGPU_EINVAL; }
  int rc = build_pc(h);
  if (rc) return rc;
  const size_t bb = (size_t)h->ndof * h->ndof;
  if (vals) CK(cudaMemcpyAsync(vals, h->fval, sizeof(double) * f.nnzb() * bb, cudaMemcpyDeviceToHost, h->stream));
  if (dinv) CK(cudaMemcpyAsync(dinv, h->fdinv, sizeof(double) * h->nNode * bb, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return ilu_check(h);
}

int cfdgpu_pc_apply_export(cfdgpu_handle *h, const double *r, double *z)
{
  if (!h || !r || !z) return CFDGPU_EINVAL;
  if (h->mixed) { h->err = "cfdgpu_pc_apply_export uses the FP64 preconditioner"; return CFDGPU_EINVAL; }
  if (!h->assembled_K) { h->err = "assemble the matrix first"; return CFDGPU_EINVAL; }
  int rc = build_pc(h);
  if (rc) return rc;
  CK(cudaMemcpyAsync(h->rhs, r, sizeof(double) * h->n, cudaMemcpyHostToDevice, h->stream));
  if ((rc = pc_apply_vec(h, h->rhs, h->dx))) return rc;
  CK(cudaMemcpyAsync(z, h->dx, sizeof(double) * h->n, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return ilu_check(h);
}

int cfdgpu_true_residual(cfdgpu_handle *h, const double *x, const double *b, double *norm)
{
  if (!h || !x || !b || !norm) return CFDGPU_EINVAL;

  if (!h->assembled_K) { h->err = "assemble the matrix first"; return CFDGPU_EINVAL; }
  // x -> dx, b -> rhs, r = b - A x -> applied-free scratch (the Krylov vector V_0)
  CK(cudaMemcpyAsync(h->dx, x, sizeof(double) * h->n, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->rhs, b, sizeof(double) * h->n, cudaMemcpyHostToDevice, h->stream));
  const int saved_pc = h->opts.pc_type;
  h->opts.pc_type = CFDGPU_PC_NONE;
  int rc = spmv_pc(h, 1, h->dx, h->rhs, h->V, nullptr, 0, nullptr);
  h->opts.pc_type = saved_pc;
  if (rc) return rc;
  return norm2(h, h->V, norm);
}

int cfdgpu_timers(cfdgpu_handle *h, double t[5])
{
  if (!h || !t) return CFDGPU_EINVAL;
  for (int i = 0; i < 5; i++) t[i] = h->timers[i];
  return 0;
}

int64_t cfdgpu_launch_count(cfdgpu_handle *h) { return h ? h->launches : -1; }

int cfdgpu_set_profiling(cfdgpu_handle *h, int on)
{
  if (!h) return CFDGPU_EINVAL;
  if (on && h->pev.empty()) {
    h->pev.resize(2 * PROF_POOL);
    h->pkind.resize(PROF_POOL);
    h->pbytes.resize(PROF_POOL);
    for (auto &e : h->pev) CK(cudaEventCreate(&e));
  }
  if (!on) prof_collect(h);
  h->prof = on != 0;
  for (int k = 0; k < CFDGPU_KIND_COUNT; k++) { h->prof_launches[k] = 0; h->prof_ms[k] = 0.0; h->prof_bytes[k] = 0.0; }
  return 0;
}

int cfdgpu_kernel_stats(cfdgpu_handle *h, int kind, int64_t *launches, double *total_ms, double *total_bytes)
{
  if (!h || kind < 0 || kind >= CFDGPU_KIND_COUNT) return CFDGPU_EINVAL;
  CK(cudaStreamSynchronize(h->stream));
  prof_collect(h);
  if (launches) *launches = h->prof_launches[kind];
  if (total_ms) *total_ms = h->prof_ms[kind];
  if (total_bytes) *total_bytes = h->prof_bytes[kind];
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free residual norm.
//
// Some callers may not allocate device memory themselves: a host code that
// runs inside another framework's memory pool (where cudaMalloc is disallowed
// or would fragment the pool), a solver embedded in a process whose GPU memory
// is budgeted up front, or code that may only enqueue work on a stream it is
// handed.  cfdgpu_residual_norm_noalloc serves them: it computes the same
// ||b - A x||_2 as cfdgpu_true_residual on a BSR matrix the caller already
// holds on the device, and keeps its scratch (the residual vector and the
// reduction partials) in the file-scope device array below instead of
// allocating.  The array is reserved when the library is loaded and every GPU
// that loads the library holds it (16 MiB + 2.6 KiB) until the process exits.
//
// Host code must not pass g_noalloc_scratch itself to a kernel: on the host that
// name is a stand-in, not a device address.  The device address is looked up
// with cudaGetSymbolAddress, with the device current, and cached per device
// under a mutex (two host threads making their first call on one device do not
// race on the cache).  Calls made outside stream capture look the address up
// again, so a cache entry left stale by cudaDeviceReset (which unloads the
// module and may place the array elsewhere on the next load) is replaced
// before it is used; a call made while its stream is being captured uses the
// cached address, which is why the first call on a device must come before any
// capture.
namespace {
constexpr int64_t NOALLOC_MAX_N = int64_t(1) << 21;          // residual entries (nNode*ndof)
constexpr int64_t NOALLOC_WORDS = NOALLOC_MAX_N + RED_BLOCKS + 32;
constexpr int NOALLOC_MAX_DEVICES = 64;
}  // namespace

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_WORDS];

static double *g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {nullptr};
static std::mutex g_noalloc_mu;

// Device address of the scratch array on the current device.
static int noalloc_scratch(cudaStream_t s, double **out)
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return CFDGPU_ENODEV;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) return CFDGPU_ECUDA;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (cap == cudaStreamCaptureStatusNone || !g_noalloc_ptr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return CFDGPU_ECUDA;
    g_noalloc_ptr[dev] = (double *)p;
  }
  *out = g_noalloc_ptr[dev];
  return 0;
}

static inline bool aligned_to(const void *p, uintptr_t a) { return ((uintptr_t)p % a) == 0; }

extern "C" int cfdgpu_residual_norm_noalloc(int nNode, int ndof, const int32_t *d_rowptr, const int32_t *d_colidx,
                                            const double *d_val, const double *d_x, const double *d_b,
                                            double *d_norm, void *stream)
{
  if (nNode <= 0 || (ndof != 3 && ndof != 4) || !d_rowptr || !d_colidx || !d_val || !d_x || !d_b || !d_norm)
    return CFDGPU_EINVAL;
  // the 4x4 kernel reads blocks and x with 16-byte loads
  if (!aligned_to(d_rowptr, 4) || !aligned_to(d_colidx, 4) || !aligned_to(d_val, 16) || !aligned_to(d_x, 16) ||
      !aligned_to(d_b, 16) || !aligned_to(d_norm, 8))
    return CFDGPU_EINVAL;
  const int64_t n = (int64_t)nNode * ndof;
  if (n > NOALLOC_MAX_N) return CFDGPU_ETOOBIG;
  cudaStream_t s = (cudaStream_t)stream;
  double *scratch = nullptr;
  int rc = noalloc_scratch(s, &scratch);
  if (rc) return rc;
  double *r = scratch;                                            // residual, n doubles
  double *partial = scratch + NOALLOC_MAX_N;                      // RED_BLOCKS doubles
  unsigned int *counter = (unsigned int *)(scratch + NOALLOC_MAX_N + RED_BLOCKS);
  // the array keeps the previous call's contents: the arrival counter must start at zero
  if (cudaMemsetAsync(counter, 0, sizeof(unsigned int), s) != cudaSuccess) return CFDGPU_ECUDA;
  if (ndof == 4) {
    const int grid = (int)((nNode * 32LL + 255) / 256);
    bsr4_spmv<1, 0, double><<<grid, 256, 0, s>>>(nNode, d_rowptr, d_colidx, d_val, d_x, d_b, nullptr, nullptr, r,
                                                nullptr, 0, nullptr);
  } else {
    const int grid = (int)((n + 255) / 256);
    bsr_spmv_generic<3, 1, 0, double><<<grid, 256, 0, s>>>(nNode, d_rowptr, d_colidx, d_val, d_x, d_b, nullptr,
                                                             nullptr, r, nullptr, 0, nullptr);
  }
  if (cudaGetLastError() != cudaSuccess) return CFDGPU_ECUDA;
  norm2_kernel<<<RED_BLOCKS, RED_THREADS, 0, s>>>(n, r, partial, counter, d_norm);
  if (cudaGetLastError() != cudaSuccess) return CFDGPU_ECUDA;
  return 0;
}
