// BiCGStab on the device with the semantics of PETSc 3.10 KSPSolve_BCGS, the
// Krylov method of the reference's input/petsc_options_bcgs.dat:1 (read
// through SolverPetsc.cpp:101): left preconditioning, x0 = 0, the
// preconditioned residual norm in KSPConvergedDefault, breakdown when
// (v, rp) = 0 or rho = 0, and the t = 0 exit (x += alpha p) of the omega
// step.  Every scalar lives in a device control block updated by the last
// CTA of a deterministic reduction (fixed grid, fixed order), so iterations
// can be enqueued in CUDA-graph chunks without host round trips; once the
// solve has ended every kernel of a later iteration returns at once.
//
// One iteration (vectors r, rp, p, v, s, t, x; M^-1 A applied by the caller
// between the kernels):
//   bcgs_p       p = r - omega_old beta v + beta p
//   (caller)     v = M^-1 A p
//   bcgs_alpha   alpha = rho / (v, rp)
//   bcgs_s       s = r - alpha v
//   (caller)     t = M^-1 A s
//   bcgs_omega   omega = (s, t) / (t, t)
//   bcgs_xr      x = alpha p + omega s + x, r = s - omega t, ||r||, rho = (r, rp)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "linalg_kernels.cuh"

namespace cfdgpu {

struct BcgsState {
  int its, reason, active, maxit;
  int tzero;                // (t, t) = 0 and (s, s) = 0: x += alpha p ends the solve
  int skip;                 // inner solve of a flexible GMRES step whose cycle has ended: nothing runs
  double rtol, atol, dtol, rnorm0, ttol;
  double rho, rhoold, alpha, omega, omegaold, beta, dp;
  unsigned int counter;
};

// KSPConvergedDefault on the BCGS control block
__device__ __forceinline__ int bcgs_converged(BcgsState *s, int n_its, double rnorm)
{
  if (n_its == 0) {
    s->rnorm0 = rnorm;
    s->ttol = fmax(s->rtol * rnorm, s->atol);
  }
  if (isnan(rnorm) || isinf(rnorm)) return -9;
  if (rnorm <= s->ttol) return (rnorm < s->atol) ? 3 : 2;
  if (rnorm >= s->dtol * s->rnorm0) return -4;
  return 0;
}

__global__ void bcgs_setup(BcgsState *st, int maxit, double rtol, double atol, double dtol,
                           const GmresState *__restrict__ outer = nullptr, int j = 0)
{
  if (threadIdx.x || blockIdx.x) return;
  st->skip = (outer && (!outer->active || outer->it != j)) ? 1 : 0;
  st->its = 0; st->reason = 0; st->active = 0; st->maxit = maxit; st->tzero = 0;
  st->rtol = rtol; st->atol = atol; st->dtol = dtol; st->rnorm0 = 0.0; st->ttol = 0.0;
  st->rho = 0.0; st->rhoold = 1.0; st->alpha = 1.0; st->omega = 1.0; st->omegaold = 1.0; st->beta = 0.0;
  st->dp = 0.0;
  st->counter = 0u;
}

// Start: r holds M^-1 b.  rp = r, p = v = 0, dp = ||r||, rho = (r, rp),
// convergence test at iteration 0.
template <typename VT>
__global__ void __launch_bounds__(RED_THREADS)
bcgs_init(int64_t n, const VT *__restrict__ r, VT *__restrict__ rp, VT *__restrict__ p, VT *__restrict__ v,
          BcgsState *st, double *__restrict__ partial)
{
  if (st->skip) return;
  __shared__ double sh[RED_THREADS / 32];
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * RED_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * RED_THREADS) {
    const VT x = r[i];
    rp[i] = x;
    p[i] = VT(0);
    v[i] = VT(0);
    s = fma((double)x, (double)x, s);
  }
  s = block_sum<RED_THREADS>(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  if (last_block(&st->counter, gridDim.x)) {
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (unsigned int k = 0; k < gridDim.x; k++) t += __ldcg(partial + k);
      const double dp = sqrt(t);
      st->dp = dp;
      st->its = 0;
      const int reason = bcgs_converged(st, 0, dp);
      st->reason = reason;
      st->active = (reason == 0 && st->maxit > 0) ? 1 : 0;
      // first iteration: rho = (r, rp), beta = (rho / 1) (1 / 1)
      st->rho = t;
      st->rhoold = 1.0; st->alpha = 1.0; st->omegaold = 1.0;
      st->beta = (st->rho / st->rhoold) * (st->alpha / st->omegaold);
    }
  }
}

template <typename VT>
__global__ void bcgs_p(int64_t n, const VT *__restrict__ r, const VT *__restrict__ v, VT *__restrict__ p,
                       const BcgsState *__restrict__ st)
{
  if (!st->active) return;
  const double b = st->beta, c = -st->omegaold * st->beta;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = (VT)(1.0 * (double)r[i] + c * (double)v[i] + b * (double)p[i]);
}

// alpha = rho / (v, rp); (v, rp) = 0 is a breakdown
template <typename VT>
__global__ void __launch_bounds__(RED_THREADS)
bcgs_alpha(int64_t n, const VT *__restrict__ v, const VT *__restrict__ rp, BcgsState *st, double *__restrict__ partial)
{
  if (!st->active) return;
  __shared__ double sh[RED_THREADS / 32];
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * RED_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * RED_THREADS)
    s = fma((double)v[i], (double)rp[i], s);
  s = block_sum<RED_THREADS>(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  if (last_block(&st->counter, gridDim.x)) {
    if (threadIdx.x == 0) {
      double d1 = 0.0;
      for (unsigned int k = 0; k < gridDim.x; k++) d1 += __ldcg(partial + k);
      if (isnan(d1) || isinf(d1)) {
        st->reason = -9; st->active = 0;      // KSP_DIVERGED_NANORINF
      } else if (d1 == 0.0) {
        st->reason = -5; st->active = 0;      // KSP_DIVERGED_BREAKDOWN
      } else {
        st->alpha = st->rho / d1;
      }
    }
  }
}

template <typename VT>
__global__ void bcgs_s(int64_t n, const VT *__restrict__ r, const VT *__restrict__ v, VT *__restrict__ s,
                       const BcgsState *__restrict__ st)
{
  if (!st->active) return;
  const double a = -st->alpha;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s[i] = (VT)(a * (double)v[i] + (double)r[i]);
}

// omega = (s, t) / (t, t); (t, t) = 0 ends the solve (x += alpha p) when
// s = 0, else it is a breakdown
template <typename VT>
__global__ void __launch_bounds__(RED_THREADS)
bcgs_omega(int64_t n, const VT *__restrict__ s, const VT *__restrict__ t, BcgsState *st, double *__restrict__ partial)
{
  if (!st->active) return;
  __shared__ double sh[RED_THREADS / 32];
  double a = 0.0, b = 0.0, c = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * RED_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * RED_THREADS) {
    const double si = (double)s[i], ti = (double)t[i];
    a = fma(si, ti, a);
    b = fma(ti, ti, b);
    c = fma(si, si, c);
  }
  a = block_sum<RED_THREADS>(a, sh);
  b = block_sum<RED_THREADS>(b, sh);
  c = block_sum<RED_THREADS>(c, sh);
  if (threadIdx.x == 0) {
    partial[3 * blockIdx.x] = a;
    partial[3 * blockIdx.x + 1] = b;
    partial[3 * blockIdx.x + 2] = c;
  }
  if (last_block(&st->counter, gridDim.x)) {
    if (threadIdx.x == 0) {
      double d1 = 0.0, d2 = 0.0, d3 = 0.0;
      for (unsigned int k = 0; k < gridDim.x; k++) {
        d1 += __ldcg(partial + 3 * k);
        d2 += __ldcg(partial + 3 * k + 1);
        d3 += __ldcg(partial + 3 * k + 2);
      }
      if (d2 == 0.0) {
        if (d3 != 0.0) {
          st->reason = -5; st->active = 0;    // singular preconditioned operator
        } else {
          st->tzero = 1;
          st->omega = 0.0;
        }
      } else {
        st->omega = d1 / d2;
      }
    }
  }
}

// x = alpha p + omega s + x, r = s - omega t; dp = ||r||, convergence test,
// then rho of the next iteration = (r, rp) and its beta
template <typename VT>
__global__ void __launch_bounds__(RED_THREADS)
bcgs_xr(int64_t n, double *__restrict__ x, const VT *__restrict__ p, const VT *__restrict__ s, const VT *__restrict__ t,
        VT *__restrict__ r, const VT *__restrict__ rp, BcgsState *st, double *__restrict__ partial)
{
  if (!st->active) return;
  __shared__ double sh[RED_THREADS / 32];
  const double alpha = st->alpha, omega = st->omega;
  const bool tz = st->tzero != 0;
  double a = 0.0, b = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * RED_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * RED_THREADS) {
    if (tz) {
      x[i] += alpha * (double)p[i];
    } else {
      x[i] = alpha * (double)p[i] + omega * (double)s[i] + 1.0 * x[i];
      const VT ri = (VT)(-omega * (double)t[i] + (double)s[i]);
      r[i] = ri;
      const double rd = (double)ri;
      a = fma(rd, rd, a);
      b = fma(rd, (double)rp[i], b);
    }
  }
  a = block_sum<RED_THREADS>(a, sh);
  b = block_sum<RED_THREADS>(b, sh);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = a;
    partial[2 * blockIdx.x + 1] = b;
  }
  if (last_block(&st->counter, gridDim.x)) {
    if (threadIdx.x == 0) {
      st->its = st->its + 1;
      if (tz) {
        st->dp = 0.0;
        st->reason = 2;                       // KSP_CONVERGED_RTOL
        st->active = 0;
      } else {
        double rr = 0.0, rrp = 0.0;
        for (unsigned int k = 0; k < gridDim.x; k++) {
          rr += __ldcg(partial + 2 * k);
          rrp += __ldcg(partial + 2 * k + 1);
        }
        const double dp = sqrt(rr);
        st->dp = dp;
        const double rho = st->rho;
        st->rhoold = rho;
        st->omegaold = omega;
        int reason = bcgs_converged(st, st->its, dp);
        if (reason == 0 && rho == 0.0) reason = -5;
        if (reason == 0 && st->its >= st->maxit) reason = -3;   // KSP_DIVERGED_ITS
        st->reason = reason;
        st->active = (reason == 0) ? 1 : 0;
        st->rho = rrp;
        st->beta = (st->rho / st->rhoold) * (st->alpha / st->omegaold);
      }
    }
  }
}

}  // namespace cfdgpu
