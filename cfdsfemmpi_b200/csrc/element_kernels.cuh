// Element residual/tangent kernels with fused, colour-ordered BSR assembly.
//
// One thread group per element: 32 lanes (one warp) for hex8, 16 lanes for
// quad4/tet4/tri3 (two elements per warp).  Per element:
//   A. the group stages the element's nodal coordinates and solution values
//      in shared memory (one lane per node);
//   B. one lane per Gauss point evaluates the basis, the mapping Jacobian and
//      the interpolated fields and stores them in shared memory;
//   C. each lane accumulates one or two nodal blocks K_ij over the Gauss
//      points in registers (hex8: lane -> node i = lane/4, j in {2(lane%4),
//      2(lane%4)+1}); lanes with j-group 0 also accumulate F_i;
//   D. iteration-0 lifting F_i -= K_ij applied_j, Dirichlet masking, and the
//      write of each block to its BSR slot: the first writer of a block (in
//      colour order) stores, later writers add.  Elements of one colour share
//      no node, so a launch per colour is race-free and every matrix entry
//      receives its contributions in the same order on every run.
//
// FORM_SEMI_IMPLICIT follows the active "semi-implicit type B" element
// routines of the reference (file:line within the reference project):
//   quad4 src/base/LagrangeElem2DNavierStokesQuad4Node.cpp:683-970
//   tri3  src/base/LagrangeElem2DNavierStokesTria3Node.cpp:683-968
//   hex8  src/base/LagrangeElem3DNavierStokesHexa8Node.cpp:764-1074
//   tet4  src/base/LagrangeElem3DNavierStokesTetra4Node.cpp:769-1078
// FORM_FULLY_IMPLICIT follows the reference's commented-out "Fully-implicit
// formulation" routines (quad4 :117-396, tri3 :117-396, hex8 :109-432, tet4
// :115-438 of the same files): convection grad(u) u with its Newton
// linearisation, SUPG weight on the current velocity with its derivative,
// PSPG, LSIC in 3D, no sign-flipped rows, CI 10 (hex8) or 4; the 2D and 3D
// texts differ (2D: SUPG without rho, af on the pressure column; 3D: SUPG
// with rho, no af on the pressure column) and are kept as written.
// with prepareElemData (basis, w*detJ, charlen) recomputed from coordinates
// instead of stored, the basis of src/base/BasisFunctionsLagrange.cpp (hexa
// p=1 derivative table as the reference writes it, :1053-1078), quadrature of
// src/base/UtilitiesQuadrature.cpp, and tau from
// src/base/stabilisationRoutines.h:128-143.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cfdgpu.h"

namespace cfdgpu {

struct ElemParams {
  double rho, mu, af, am, acceFact;
  double stab0, stab1, stab2;   // SUPG, PSPG, LSIC factors
};

template <int ET> struct ElemTraits;
template <> struct ElemTraits<CFDGPU_HEX8> {
  static constexpr int NDIM = 3, NPE = 8, NGP = 8, GS = 32, PPL = 2;
  static constexpr bool SUPG = false;
  static constexpr double CS = -1.0, CI = 10.0;
};
template <> struct ElemTraits<CFDGPU_TET4> {
  static constexpr int NDIM = 3, NPE = 4, NGP = 1, GS = 16, PPL = 1;
  static constexpr bool SUPG = false;
  static constexpr double CS = 1.0, CI = 10.0;
};
template <> struct ElemTraits<CFDGPU_QUAD4> {
  static constexpr int NDIM = 2, NPE = 4, NGP = 4, GS = 16, PPL = 1;
  static constexpr bool SUPG = true;
  static constexpr double CS = 1.0, CI = 4.0;
};
template <> struct ElemTraits<CFDGPU_TRI3> {
  static constexpr int NDIM = 2, NPE = 3, NGP = 1, GS = 16, PPL = 1;
  static constexpr bool SUPG = true;
  static constexpr double CS = 1.0, CI = 4.0;
};

#define CFD_PI 3.141592653589793238462643383279502884197169399375105

// Quadrature point g of element type ET (UtilitiesQuadrature.cpp:17-28,
// 224-257, 263-301, 448-455; tri3 uses the 1-point quad rule, (0,0) w=4).
template <int ET>
__device__ __forceinline__ void gauss_point(int g, double xi[3], double &w)
{
  const double q = 0.577350269189626;
  if (ET == CFDGPU_HEX8) {
    xi[0] = (g & 1) ? q : -q; xi[1] = (g & 2) ? q : -q; xi[2] = (g & 4) ? q : -q; w = 1.0;
  } else if (ET == CFDGPU_QUAD4) {
    xi[0] = (g & 1) ? q : -q; xi[1] = (g & 2) ? q : -q; xi[2] = 0.0; w = 1.0;
  } else if (ET == CFDGPU_TET4) {
    xi[0] = 0.25; xi[1] = 0.25; xi[2] = 0.25; w = 1.0 / 6.0;
  } else {
    xi[0] = 0.0; xi[1] = 0.0; xi[2] = 0.0; w = 4.0;
  }
}

// Reference-element basis and derivatives.
template <int ET>
__device__ __forceinline__ void basis_ref(const double xi[3], double *N, double *d1, double *d2, double *d3)
{
  if (ET == CFDGPU_HEX8) {
    const double v11 = 1.0 - xi[0], v12 = 1.0 + xi[0];
    const double v21 = 1.0 - xi[1], v22 = 1.0 + xi[1];
    const double v31 = 1.0 - xi[2], v32 = 1.0 + xi[2];
    N[0] = 0.125 * v11 * v21 * v31; N[1] = 0.125 * v12 * v21 * v31;
    N[2] = 0.125 * v12 * v22 * v31; N[3] = 0.125 * v11 * v22 * v31;
    N[4] = 0.125 * v11 * v21 * v32; N[5] = 0.125 * v12 * v21 * v32;
    N[6] = 0.125 * v12 * v22 * v32; N[7] = 0.125 * v11 * v22 * v32;
    d1[0] = -0.125 * v21 * v31; d1[1] = 0.125 * v21 * v31;
    d1[2] = 0.125 * v22 * v31;  d1[3] = -0.125 * v22 * v31;
    d1[4] = -0.125 * v21 * v32; d1[5] = 0.125 * v21 * v32;
    d1[6] = 0.125 * v22 * v32;  d1[7] = -0.125 * v22 * v32;
    // xi2/xi3 rows: the reference's table (nodes 2,3 and 6,7 take the
    // factors v11/v12 in this order), kept for parity.
    d2[0] = -0.125 * v11 * v31; d2[1] = -0.125 * v12 * v31;
    d2[2] = 0.125 * v11 * v31;  d2[3] = 0.125 * v12 * v31;
    d2[4] = -0.125 * v11 * v32; d2[5] = -0.125 * v12 * v32;
    d2[6] = 0.125 * v11 * v32;  d2[7] = 0.125 * v12 * v32;
    d3[0] = -0.125 * v11 * v21; d3[1] = -0.125 * v12 * v21;
    d3[2] = -0.125 * v11 * v22; d3[3] = -0.125 * v12 * v22;
    d3[4] = 0.125 * v11 * v21;  d3[5] = 0.125 * v12 * v21;
    d3[6] = 0.125 * v11 * v22;  d3[7] = 0.125 * v12 * v22;
  } else if (ET == CFDGPU_QUAD4) {
    const double b1 = 0.5 * (1.0 - xi[1]), b2 = 0.5 * (1.0 + xi[1]);
    const double a1 = 0.5 * (1.0 - xi[0]), a2 = 0.5 * (1.0 + xi[0]);
    N[0] = b1 * a1; N[1] = b1 * a2; N[2] = b2 * a2; N[3] = b2 * a1;
    d1[0] = b1 * -0.5; d1[1] = b1 * 0.5; d1[2] = b2 * 0.5; d1[3] = b2 * -0.5;
    d2[0] = -0.5 * a1; d2[1] = -0.5 * a2; d2[2] = 0.5 * a2; d2[3] = 0.5 * a1;
  } else if (ET == CFDGPU_TET4) {
    N[0] = 1.0 - xi[0] - xi[1] - xi[2]; N[1] = xi[0]; N[2] = xi[1]; N[3] = xi[2];
    d1[0] = -1.0; d1[1] = 1.0; d1[2] = 0.0; d1[3] = 0.0;
    d2[0] = -1.0; d2[1] = 0.0; d2[2] = 1.0; d2[3] = 0.0;
    d3[0] = -1.0; d3[1] = 0.0; d3[2] = 0.0; d3[3] = 1.0;
  } else {
    N[0] = 1.0 - xi[0] - xi[1]; N[1] = xi[0]; N[2] = xi[1];
    d1[0] = -1.0; d1[1] = 1.0; d1[2] = 0.0;
    d2[0] = -1.0; d2[1] = 0.0; d2[2] = 1.0;
  }
}

template <int NDIM, int NPE, int NGP, int JG>
struct ElemSmem {
  double X[NPE][NDIM];
  double prev[NPE][NDIM];
  double cur[NPE][NDIM + 1];
  double dot[NPE][NDIM];
  double app[NPE][NDIM + 1];
  uint32_t fix[NPE];
  int32_t node[NPE];
  // per Gauss point
  double N[NGP][NPE];
  double dN[NGP][NDIM][NPE];
  double dvol[NGP];
  double vP[NGP][NDIM];
  double gP[NGP][NDIM][NDIM];
  double tau0[NGP], tau1[NGP], tau2[NGP];
  double res2[NGP][NDIM];
  double stress[NGP][NDIM][NDIM];
  double rStab[NGP][NDIM];
  double trg[NGP];
  int negjac;
  double Fpart[NPE][JG][NDIM + 1];
};

enum { MODE_ASSEMBLE = 0, MODE_RESIDUAL = 1, MODE_EXPORT = 2 };
enum { FORM_SEMI_IMPLICIT = 0, FORM_FULLY_IMPLICIT = 1 };

// CT: arithmetic type of the tangent accumulation; KST: stored BSR type.
// MODE_ASSEMBLE: K and F into the BSR/RHS (LIFT adds the iteration-0 lifting);
// MODE_RESIDUAL: F only; MODE_EXPORT: raw K_e/F_e into dense per-element output.
// FORM: FORM_SEMI_IMPLICIT or FORM_FULLY_IMPLICIT.
template <int ET, typename CT, typename KST, int MODE, bool LIFT, int GROUPS, int FORM>
__global__ void __launch_bounds__(ElemTraits<ET>::GS * GROUPS)
element_kernel(const int32_t *__restrict__ elems, int nel, const int32_t *__restrict__ conn,
               const double *__restrict__ coords, const double *__restrict__ solnPrev,
               const double *__restrict__ solnCur, const double *__restrict__ solnDotCur,
               const double *__restrict__ applied, const uint8_t *__restrict__ fixmask, ElemParams P,
               const int32_t *__restrict__ slot, KST *__restrict__ bsr, double *__restrict__ rhs,
               double *__restrict__ outK, double *__restrict__ outF, int *__restrict__ negjac_flag)
{
  using T = ElemTraits<ET>;
  constexpr int NDIM = T::NDIM, NPE = T::NPE, NGP = T::NGP, GS = T::GS, PPL = T::PPL;
  constexpr int NDOF = NDIM + 1, JG = NPE / PPL, NSIZE = NPE * NDOF;
  constexpr bool FI = (FORM == FORM_FULLY_IMPLICIT);
  constexpr double CS = FI ? 1.0 : T::CS;                       // continuity row sign
  constexpr double CI = FI ? ((ET == CFDGPU_HEX8) ? 10.0 : 4.0) : T::CI;
  constexpr bool SUPG = FI || T::SUPG;
  __shared__ ElemSmem<NDIM, NPE, NGP, JG> smem_all[GROUPS];

  const int grp = threadIdx.x / GS;
  const int lane = threadIdx.x % GS;
  const int k = blockIdx.x * GROUPS + grp;
  const bool active = k < nel;
  ElemSmem<NDIM, NPE, NGP, JG> &S = smem_all[grp];
  const int e = active ? (elems ? elems[k] : k) : 0;

  // A. stage nodal data
  if (active && lane < NPE) {
    const int n = conn[(int64_t)e * NPE + lane];
    S.node[lane] = n;
#pragma unroll
    for (int c = 0; c < NDIM; c++) S.X[lane][c] = coords[(int64_t)n * NDIM + c];
#pragma unroll
    for (int c = 0; c < NDIM; c++) S.prev[lane][c] = solnPrev[(int64_t)n * NDOF + c];
#pragma unroll
    for (int c = 0; c < NDOF; c++) S.cur[lane][c] = solnCur[(int64_t)n * NDOF + c];
#pragma unroll
    for (int c = 0; c < NDIM; c++) S.dot[lane][c] = solnDotCur[(int64_t)n * NDOF + c];
    if (MODE == MODE_ASSEMBLE || MODE == MODE_RESIDUAL) S.fix[lane] = fixmask[n];
    if (LIFT) {
#pragma unroll
      for (int c = 0; c < NDOF; c++) S.app[lane][c] = applied[(int64_t)n * NDOF + c];
    }
    if (lane == 0) S.negjac = 0;
  }
  __syncwarp();

  // B1. basis and w*detJ at Gauss point g = lane
  if (active && lane < NGP) {
    double xi[3], w;
    gauss_point<ET>(lane, xi, w);
    double N[NPE], d1[NPE], d2[NPE], d3[NPE];
    basis_ref<ET>(xi, N, d1, d2, d3);
    double J;
    if (NDIM == 2) {
      double B00 = 0, B01 = 0, B10 = 0, B11 = 0;
#pragma unroll
      for (int ii = 0; ii < NPE; ii++) {
        const double xx = S.X[ii][0], yy = S.X[ii][NDIM > 1 ? 1 : 0];
        B00 += (xx * d1[ii]); B10 += (xx * d2[ii]);
        B01 += (yy * d1[ii]); B11 += (yy * d2[ii]);
      }
      J = B00 * B11 - B01 * B10;
      const double detinv = 1.0 / J;
      const double I00 = B11 * detinv, I01 = -B01 * detinv, I10 = -B10 * detinv, I11 = B00 * detinv;
#pragma unroll
      for (int ii = 0; ii < NPE; ii++) {
        S.dN[lane][0][ii] = d1[ii] * I00 + d2[ii] * I01;
        S.dN[lane][NDIM > 1 ? 1 : 0][ii] = d1[ii] * I10 + d2[ii] * I11;
      }
    } else {
      double B[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
      for (int ii = 0; ii < NPE; ii++) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const double xc = S.X[ii][c < NDIM ? c : 0];
          B[0][c] += (xc * d1[ii]); B[1][c] += (xc * d2[ii]); B[2][c] += (xc * d3[ii]);
        }
      }
      double C[3][3];
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
          const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
          C[i][j] = B[i1][j1] * B[i2][j2] - B[i1][j2] * B[i2][j1];
        }
      J = B[0][0] * C[0][0] + B[0][1] * C[0][1] + B[0][2] * C[0][2];
      const double invdet = 1.0 / J;
#pragma unroll
      for (int ii = 0; ii < NPE; ii++) {
        // Binv(r,a) = C(a,r)/det
#pragma unroll
        for (int r = 0; r < NDIM; r++)
          S.dN[lane][r][ii] = d1[ii] * (C[0][r] * invdet) + d2[ii] * (C[1][r] * invdet) + d3[ii] * (C[2][r] * invdet);
      }
    }
#pragma unroll
    for (int ii = 0; ii < NPE; ii++) S.N[lane][ii] = N[ii];
    S.dvol[lane] = w * J;
    if (J < 0.0) S.negjac = 1;
  }
  __syncwarp();

  // B2. element size, tau, interpolated fields at Gauss point g = lane
  if (active && lane < NGP) {
    const int gp = lane;
    double elemVol = 0.0;
#pragma unroll
    for (int g = 0; g < NGP; g++) elemVol += S.dvol[g];
    const double charlen = (NDIM == 2) ? sqrt(4.0 * fabs(elemVol) / CFD_PI) : pow(6.0 * fabs(elemVol) / CFD_PI, 1.0 / 3.0);
    const double fact = 4.0 / charlen / charlen;
    double vP[NDIM], gP[NDIM][NDIM], vel[NDIM], grad[NDIM][NDIM], dp[NDIM], vD[NDIM], pres = 0.0;
#pragma unroll
    for (int a = 0; a < NDIM; a++) {
      vP[a] = 0.0; vel[a] = 0.0; dp[a] = 0.0; vD[a] = 0.0;
#pragma unroll
      for (int c = 0; c < NDIM; c++) { gP[a][c] = 0.0; grad[a][c] = 0.0; }
    }
#pragma unroll
    for (int ii = 0; ii < NPE; ii++) {
      const double Ni = S.N[gp][ii];
#pragma unroll
      for (int a = 0; a < NDIM; a++) {
        const double b = S.prev[ii][a];
        vP[a] += b * Ni;
#pragma unroll
        for (int c = 0; c < NDIM; c++) gP[a][c] += b * S.dN[gp][c][ii];
      }
#pragma unroll
      for (int a = 0; a < NDIM; a++) {
        const double b = S.cur[ii][a];
        vel[a] += b * Ni;
#pragma unroll
        for (int c = 0; c < NDIM; c++) grad[a][c] += b * S.dN[gp][c][ii];
      }
      const double b4 = S.cur[ii][NDIM];
      pres += b4 * Ni;
#pragma unroll
      for (int c = 0; c < NDIM; c++) dp[c] += b4 * S.dN[gp][c][ii];
#pragma unroll
      for (int a = 0; a < NDIM; a++) vD[a] += S.dot[ii][a] * Ni;
    }
    const double rho = P.rho, mu = P.mu;
    double tr = 0.0;
#pragma unroll
    for (int a = 0; a < NDIM; a++) {
#pragma unroll
      for (int c = 0; c < NDIM; c++) S.stress[gp][a][c] = mu * grad[a][c] - ((a == c) ? pres : 0.0);
      double r2;
      if (FI) {
        double g = 0;
#pragma unroll
        for (int c = 0; c < NDIM; c++) g += grad[a][c] * vel[c];
        r2 = rho * (vD[a] + g - 0.0);
      } else {
        double t1 = 0, t2 = 0, t3 = 0;
#pragma unroll
        for (int c = 0; c < NDIM; c++) {
          t1 += gP[a][c] * vel[c];
          t2 += grad[a][c] * vP[c];
          t3 += gP[a][c] * vP[c];
        }
        r2 = rho * (vD[a] + (t1 + t2 - t3) - 0.0);
      }
      S.res2[gp][a] = r2;
      S.rStab[gp][a] = r2 - mu * 0.0 + dp[a];
      tr += grad[a][a];
      // the tangent's advection velocity and gradient: the previous step's
      // (semi-implicit) or the current iterate's (fully implicit)
      S.vP[gp][a] = FI ? vel[a] : vP[a];
#pragma unroll
      for (int c = 0; c < NDIM; c++) S.gP[gp][a][c] = FI ? grad[a][c] : gP[a][c];
    }
    S.trg[gp] = tr;
    // evaluateStabParams_algo3 with G = fact*I (2D: third diagonal entry 0)
    double uGu = 0.0;
#pragma unroll
    for (int a = 0; a < NDIM; a++) uGu += vP[a] * (fact * vP[a]);
    const double sumG2 = NDIM * (fact * fact);
    double t0 = uGu + CI * (mu * mu / rho / rho) * sumG2;
    t0 = 1.0 / sqrt(t0);
    S.tau2[gp] = P.stab2 / (t0 * (NDIM * fact));
    t0 = t0 / rho;
    S.tau0[gp] = t0 * P.stab0;
    S.tau1[gp] = t0 * P.stab1;
  }
  __syncwarp();

  // C. tangent blocks (registers) and residual rows
  const int pl = lane;                  // pair lane
  const int ii = pl / JG;               // test node
  const int jg = pl % JG;               // j-group
  const bool pair_lane = active && pl < NPE * JG;
  const bool f_lane = pair_lane && jg == 0;
  CT acc[PPL][NDOF][NDOF];
#pragma unroll
  for (int p = 0; p < PPL; p++)
#pragma unroll
    for (int a = 0; a < NDOF; a++)
#pragma unroll
      for (int b = 0; b < NDOF; b++) acc[p][a][b] = CT(0);
  double Fi[NDOF];
#pragma unroll
  for (int a = 0; a < NDOF; a++) Fi[a] = 0.0;

  if (pair_lane) {
    const double rho = P.rho, af = P.af, acceFact = P.acceFact, muTaf = P.mu * P.af;
    for (int gp = 0; gp < NGP; gp++) {
      const double dvol = S.dvol[gp];
      double bb[NDIM];
#pragma unroll
      for (int a = 0; a < NDIM; a++) bb[a] = S.dN[gp][a][ii] * dvol;
      const double b4 = S.N[gp][ii] * dvol;
      const double b8 = af * b4;
      const double tau0 = S.tau0[gp], tau1 = S.tau1[gp], tau2 = S.tau2[gp];
      double vP[NDIM];
#pragma unroll
      for (int a = 0; a < NDIM; a++) vP[a] = S.vP[gp][a];
      double Da = 0.0;
#pragma unroll
      for (int a = 0; a < NDIM; a++) Da += vP[a] * bb[a];
      Da = (FI && NDIM == 2) ? Da * tau0 : rho * Da * tau0;

      if (MODE != MODE_RESIDUAL || LIFT) {
        const CT cb8 = CT(b8), cDa = CT(Da), ctau1 = CT(tau1), caf = CT(af), cb4 = CT(b4);
        CT cbb[NDIM], cbm[NDIM], cvP[NDIM], cgP[NDIM][NDIM];
#pragma unroll
        for (int a = 0; a < NDIM; a++) {
          cbb[a] = CT(bb[a]);
          cbm[a] = CT(muTaf * bb[a]);
          cvP[a] = CT(vP[a]);
#pragma unroll
          for (int c = 0; c < NDIM; c++) cgP[a][c] = CT(S.gP[gp][a][c]);
        }
        const CT crho = CT(rho), crhoacc = CT(rho * acceFact);
#pragma unroll
        for (int p = 0; p < PPL; p++) {
          const int jj = jg * PPL + p;
          const CT Nj = CT(S.N[gp][jj]);
          CT dNj[NDIM];
#pragma unroll
          for (int a = 0; a < NDIM; a++) dNj[a] = CT(S.dN[gp][a][jj]);
          const CT fact2 = crhoacc * Nj;
          CT f = cb4 * fact2;
          CT dif = CT(0);
#pragma unroll
          for (int a = 0; a < NDIM; a++) dif += cbm[a] * dNj[a];
          f += dif;
          const CT rN = crho * Nj;
          CT Db = CT(0);
#pragma unroll
          for (int a = 0; a < NDIM; a++) Db += cvP[a] * dNj[a];
          Db = crho * Db;
          CT gN[NDIM][NDIM];
#pragma unroll
          for (int a = 0; a < NDIM; a++)
#pragma unroll
            for (int c = 0; c < NDIM; c++) gN[a][c] = cgP[a][c] * rN + ((a == c) ? Db : CT(0));
#pragma unroll
          for (int a = 0; a < NDIM; a++) {
            acc[p][a][a] += f;
#pragma unroll
            for (int c = 0; c < NDIM; c++) acc[p][a][c] += cb8 * gN[a][c];
            if (FI && NDIM == 3) acc[p][a][NDIM] -= cbb[a] * Nj;
            else acc[p][a][NDIM] -= cbb[a] * caf * Nj;
          }
#pragma unroll
          for (int c = 0; c < NDIM; c++) acc[p][NDIM][c] += CT(CS) * (cb8 * dNj[c]);
          // Dj = af*gN + fact2*I | af*dN
          CT Dj[NDIM][NDOF];
#pragma unroll
          for (int a = 0; a < NDIM; a++) {
#pragma unroll
            for (int c = 0; c < NDIM; c++) Dj[a][c] = gN[a][c] * caf + ((a == c) ? fact2 : CT(0));
            Dj[a][NDIM] = caf * dNj[a];
          }
          if (SUPG) {
#pragma unroll
            for (int a = 0; a < NDIM; a++)
#pragma unroll
              for (int c = 0; c < NDOF; c++) acc[p][a][c] += cDa * Dj[a][c];
          }
          if (FI) {
            // derivative of the SUPG weight (u . grad N_i) tau0 [rho]
            const CT c1 = (NDIM == 3) ? CT(tau0 * af * rho) * Nj : CT(tau0 * af) * Nj;
#pragma unroll
            for (int a = 0; a < NDIM; a++) {
              const CT rs = CT(S.rStab[gp][a]);
#pragma unroll
              for (int c = 0; c < NDIM; c++) acc[p][a][c] += c1 * cbb[c] * rs;
            }
          }
#pragma unroll
          for (int c = 0; c < NDOF; c++) {
            CT s = CT(0);
#pragma unroll
            for (int a = 0; a < NDIM; a++) s += cbb[a] * Dj[a][c];
            acc[p][NDIM][c] += CT(CS) * (s * ctau1);
          }
          if (FI && NDIM == 3) {
            // LSIC
            const CT f2 = CT(rho * af * tau2);
#pragma unroll
            for (int a = 0; a < NDIM; a++)
#pragma unroll
              for (int c = 0; c < NDIM; c++) acc[p][a][c] += (cbb[a] * dNj[c]) * f2;
          }
        }
      }
      if (f_lane) {
#pragma unroll
        for (int a = 0; a < NDIM; a++) {
          double s = b4 * S.res2[gp][a];
#pragma unroll
          for (int c = 0; c < NDIM; c++) s += bb[c] * S.stress[gp][a][c];
          Fi[a] -= s;
        }
        Fi[NDIM] -= CS * (b4 * S.trg[gp]);
        if (SUPG) {
#pragma unroll
          for (int a = 0; a < NDIM; a++) Fi[a] -= Da * S.rStab[gp][a];
        }
        double s = 0.0;
#pragma unroll
        for (int a = 0; a < NDIM; a++) s += bb[a] * S.rStab[gp][a];
        Fi[NDIM] -= CS * (tau1 * s);
        if (FI && NDIM == 3) {
          const double f2 = tau2 * rho * S.trg[gp];
#pragma unroll
          for (int a = 0; a < NDIM; a++) Fi[a] -= bb[a] * f2;
        }
      }
    }
  }

  if (MODE == MODE_EXPORT) {
    if (pair_lane) {
#pragma unroll
      for (int p = 0; p < PPL; p++) {
        const int jj = jg * PPL + p;
#pragma unroll
        for (int a = 0; a < NDOF; a++)
#pragma unroll
          for (int b = 0; b < NDOF; b++)
            outK[(int64_t)k * NSIZE * NSIZE + (int64_t)(ii * NDOF + a) * NSIZE + jj * NDOF + b] = (double)acc[p][a][b];
      }
      if (f_lane) {
#pragma unroll
        for (int a = 0; a < NDOF; a++) outF[(int64_t)k * NSIZE + ii * NDOF + a] = Fi[a];
      }
    }
    if (active && lane == 0 && S.negjac) atomicExch(negjac_flag, 1);
    return;
  }

  // D. lifting (iteration 0): F_i -= K_ij * applied_j over prescribed (j, b)
  if (LIFT) {
    if (pair_lane) {
      const uint32_t fi = S.fix[ii];
      double part[NDOF];
#pragma unroll
      for (int a = 0; a < NDOF; a++) part[a] = 0.0;
#pragma unroll
      for (int p = 0; p < PPL; p++) {
        const int jj = jg * PPL + p;
        const uint32_t fj = S.fix[jj];
#pragma unroll
        for (int b = 0; b < NDOF; b++) {
          const double app = S.app[jj][b];
          if (((fj >> b) & 1u) && fabs(app) > 1.0e-10) {
#pragma unroll
            for (int a = 0; a < NDOF; a++)
              if (!((fi >> a) & 1u)) part[a] -= (double)acc[p][a][b] * app;
          }
        }
      }
#pragma unroll
      for (int a = 0; a < NDOF; a++) S.Fpart[ii][jg][a] = part[a];
    }
    __syncwarp();
    if (f_lane) {
#pragma unroll
      for (int g = 0; g < JG; g++)
#pragma unroll
        for (int a = 0; a < NDOF; a++) Fi[a] += S.Fpart[ii][g][a];
    }
  }

  // E. masked writes
  if (pair_lane) {
    const uint32_t fi = S.fix[ii];
    if (MODE == MODE_ASSEMBLE) {
#pragma unroll
      for (int p = 0; p < PPL; p++) {
        const int jj = jg * PPL + p;
        const uint32_t fj = S.fix[jj];
        int32_t s = slot[((int64_t)e * NPE + ii) * NPE + jj];
        const bool first = s < 0;
        const int64_t base = (int64_t)(first ? -s - 1 : s) * (NDOF * NDOF);
        KST vals[NDOF * NDOF];
#pragma unroll
        for (int a = 0; a < NDOF; a++)
#pragma unroll
          for (int b = 0; b < NDOF; b++) {
            const bool m = ((fi >> a) & 1u) || ((fj >> b) & 1u);
            vals[a * NDOF + b] = m ? KST(0) : KST(acc[p][a][b]);
          }
        if (first) {
#pragma unroll
          for (int q = 0; q < NDOF * NDOF; q++) bsr[base + q] = vals[q];
        } else {
#pragma unroll
          for (int q = 0; q < NDOF * NDOF; q++) bsr[base + q] += vals[q];
        }
      }
    }
    if (f_lane) {
      const int64_t r = (int64_t)S.node[ii] * NDOF;
#pragma unroll
      for (int a = 0; a < NDOF; a++)
        if (!((fi >> a) & 1u)) rhs[r + a] += Fi[a];
    }
  }
  if (active && lane == 0 && S.negjac) atomicExch(negjac_flag, 1);
}

}  // namespace cfdgpu
