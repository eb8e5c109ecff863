/*
 * oracle.c -- CPU restatement of the cfdsfemmpi per-time-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * library in cfdsfemmpi_b200/csrc and the timed CPU baseline of bench.py's
 * reference arm.  Nothing in the product links, loads or calls it.
 *
 * What it restates (file:line within the reference project):
 *   - element routines, active "semi-implicit type B" variants:
 *       quad4  src/base/LagrangeElem2DNavierStokesQuad4Node.cpp:36-113, 683-970
 *       tri3   src/base/LagrangeElem2DNavierStokesTria3Node.cpp:36-113, 683-968
 *       hex8   src/base/LagrangeElem3DNavierStokesHexa8Node.cpp:31-106, 764-1074
 *       tet4   src/base/LagrangeElem3DNavierStokesTetra4Node.cpp:31-112, 769-1078
 *   - basis functions  src/base/BasisFunctionsLagrange.cpp:18-186 (mapping),
 *       517-546 (tria p=1), 703-731 (quad p=1), 889-910 (tetra p=1),
 *       1035-1079 (hexa p=1, including its derivative table as written)
 *   - quadrature  src/base/UtilitiesQuadrature.cpp:17-28, 224-257, 263-301, 448-455
 *   - stabilisation  src/base/stabilisationRoutines.h:128-143 (algo3)
 *   - per-element Dirichlet lifting  src/base/StabFEM2.cpp:678-703
 *   - scatter into the free-dof matrix  src/base/SolverPetsc.cpp:304-314
 *   - free-dof pattern  src/base/StabFEM2.cpp:57-81, 192-227
 *   - Krylov solve: PETSc 3.10.5 KSPGMRES with classical Gram-Schmidt (no
 *     refinement), left preconditioning, preconditioned-residual norm,
 *     x0 = 0, and KSPConvergedDefault; PC "jacobi" (inverse diagonal); KSPBCGS;
 *     PCBJACOBI with ILU(k) blocks.  PETSc is a third-party dependency that is
 *     not part of the reference tree; the algorithms below are its published
 *     ones, called from SolverPetsc.cpp:253.
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off -fopenmp).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.141592653589793238462643383279502884197169399375105

enum { ORC_TRI3 = 0, ORC_QUAD4 = 1, ORC_TET4 = 2, ORC_HEX8 = 3 };

static void einfo(int et, int *ndim, int *npe, int *ngp)
{
  switch (et) {
    case ORC_TRI3:  *ndim = 2; *npe = 3; *ngp = 1; break;
    case ORC_QUAD4: *ndim = 2; *npe = 4; *ngp = 4; break;
    case ORC_TET4:  *ndim = 3; *npe = 4; *ngp = 1; break;
    default:        *ndim = 3; *npe = 8; *ngp = 8; break;
  }
}

int orc_element_info(int et, int *ndim, int *npe, int *ngp)
{
  einfo(et, ndim, npe, ngp);
  return 0;
}

/* ---------------- quadrature (UtilitiesQuadrature.cpp) ---------------- */
static void gauss_points(int et, double gp[][3], double *w)
{
  const double g2[2] = {-0.577350269189626, 0.577350269189626};
  int ind = 0;
  if (et == ORC_QUAD4) {           /* :224-257, xi1 fastest */
    for (int jj = 0; jj < 2; jj++)
      for (int ii = 0; ii < 2; ii++) {
        gp[ind][0] = g2[ii]; gp[ind][1] = g2[jj]; gp[ind][2] = 0.0;
        w[ind] = 1.0 * 1.0; ind++;
      }
  } else if (et == ORC_TRI3) {     /* tri3 calls getGaussPointsQuad(1): (0,0), w = 2*2 */
    gp[0][0] = 0.0; gp[0][1] = 0.0; gp[0][2] = 0.0; w[0] = 2.0 * 2.0;
  } else if (et == ORC_TET4) {     /* :448-455 */
    gp[0][0] = 0.25; gp[0][1] = 0.25; gp[0][2] = 0.25; w[0] = 1.0 / 6.0;
  } else {                         /* :263-301, xi1 fastest, then xi2, then xi3 */
    for (int kk = 0; kk < 2; kk++)
      for (int jj = 0; jj < 2; jj++)
        for (int ii = 0; ii < 2; ii++) {
          gp[ind][0] = g2[ii]; gp[ind][1] = g2[jj]; gp[ind][2] = g2[kk];
          w[ind] = 1.0 * 1.0 * 1.0; ind++;
        }
  }
}

/* ---------------- reference-element basis (BasisFunctionsLagrange.cpp) -- */
static void basis_ref(int et, const double *xi, double *N, double *d1, double *d2, double *d3)
{
  if (et == ORC_TRI3) {
    double xi3 = 1.0 - xi[0] - xi[1];
    N[0] = xi3; N[1] = xi[0]; N[2] = xi[1];
    d1[0] = -1.0; d1[1] = 1.0; d1[2] = 0.0;
    d2[0] = -1.0; d2[1] = 0.0; d2[2] = 1.0;
  } else if (et == ORC_QUAD4) {
    double b1 = 0.5 * (1.0 - xi[1]), b2 = 0.5 * (1.0 + xi[1]);
    double db1 = -0.5, db2 = 0.5;
    double a1 = 0.5 * (1.0 - xi[0]), a2 = 0.5 * (1.0 + xi[0]);
    double da1 = -0.5, da2 = 0.5;
    N[0] = b1 * a1; N[1] = b1 * a2; N[2] = b2 * a2; N[3] = b2 * a1;
    d1[0] = b1 * da1; d1[1] = b1 * da2; d1[2] = b2 * da2; d1[3] = b2 * da1;
    d2[0] = db1 * a1; d2[1] = db1 * a2; d2[2] = db2 * a2; d2[3] = db2 * a1;
  } else if (et == ORC_TET4) {
    double xi4 = 1.0 - xi[0] - xi[1] - xi[2];
    N[0] = xi4; N[1] = xi[0]; N[2] = xi[1]; N[3] = xi[2];
    d1[0] = -1.0; d1[1] = 1.0; d1[2] = 0.0; d1[3] = 0.0;
    d2[0] = -1.0; d2[1] = 0.0; d2[2] = 1.0; d2[3] = 0.0;
    d3[0] = -1.0; d3[1] = 0.0; d3[2] = 0.0; d3[3] = 1.0;
  } else {
    /* BasisFunctionsLagrange.cpp:1037-1078.  The xi2 and xi3 derivative
     * rows pair local nodes 2<->3 and 6<->7 differently from N; this is the
     * reference's table and is kept as written. */
    double v11 = 1.0 - xi[0], v12 = 1.0 + xi[0];
    double v21 = 1.0 - xi[1], v22 = 1.0 + xi[1];
    double v31 = 1.0 - xi[2], v32 = 1.0 + xi[2];
    N[0] = 0.125 * v11 * v21 * v31; N[1] = 0.125 * v12 * v21 * v31;
    N[2] = 0.125 * v12 * v22 * v31; N[3] = 0.125 * v11 * v22 * v31;
    N[4] = 0.125 * v11 * v21 * v32; N[5] = 0.125 * v12 * v21 * v32;
    N[6] = 0.125 * v12 * v22 * v32; N[7] = 0.125 * v11 * v22 * v32;
    d1[0] = -0.125 * v21 * v31; d1[1] = 0.125 * v21 * v31;
    d1[2] = 0.125 * v22 * v31;  d1[3] = -0.125 * v22 * v31;
    d1[4] = -0.125 * v21 * v32; d1[5] = 0.125 * v21 * v32;
    d1[6] = 0.125 * v22 * v32;  d1[7] = -0.125 * v22 * v32;
    d2[0] = -0.125 * v11 * v31; d2[1] = -0.125 * v12 * v31;
    d2[2] = 0.125 * v11 * v31;  d2[3] = 0.125 * v12 * v31;
    d2[4] = -0.125 * v11 * v32; d2[5] = -0.125 * v12 * v32;
    d2[6] = 0.125 * v11 * v32;  d2[7] = 0.125 * v12 * v32;
    d3[0] = -0.125 * v11 * v21; d3[1] = -0.125 * v12 * v21;
    d3[2] = -0.125 * v11 * v22; d3[3] = -0.125 * v12 * v22;
    d3[4] = 0.125 * v11 * v21;  d3[5] = 0.125 * v12 * v21;
    d3[6] = 0.125 * v11 * v22;  d3[7] = 0.125 * v12 * v22;
  }
}

/* Physical-space basis at one quadrature point: BasisFunctionsLagrange.cpp:18-97
 * (2D, closed-form inverse) and :101-186 (3D, determinant and inverse of the
 * 3x3 mapping gradient B(a,b) = d x_b / d xi_a, written here by cofactors). */
static void basis_phys(int et, int ndim, int npe, const double *xi, const double *X,
                       double *N, double *dx, double *dy, double *dz, double *Jac)
{
  double d1[8], d2[8], d3[8];
  basis_ref(et, xi, N, d1, d2, d3);
  if (ndim == 2) {
    double B00 = 0, B01 = 0, B10 = 0, B11 = 0;
    for (int ii = 0; ii < npe; ii++) {
      double xx = X[ii * 2 + 0], yy = X[ii * 2 + 1];
      B00 += (xx * d1[ii]); B10 += (xx * d2[ii]);
      B01 += (yy * d1[ii]); B11 += (yy * d2[ii]);
    }
    double J = B00 * B11 - B01 * B10;
    double detinv = 1.0 / J;
    double I00 = B11 * detinv, I01 = -B01 * detinv, I10 = -B10 * detinv, I11 = B00 * detinv;
    for (int ii = 0; ii < npe; ii++) {
      dx[ii] = d1[ii] * I00 + d2[ii] * I01;
      dy[ii] = d1[ii] * I10 + d2[ii] * I11;
    }
    *Jac = J;
  } else {
    double B[3][3] = {{0}};
    for (int ii = 0; ii < npe; ii++) {
      double xx = X[ii * 3 + 0], yy = X[ii * 3 + 1], zz = X[ii * 3 + 2];
      B[0][0] += (xx * d1[ii]); B[1][0] += (xx * d2[ii]); B[2][0] += (xx * d3[ii]);
      B[0][1] += (yy * d1[ii]); B[1][1] += (yy * d2[ii]); B[2][1] += (yy * d3[ii]);
      B[0][2] += (zz * d1[ii]); B[1][2] += (zz * d2[ii]); B[2][2] += (zz * d3[ii]);
    }
    /* cofactors C(i,j); inverse(i,j) = C(j,i)/det */
    double C[3][3];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
        C[i][j] = B[i1][j1] * B[i2][j2] - B[i1][j2] * B[i2][j1];
      }
    double J = B[0][0] * C[0][0] + B[0][1] * C[0][1] + B[0][2] * C[0][2];
    double invdet = 1.0 / J;
    double I[3][3];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) I[i][j] = C[j][i] * invdet;
    for (int ii = 0; ii < npe; ii++) {
      dx[ii] = d1[ii] * I[0][0] + d2[ii] * I[0][1] + d3[ii] * I[0][2];
      dy[ii] = d1[ii] * I[1][0] + d2[ii] * I[1][1] + d3[ii] * I[1][2];
      dz[ii] = d1[ii] * I[2][0] + d2[ii] * I[2][1] + d3[ii] * I[2][2];
    }
    *Jac = J;
  }
}

/*
 * One element: K (nsize x nsize, row-major, local index node*ndof+dof) and F.
 * X: npe*ndim coordinates; prev/cur/dotcur: npe*ndof nodal values of
 * solnPrev, solnCur, solnDotCur.  elemData as StabFEM::readControlParameters
 * fills it (StabFEM.cpp:285-294): [0]=rho, [1]=mu, [8..10]=SUPG/PSPG/LSIC.
 * td: SolutionData::td (UtilitiesGeneral.cpp:5-205).
 * info (optional, 2 doubles): elemVol, charlen.
 * Returns 0, or -1 for a negative Jacobian (the reference exits there).
 */
int orc_element(int et, const double *X, const double *prev, const double *cur,
                const double *dotcur, const double *elemData, const double *td,
                double *K, double *F, double *info)
{
  int ndim, npe, ngp;
  einfo(et, &ndim, &npe, &ngp);
  const int ndof = ndim + 1, nsize = npe * ndof;
  double gpx[8][3], gw[8];
  gauss_points(et, gpx, gw);

  /* prepareElemData */
  double Nv[8][8], Dx[8][8], Dy[8][8], Dz[8][8], dv[8];
  double elemVol = 0.0;
  int neg = 0;
  for (int gp = 0; gp < ngp; gp++) {
    double Jac;
    basis_phys(et, ndim, npe, gpx[gp], X, Nv[gp], Dx[gp], Dy[gp], Dz[gp], &Jac);
    if (Jac < 0.0) neg = 1;
    dv[gp] = gw[gp] * Jac;
    elemVol += dv[gp];
  }
  double charlen = (ndim == 2) ? sqrt(4.0 * fabs(elemVol) / ORC_PI)
                               : pow(6.0 * fabs(elemVol) / ORC_PI, 1.0 / 3.0);
  if (info) { info[0] = elemVol; info[1] = charlen; }

  /* calcStiffnessAndResidual (active semi-implicit type B routine) */
  const double CI = (ndim == 2) ? 4.0 : 10.0;
  const double cs = (et == ORC_HEX8) ? -1.0 : 1.0;   /* hex8 continuity row sign */
  const int supg = (ndim == 2);                       /* SUPG is commented out in 3D */
  double fact = 4.0 / charlen / charlen;
  double G[3] = {fact, fact, (ndim == 3) ? fact : 0.0};
  double sumG2 = G[0] * G[0] + G[1] * G[1] + G[2] * G[2];
  double trG = G[0] + G[1] + G[2];

  const double rho = elemData[0], mu = elemData[1];
  const double af = td[2], acceFact = td[8];
  const double muTaf = mu * af;

  memset(K, 0, sizeof(double) * nsize * nsize);
  memset(F, 0, sizeof(double) * nsize);

  for (int gp = 0; gp < ngp; gp++) {
    const double *N = Nv[gp];
    const double *dN[3] = {Dx[gp], Dy[gp], Dz[gp]};
    double velPrev[3] = {0, 0, 0}, vel[3] = {0, 0, 0}, velDot[3] = {0, 0, 0}, dp[3] = {0, 0, 0};
    double gradPrev[3][3] = {{0}}, grad[3][3] = {{0}};
    double pres = 0.0;
    for (int ii = 0; ii < npe; ii++) {
      const int TI = ii * ndof;
      for (int a = 0; a < ndim; a++) {
        double b = prev[TI + a];
        velPrev[a] += b * N[ii];
        for (int c = 0; c < ndim; c++) gradPrev[a][c] += b * dN[c][ii];
      }
      for (int a = 0; a < ndim; a++) {
        double b = cur[TI + a];
        vel[a] += b * N[ii];
        for (int c = 0; c < ndim; c++) grad[a][c] += b * dN[c][ii];
      }
      double b4 = cur[TI + ndim];
      pres += b4 * N[ii];
      for (int c = 0; c < ndim; c++) dp[c] += b4 * dN[c][ii];
      for (int a = 0; a < ndim; a++) velDot[a] += dotcur[TI + a] * N[ii];
    }
    double stress[3][3];
    for (int a = 0; a < ndim; a++)
      for (int c = 0; c < ndim; c++) stress[a][c] = mu * grad[a][c];
    for (int a = 0; a < ndim; a++) stress[a][a] -= pres;

    double gradTvel[3], res2[3], rStab[3];
    for (int a = 0; a < ndim; a++) {
      double t1 = 0, t2 = 0, t3 = 0;
      for (int c = 0; c < ndim; c++) {
        t1 += gradPrev[a][c] * vel[c];
        t2 += grad[a][c] * velPrev[c];
        t3 += gradPrev[a][c] * velPrev[c];
      }
      gradTvel[a] = t1 + t2 - t3;
    }
    for (int a = 0; a < ndim; a++) {
      res2[a] = rho * (velDot[a] + gradTvel[a] - 0.0);
      rStab[a] = res2[a] - mu * 0.0 + dp[a];
    }

    /* evaluateStabParams_algo3 at velPrev (3-vector, zero 3rd entry in 2D) */
    double uGu = 0.0;
    for (int a = 0; a < 3; a++) {
      double ua = (a < ndim) ? velPrev[a] : 0.0;
      uGu += ua * (G[a] * ua);
    }
    double tau0 = uGu + CI * (mu * mu / rho / rho) * sumG2;
    tau0 = 1.0 / sqrt(tau0);
    double tau2 = 1.0 / (tau0 * trG);
    tau0 = tau0 / rho;
    double tau1 = tau0;
    tau0 *= elemData[8];
    tau1 *= elemData[9];
    tau2 *= elemData[10];
    (void)tau2;                                   /* LSIC terms are commented out */

    const double dvol = dv[gp];
    for (int ii = 0; ii < npe; ii++) {
      const int TI = ndof * ii;
      double bb[3], b4, bm[3], b8;
      for (int a = 0; a < ndim; a++) bb[a] = dN[a][ii] * dvol;
      b4 = N[ii] * dvol;
      for (int a = 0; a < ndim; a++) bm[a] = muTaf * bb[a];
      b8 = af * b4;
      double Da = 0.0;
      for (int a = 0; a < ndim; a++) Da += velPrev[a] * bb[a];
      Da = rho * Da * tau0;

      for (int jj = 0; jj < npe; jj++) {
        const int TJ = ndof * jj;
        double fact2 = rho * acceFact * N[jj];
        double f = b4 * fact2;
        double dif = 0.0;
        for (int a = 0; a < ndim; a++) dif += bm[a] * dN[a][jj];
        f += dif;
        for (int a = 0; a < ndim; a++) K[(TI + a) * nsize + TJ + a] += f;

        double gradN[3][3];
        double rN = rho * N[jj];
        for (int a = 0; a < ndim; a++)
          for (int c = 0; c < ndim; c++) gradN[a][c] = gradPrev[a][c] * rN;
        double Db = 0.0;
        for (int a = 0; a < ndim; a++) Db += velPrev[a] * dN[a][jj];
        Db = rho * Db;
        for (int a = 0; a < ndim; a++) gradN[a][a] += Db;

        for (int a = 0; a < ndim; a++)
          for (int c = 0; c < ndim; c++) K[(TI + a) * nsize + TJ + c] += (b8 * gradN[a][c]);
        for (int a = 0; a < ndim; a++) K[(TI + a) * nsize + TJ + ndim] -= (bb[a] * af * N[jj]);
        for (int c = 0; c < ndim; c++) K[(TI + ndim) * nsize + TJ + c] += cs * (b8 * dN[c][jj]);

        for (int a = 0; a < ndim; a++)
          for (int c = 0; c < ndim; c++) gradN[a][c] *= af;
        double Dj[3][4];
        for (int a = 0; a < ndim; a++) {
          for (int c = 0; c < ndim; c++) Dj[a][c] = gradN[a][c] + ((a == c) ? fact2 : 0.0);
          Dj[a][ndim] = af * dN[a][jj];
        }
        if (supg) {
          for (int a = 0; a < ndim; a++)
            for (int c = 0; c <= ndim; c++) K[(TI + a) * nsize + TJ + c] += Da * Dj[a][c];
        }
        for (int c = 0; c <= ndim; c++) {
          double s = 0.0;
          for (int a = 0; a < ndim; a++) s += bb[a] * Dj[a][c];
          K[(TI + ndim) * nsize + TJ + c] += cs * (s * tau1);
        }
      }

      for (int a = 0; a < ndim; a++) {
        double s = b4 * res2[a];
        for (int c = 0; c < ndim; c++) s += bb[c] * stress[a][c];
        F[TI + a] -= s;
      }
      double tr = 0.0;
      for (int a = 0; a < ndim; a++) tr += grad[a][a];
      F[TI + ndim] -= cs * (b4 * tr);
      if (supg)
        for (int a = 0; a < ndim; a++) F[TI + a] -= Da * rStab[a];
      double s = 0.0;
      for (int a = 0; a < ndim; a++) s += bb[a] * rStab[a];
      F[TI + ndim] -= cs * (tau1 * s);
    }
  }
  return neg ? -1 : 0;
}

/*
 * Fully-implicit element routine: the reference's commented-out variant
 * "Fully-implicit formulation" (quad4 LagrangeElem2DNavierStokesQuad4Node.cpp:117-396,
 * tri3 LagrangeElem2DNavierStokesTria3Node.cpp:117-396, hex8
 * LagrangeElem3DNavierStokesHexa8Node.cpp:109-432, tet4
 * LagrangeElem3DNavierStokesTetra4Node.cpp:115-438).  Convection is
 * grad(u_cur) u_cur with its full Newton linearisation, SUPG and PSPG act on
 * the current velocity, LSIC is active in 3D (scaled by elemData[10]), and no
 * row is sign-flipped.  The 2D and 3D texts differ and are kept as written:
 * 2D SUPG has no rho factor and its pressure column carries af; 3D SUPG has
 * rho, its pressure column has no af; CI is 10 for hex8 and 4 otherwise.
 * Same arguments and return value as orc_element.
 */
int orc_element_fi(int et, const double *X, const double *prev, const double *cur,
                   const double *dotcur, const double *elemData, const double *td,
                   double *K, double *F, double *info)
{
  int ndim, npe, ngp;
  einfo(et, &ndim, &npe, &ngp);
  const int ndof = ndim + 1, nsize = npe * ndof;
  double gpx[8][3], gw[8];
  gauss_points(et, gpx, gw);

  double Nv[8][8], Dx[8][8], Dy[8][8], Dz[8][8], dv[8];
  double elemVol = 0.0;
  int neg = 0;
  for (int gp = 0; gp < ngp; gp++) {
    double Jac;
    basis_phys(et, ndim, npe, gpx[gp], X, Nv[gp], Dx[gp], Dy[gp], Dz[gp], &Jac);
    if (Jac < 0.0) neg = 1;
    dv[gp] = gw[gp] * Jac;
    elemVol += dv[gp];
  }
  double charlen = (ndim == 2) ? sqrt(4.0 * fabs(elemVol) / ORC_PI)
                               : pow(6.0 * fabs(elemVol) / ORC_PI, 1.0 / 3.0);
  if (info) { info[0] = elemVol; info[1] = charlen; }

  const double CI = (et == ORC_HEX8) ? 10.0 : 4.0;
  double fact = 4.0 / charlen / charlen;
  double G[3] = {fact, fact, (ndim == 3) ? fact : 0.0};
  double sumG2 = G[0] * G[0] + G[1] * G[1] + G[2] * G[2];
  double trG = G[0] + G[1] + G[2];

  const double rho = elemData[0], mu = elemData[1];
  const double af = td[2], acceFact = td[8];
  const double muTaf = mu * af;

  memset(K, 0, sizeof(double) * nsize * nsize);
  memset(F, 0, sizeof(double) * nsize);

  for (int gp = 0; gp < ngp; gp++) {
    const double *N = Nv[gp];
    const double *dN[3] = {Dx[gp], Dy[gp], Dz[gp]};
    double velPrev[3] = {0, 0, 0}, vel[3] = {0, 0, 0}, velDot[3] = {0, 0, 0}, dp[3] = {0, 0, 0};
    double grad[3][3] = {{0}};
    double pres = 0.0;
    for (int ii = 0; ii < npe; ii++) {
      const int TI = ii * ndof;
      for (int a = 0; a < ndim; a++) velPrev[a] += prev[TI + a] * N[ii];
      for (int a = 0; a < ndim; a++) {
        double b = cur[TI + a];
        vel[a] += b * N[ii];
        for (int c = 0; c < ndim; c++) grad[a][c] += b * dN[c][ii];
      }
      double b4 = cur[TI + ndim];
      pres += b4 * N[ii];
      for (int c = 0; c < ndim; c++) dp[c] += b4 * dN[c][ii];
      for (int a = 0; a < ndim; a++) velDot[a] += dotcur[TI + a] * N[ii];
    }
    double stress[3][3];
    for (int a = 0; a < ndim; a++)
      for (int c = 0; c < ndim; c++) stress[a][c] = mu * grad[a][c];
    for (int a = 0; a < ndim; a++) stress[a][a] -= pres;
    double res2[3], rStab[3], tr = 0.0;
    for (int a = 0; a < ndim; a++) {
      double g = 0.0;
      for (int c = 0; c < ndim; c++) g += grad[a][c] * vel[c];
      res2[a] = rho * (velDot[a] + g - 0.0);
      rStab[a] = res2[a] - mu * 0.0 + dp[a];
      tr += grad[a][a];
    }
    /* evaluateStabParams_algo3 at velPrev */
    double uGu = 0.0;
    for (int a = 0; a < 3; a++) {
      double ua = (a < ndim) ? velPrev[a] : 0.0;
      uGu += ua * (G[a] * ua);
    }
    double tau0 = uGu + CI * (mu * mu / rho / rho) * sumG2;
    tau0 = 1.0 / sqrt(tau0);
    double tau2 = 1.0 / (tau0 * trG);
    tau0 = tau0 / rho;
    double tau1 = tau0;
    tau0 *= elemData[8];
    tau1 *= elemData[9];
    tau2 *= elemData[10];

    const double dvol = dv[gp];
    for (int ii = 0; ii < npe; ii++) {
      const int TI = ndof * ii;
      double bb[3], b4, bm[3], b8;
      for (int a = 0; a < ndim; a++) bb[a] = dN[a][ii] * dvol;
      b4 = N[ii] * dvol;
      for (int a = 0; a < ndim; a++) bm[a] = muTaf * bb[a];
      b8 = af * b4;
      double Da = 0.0;
      for (int a = 0; a < ndim; a++) Da += vel[a] * bb[a];
      Da = (ndim == 3) ? Da * tau0 * rho : Da * tau0;

      for (int jj = 0; jj < npe; jj++) {
        const int TJ = ndof * jj;
        double fact2 = rho * acceFact * N[jj];
        double f = b4 * fact2;
        double dif = 0.0;
        for (int a = 0; a < ndim; a++) dif += bm[a] * dN[a][jj];
        f += dif;
        for (int a = 0; a < ndim; a++) K[(TI + a) * nsize + TJ + a] += f;

        double gradN[3][3];
        for (int a = 0; a < ndim; a++)
          for (int c = 0; c < ndim; c++) gradN[a][c] = grad[a][c] * (rho * N[jj]);
        double Db = 0.0;
        for (int a = 0; a < ndim; a++) Db += vel[a] * dN[a][jj];
        Db = rho * Db;
        for (int a = 0; a < ndim; a++) gradN[a][a] += Db;
        if (ndim == 3) {
          for (int a = 0; a < ndim; a++)
            for (int c = 0; c < ndim; c++) gradN[a][c] *= af;
          for (int a = 0; a < ndim; a++)
            for (int c = 0; c < ndim; c++) K[(TI + a) * nsize + TJ + c] += (b4 * gradN[a][c]);
          for (int a = 0; a < ndim; a++) K[(TI + a) * nsize + TJ + ndim] -= (bb[a] * N[jj]);
        } else {
          for (int a = 0; a < ndim; a++)
            for (int c = 0; c < ndim; c++) K[(TI + a) * nsize + TJ + c] += (b8 * gradN[a][c]);
          for (int a = 0; a < ndim; a++) K[(TI + a) * nsize + TJ + ndim] -= (bb[a] * af * N[jj]);
        }
        for (int c = 0; c < ndim; c++) K[(TI + ndim) * nsize + TJ + c] += (b8 * dN[c][jj]);
        if (ndim == 2)
          for (int a = 0; a < ndim; a++)
            for (int c = 0; c < ndim; c++) gradN[a][c] *= af;

        double Dj[3][4];
        for (int a = 0; a < ndim; a++) {
          for (int c = 0; c < ndim; c++) Dj[a][c] = gradN[a][c] + ((a == c) ? fact2 : 0.0);
          Dj[a][ndim] = af * dN[a][jj];
        }
        /* SUPG */
        for (int a = 0; a < ndim; a++)
          for (int c = 0; c <= ndim; c++) K[(TI + a) * nsize + TJ + c] += Da * Dj[a][c];
        const double c1 = (ndim == 3) ? tau0 * af * rho * N[jj] : (tau0 * af);
        for (int a = 0; a < ndim; a++)
          for (int c = 0; c < ndim; c++) {
            if (ndim == 3) K[(TI + a) * nsize + TJ + c] += (c1 * bb[c] * rStab[a]);
            else K[(TI + a) * nsize + TJ + c] += (c1 * bb[c] * rStab[a] * N[jj]);
          }
        /* PSPG */
        for (int c = 0; c <= ndim; c++) {
          double s = 0.0;
          for (int a = 0; a < ndim; a++) s += bb[a] * Dj[a][c];
          K[(TI + ndim) * nsize + TJ + c] += s * tau1;
        }
        /* LSIC (3D only; commented out in the 2D text) */
        if (ndim == 3) {
          double f2 = rho * af * tau2;
          for (int a = 0; a < ndim; a++)
            for (int c = 0; c < ndim; c++) K[(TI + a) * nsize + TJ + c] += (bb[a] * dN[c][jj]) * f2;
        }
      }

      for (int a = 0; a < ndim; a++) {
        double s = b4 * res2[a];
        for (int c = 0; c < ndim; c++) s += bb[c] * stress[a][c];
        F[TI + a] -= s;
      }
      F[TI + ndim] -= (b4 * tr);
      for (int a = 0; a < ndim; a++) F[TI + a] -= Da * rStab[a];
      double s = 0.0;
      for (int a = 0; a < ndim; a++) s += bb[a] * rStab[a];
      F[TI + ndim] -= (tau1 * s);
      if (ndim == 3) {
        double f2 = tau2 * rho * tr;
        for (int a = 0; a < ndim; a++) F[TI + a] -= bb[a] * f2;
      }
    }
  }
  return neg ? -1 : 0;
}

/* element formulation used by orc_assemble: 0 = semi-implicit type B (the
 * reference's active routine), 1 = fully implicit (orc_element_fi) */
static int g_form = 0;
void orc_set_formulation(int form) { g_form = form; }

/* ---------------- free-dof pattern (StabFEM2.cpp:57-81, 192-227) -------- */

/* node -> sorted unique neighbour nodes (nodes sharing an element) */
static int build_node_graph(int nNode, int nElem, int npe, const int *conn, int **nptr_out, int **nadj_out)
{
  int *ecount = calloc(nNode + 1, sizeof(int));
  for (int e = 0; e < nElem; e++)
    for (int a = 0; a < npe; a++) ecount[conn[e * npe + a] + 1]++;
  for (int n = 0; n < nNode; n++) ecount[n + 1] += ecount[n];
  int *elist = malloc(sizeof(int) * (size_t)ecount[nNode]);
  int *fill = calloc(nNode, sizeof(int));
  for (int e = 0; e < nElem; e++)
    for (int a = 0; a < npe; a++) {
      int n = conn[e * npe + a];
      elist[ecount[n] + fill[n]++] = e;
    }
  int *nptr = calloc(nNode + 1, sizeof(int));
  int *mark = malloc(sizeof(int) * nNode);
  for (int n = 0; n < nNode; n++) mark[n] = -1;
  /* count */
  for (int n = 0; n < nNode; n++) {
    int cnt = 0;
    for (int k = ecount[n]; k < ecount[n + 1]; k++) {
      int e = elist[k];
      for (int a = 0; a < npe; a++) {
        int m = conn[e * npe + a];
        if (mark[m] != n) { mark[m] = n; cnt++; }
      }
    }
    nptr[n + 1] = nptr[n] + cnt;
  }
  int *nadj = malloc(sizeof(int) * (size_t)nptr[nNode]);
  for (int n = 0; n < nNode; n++) mark[n] = -1;
  for (int n = 0; n < nNode; n++) {
    int pos = nptr[n];
    for (int k = ecount[n]; k < ecount[n + 1]; k++) {
      int e = elist[k];
      for (int a = 0; a < npe; a++) {
        int m = conn[e * npe + a];
        if (mark[m] != n) { mark[m] = n; nadj[pos++] = m; }
      }
    }
    /* insertion sort (short lists) */
    for (int i = nptr[n] + 1; i < nptr[n + 1]; i++) {
      int v = nadj[i], j = i - 1;
      while (j >= nptr[n] && nadj[j] > v) { nadj[j + 1] = nadj[j]; j--; }
      nadj[j + 1] = v;
    }
  }
  free(ecount); free(elist); free(fill); free(mark);
  *nptr_out = nptr; *nadj_out = nadj;
  return 0;
}

/* dofmap[n*ndof+d] = free index or -1.  Pass colidx == NULL to only count:
 * returns nnz.  rowptr has ntot+1 entries. */
long orc_pattern(int nNode, int ndof, int nElem, int npe, const int *conn, const int *dofmap,
                 int ntot, int *rowptr, int *colidx)
{
  int *nptr, *nadj;
  build_node_graph(nNode, nElem, npe, conn, &nptr, &nadj);
  long nnz = 0;
  for (int n = 0; n < nNode; n++) {
    for (int d = 0; d < ndof; d++) {
      int r = dofmap[n * ndof + d];
      if (r < 0) continue;
      rowptr[r] = (int)nnz;
      for (int k = nptr[n]; k < nptr[n + 1]; k++) {
        int m = nadj[k];
        for (int e2 = 0; e2 < ndof; e2++) {
          int c = dofmap[m * ndof + e2];
          if (c < 0) continue;
          if (colidx) colidx[nnz] = c;
          nnz++;
        }
      }
    }
  }
  rowptr[ntot] = (int)nnz;
  free(nptr); free(nadj);
  return nnz;
}

/* ---------------- assembly into the free-dof CSR ---------------- */
static inline int find_col(const int *colidx, int lo, int hi, int c)
{
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (colidx[mid] < c) lo = mid + 1; else hi = mid;
  }
  return lo;
}

static int assemble_one(int et, int e, int ndim, int npe, const int *conn, const double *coords,
                        const int *dofmap, const double *solnPrev, const double *solnCur,
                        const double *solnDotCur, const double *solnApplied,
                        const double *elemData, const double *td, int iter, int want_K,
                        const int *rowptr, const int *colidx, double *vals, double *rhs)
{
  const int ndof = ndim + 1, nsize = npe * ndof;
  double X[24], pv[32], cv[32], dc[32], K[32 * 32], F[32];
  int fa[32], gdof[32];
  for (int a = 0; a < npe; a++) {
    int n = conn[e * npe + a];
    for (int c = 0; c < ndim; c++) X[a * ndim + c] = coords[(size_t)n * ndim + c];
    for (int d = 0; d < ndof; d++) {
      size_t g = (size_t)n * ndof + d;
      pv[a * ndof + d] = solnPrev[g];
      cv[a * ndof + d] = solnCur[g];
      dc[a * ndof + d] = solnDotCur[g];
      fa[a * ndof + d] = dofmap[g];
      gdof[a * ndof + d] = (int)g;
    }
  }
  int rc = g_form ? orc_element_fi(et, X, pv, cv, dc, elemData, td, K, F, NULL)
                  : orc_element(et, X, pv, cv, dc, elemData, td, K, F, NULL);
  if (iter == 0) {                                  /* StabFEM2.cpp:678-703 */
    for (int ii = 0; ii < nsize; ii++) {
      if (fa[ii] == -1) {
        double fact = solnApplied[gdof[ii]];
        if (fabs(fact) > 1.0e-10) {
          for (int jj = 0; jj < nsize; jj++)
            if (fa[jj] != -1) F[jj] -= K[jj * nsize + ii] * fact;
        }
      }
    }
  }
  for (int ii = 0; ii < nsize; ii++) {              /* SolverPetsc.cpp:304-314 */
    int r = fa[ii];
    if (r < 0) continue;
    rhs[r] += F[ii];
    if (!want_K) continue;
    int lo = rowptr[r], hi = rowptr[r + 1];
    for (int jj = 0; jj < nsize; jj++) {
      int c = fa[jj];
      if (c < 0) continue;
      int p = find_col(colidx, lo, hi, c);
      vals[p] += K[ii * nsize + jj];
    }
  }
  return rc;
}

/*
 * Assemble all elements for one Newton iteration (StabFEM2.cpp:669-708).
 * vals/rhs are zeroed here (SolverPetsc::zeroMtx).  With ncolors == 0 the
 * elements run serially in element order (the reference's order); with a
 * colouring (color_ptr/color_elems) they run colour by colour, in parallel
 * inside a colour, so every entry receives its sums in a fixed order.
 * want_K == 0 assembles only the residual.  Returns the number of elements
 * with a negative Jacobian.
 */
int orc_assemble(int et, int nNode, int nElem, const int *conn, const double *coords,
                 const int *dofmap, const double *solnPrev, const double *solnCur,
                 const double *solnDotCur, const double *solnApplied, const double *elemData,
                 const double *td, int iter, int want_K, const int *rowptr, const int *colidx,
                 long nnz, double *vals, int ntot, double *rhs, int ncolors,
                 const int *color_ptr, const int *color_elems, int nthreads)
{
  int ndim, npe, ngp;
  einfo(et, &ndim, &npe, &ngp);
  (void)nNode;
  if (want_K) memset(vals, 0, sizeof(double) * (size_t)nnz);
  memset(rhs, 0, sizeof(double) * (size_t)ntot);
  int nneg = 0;
  if (ncolors <= 0) {
    for (int e = 0; e < nElem; e++)
      nneg += assemble_one(et, e, ndim, npe, conn, coords, dofmap, solnPrev, solnCur, solnDotCur,
                           solnApplied, elemData, td, iter, want_K, rowptr, colidx, vals, rhs) != 0;
  } else {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    for (int c = 0; c < ncolors; c++) {
      int lo = color_ptr[c], hi = color_ptr[c + 1];
      int neg_c = 0;
#pragma omp parallel for schedule(static) reduction(+ : neg_c)
      for (int k = lo; k < hi; k++)
        neg_c += assemble_one(et, color_elems[k], ndim, npe, conn, coords, dofmap, solnPrev, solnCur,
                              solnDotCur, solnApplied, elemData, td, iter, want_K, rowptr, colidx,
                              vals, rhs) != 0;
      nneg += neg_c;
    }
  }
  return nneg;
}

/* ---------------- vector kernels ---------------- */
static double vdot(int n, const double *a, const double *b)
{
  double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s)
  for (int i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

double orc_norm2(int n, const double *a) { return sqrt(vdot(n, a, a)); }

static void spmv(int n, const int *rowptr, const int *colidx, const double *vals, const double *x, double *y)
{
#pragma omp parallel for schedule(static)
  for (int r = 0; r < n; r++) {
    double s = 0.0;
    for (int k = rowptr[r]; k < rowptr[r + 1]; k++) s += vals[k] * x[colidx[k]];
    y[r] = s;
  }
}

void orc_spmv(int n, const int *rowptr, const int *colidx, const double *vals, const double *x, double *y, int nthreads)
{
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  spmv(n, rowptr, colidx, vals, x, y);
}

/* Point-block Jacobi blocks for pc == 2: runs of consecutive free dofs that
 * belong to one node (the free numbering is node-major, so a node's free
 * dofs are contiguous).  Set by orc_set_blocks before orc_gmres. */
static int g_nblk = 0;
static const int *g_blk_ptr = NULL;

void orc_set_blocks(int nblk, const int *blk_ptr) { g_nblk = nblk; g_blk_ptr = blk_ptr; }

/* invert a small dense row-major block in place (Gauss-Jordan, partial pivoting) */
static int small_inverse(int b, double *A)
{
  double inv[16];
  for (int i = 0; i < b * b; i++) inv[i] = 0.0;
  for (int i = 0; i < b; i++) inv[i * b + i] = 1.0;
  for (int c = 0; c < b; c++) {
    int piv = c;
    for (int r = c + 1; r < b; r++) if (fabs(A[r * b + c]) > fabs(A[piv * b + c])) piv = r;
    if (A[piv * b + c] == 0.0) return -1;
    if (piv != c)
      for (int k = 0; k < b; k++) {
        double t = A[c * b + k]; A[c * b + k] = A[piv * b + k]; A[piv * b + k] = t;
        t = inv[c * b + k]; inv[c * b + k] = inv[piv * b + k]; inv[piv * b + k] = t;
      }
    double d = 1.0 / A[c * b + c];
    for (int k = 0; k < b; k++) { A[c * b + k] *= d; inv[c * b + k] *= d; }
    for (int r = 0; r < b; r++) {
      if (r == c) continue;
      double f = A[r * b + c];
      if (f == 0.0) continue;
      for (int k = 0; k < b; k++) { A[r * b + k] -= f * A[c * b + k]; inv[r * b + k] -= f * inv[c * b + k]; }
    }
  }
  for (int i = 0; i < b * b; i++) A[i] = inv[i];
  return 0;
}

/* ---------------- block Jacobi with ILU(k) blocks ----------------
 *
 * PETSc's PCBJACOBI with sub-KSP preonly and sub-PC ILU(levels), the
 * preconditioner of the reference's iterative option files
 * (input/petsc_options_gmres.dat:2-5, input/petsc_options_bcgs.dat:2-5, read
 * through SolverPetsc.cpp:101,111).  PETSc is not part of the reference tree;
 * this restates its published algorithm: the matrix is cut into diagonal
 * blocks of contiguous rows (one per MPI rank in the reference, or the
 * -pc_bjacobi_blocks count), couplings between blocks are dropped, and each
 * block gets an incomplete LU factorisation in natural ordering with
 * level-of-fill k (MatILUFactorSymbolic_SeqAIJ: lev(i,j) = min over pivots p
 * of lev(i,p) + lev(p,j) + 1, entries of A at level 0, fill kept while
 * lev <= k) followed by row-oriented numeric elimination
 * (MatLUFactorNumeric_SeqAIJ: for row i, for each pivot p < i in the row's
 * pattern in increasing order, l = w_p / u_pp, w_j -= l u_pj on the row's
 * pattern).  Applying it solves L y = r (unit lower) and U z = y per block.
 * The factors live in one CSR over all rows (block-local columns only).
 * A very large level limit keeps all fill: the complete LU (-pc_type lu).
 */
typedef struct {
  int n, nblk, levels;
  int *blk;              /* nblk+1 row offsets */
  int *fptr, *fcol;      /* factored pattern (sorted columns), n+1 / nnz */
  int *fdiag;            /* position of the diagonal in each row */
  double *fval;          /* L (unit, strict lower) and U (upper incl. diagonal) */
  long nnz;
  int zero_pivot_row;    /* first row with a zero pivot, -1 if none */
  /* level sets: rows whose lower (upper) dependencies all lie in earlier
   * sets; rows inside a set are independent, so the factorisation and the
   * lower solve run set by set over lrows, the upper solve over urows, each
   * row with the same arithmetic as in row order */
  int nlev_l, nlev_u;
  int *lptr, *lrows, *uptr, *urows;
} orc_ilu_t;

static orc_ilu_t g_ilu = {0};

static void ilu_free(orc_ilu_t *f)
{
  free(f->blk); free(f->fptr); free(f->fcol); free(f->fdiag); free(f->fval);
  free(f->lptr); free(f->lrows); free(f->uptr); free(f->urows);
  memset(f, 0, sizeof(*f));
}

/* group rows by level: lev[] per row -> (ptr[nlev+1], rows[n]), row order
 * inside a level */
static int level_sets(int n, const int *lev, int **ptr_out, int **rows_out)
{
  int nlev = 0;
  for (int i = 0; i < n; i++) if (lev[i] + 1 > nlev) nlev = lev[i] + 1;
  int *ptr = calloc((size_t)nlev + 1, sizeof(int));
  int *rows = malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; i++) ptr[lev[i] + 1]++;
  for (int k = 0; k < nlev; k++) ptr[k + 1] += ptr[k];
  int *fill = calloc((size_t)nlev + 1, sizeof(int));
  for (int i = 0; i < n; i++) rows[ptr[lev[i]] + fill[lev[i]]++] = i;
  free(fill);
  *ptr_out = ptr; *rows_out = rows;
  return nlev;
}

/* Symbolic ILU(levels) of the diagonal blocks of the CSR (rowptr, colidx),
 * blocks given as nblk+1 row offsets.  Returns nnz of the factors. */
long orc_ilu_symbolic(int n, const int *rowptr, const int *colidx, int nblk, const int *blk, int levels)
{
  ilu_free(&g_ilu);
  orc_ilu_t *f = &g_ilu;
  f->n = n; f->nblk = nblk; f->levels = levels; f->zero_pivot_row = -1;
  f->blk = malloc(sizeof(int) * (nblk + 1));
  memcpy(f->blk, blk, sizeof(int) * (nblk + 1));
  long cap = (long)rowptr[n] + 16;
  int *col = malloc(sizeof(int) * cap);
  int *lev = malloc(sizeof(int) * cap);      /* level of each stored entry */
  int *ptr = malloc(sizeof(int) * (n + 1));
  int *dg = malloc(sizeof(int) * (n > 0 ? n : 1));
  int *next = malloc(sizeof(int) * (n + 1)); /* sorted linked list over columns, n = end marker */
  int *lv = malloc(sizeof(int) * (n > 0 ? n : 1));
  long nnz = 0;
  ptr[0] = 0;
  for (int b = 0; b < nblk; b++) {
    const int r0 = blk[b], r1 = blk[b + 1];
    for (int i = r0; i < r1; i++) {
      /* row i of A inside the block, level 0 */
      int head = n, tail = -1;
      for (int k = rowptr[i]; k < rowptr[i + 1]; k++) {
        int c = colidx[k];
        if (c < r0 || c >= r1) continue;
        lv[c] = 0;
        if (tail < 0) head = c; else next[tail] = c;
        tail = c;
      }
      if (tail >= 0) next[tail] = n;
      /* eliminate pivots p < i in increasing order */
      for (int p = head; p < i; p = next[p]) {
        const int lp = lv[p];
        if (lp + 1 > levels) continue;
        int ins = p;   /* list position to search from: U columns of row p are > p, ascending */
        for (long q = dg[p] + 1; q < ptr[p + 1]; q++) {
          const int j = col[q];
          const int l = lp + lev[q] + 1;
          if (l > levels) continue;
          while (next[ins] < j) ins = next[ins];
          if (next[ins] == j) { if (l < lv[j]) lv[j] = l; }
          else { next[j] = next[ins]; next[ins] = j; lv[j] = l; }
          ins = j;
        }
      }
      /* store row i */
      long cnt = 0;
      for (int c = head; c < n; c = next[c]) cnt++;
      if (nnz + cnt > cap) {
        while (nnz + cnt > cap) cap *= 2;
        col = realloc(col, sizeof(int) * cap);
        lev = realloc(lev, sizeof(int) * cap);
      }
      dg[i] = -1;
      for (int c = head; c < n; c = next[c]) {
        if (c == i) dg[i] = (int)nnz;
        col[nnz] = c; lev[nnz] = lv[c]; nnz++;
      }
      ptr[i + 1] = (int)nnz;
    }
  }
  free(next); free(lv); free(lev);
  f->fptr = ptr; f->fcol = col; f->fdiag = dg; f->nnz = nnz;
  f->fval = calloc((size_t)(nnz > 0 ? nnz : 1), sizeof(double));
  /* dependency levels of the factorisation / lower solve (ascending) and of
   * the upper solve (descending) */
  int *dl = malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; i++) {
    int d = 0;
    for (int q = ptr[i]; q < dg[i]; q++) if (dl[col[q]] + 1 > d) d = dl[col[q]] + 1;
    dl[i] = d;
  }
  f->nlev_l = level_sets(n, dl, &f->lptr, &f->lrows);
  for (int i = n - 1; i >= 0; i--) {
    int d = 0;
    for (int q = dg[i] + 1; q < ptr[i + 1]; q++) if (dl[col[q]] + 1 > d) d = dl[col[q]] + 1;
    dl[i] = d;
  }
  f->nlev_u = level_sets(n, dl, &f->uptr, &f->urows);
  free(dl);
  return nnz;
}

/* export the factored pattern (rowptr n+1, colidx nnz, diag n) */
void orc_ilu_pattern(int *fptr, int *fcol, int *fdiag)
{
  const orc_ilu_t *f = &g_ilu;
  if (fptr) memcpy(fptr, f->fptr, sizeof(int) * (f->n + 1));
  if (fcol) memcpy(fcol, f->fcol, sizeof(int) * f->nnz);
  if (fdiag) memcpy(fdiag, f->fdiag, sizeof(int) * f->n);
}

/* Numeric ILU of (rowptr, colidx, vals) on the symbolic pattern, level set by
 * level set (rows of a set in parallel).  Returns 0, or -1 on a zero pivot
 * (the reference's PETSc would stop with a zero-pivot error). */
int orc_ilu_numeric(const int *rowptr, const int *colidx, const double *vals, int nthreads)
{
  orc_ilu_t *f = &g_ilu;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  const int n = f->n;
  int *blk_of = malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for (int b = 0; b < f->nblk; b++)
    for (int i = f->blk[b]; i < f->blk[b + 1]; i++) blk_of[i] = b;
  int bad = n;
#pragma omp parallel
  {
    double *w = calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    int mybad = n;
    for (int k = 0; k < f->nlev_l; k++) {
#pragma omp for schedule(static)
      for (int t = f->lptr[k]; t < f->lptr[k + 1]; t++) {
        const int i = f->lrows[t];
        const int r0 = f->blk[blk_of[i]], r1 = f->blk[blk_of[i] + 1];
        for (int q = f->fptr[i]; q < f->fptr[i + 1]; q++) w[f->fcol[q]] = 0.0;
        for (int kk = rowptr[i]; kk < rowptr[i + 1]; kk++) {
          int c = colidx[kk];
          if (c >= r0 && c < r1) w[c] = vals[kk];
        }
        for (int q = f->fptr[i]; q < f->fdiag[i]; q++) {
          const int p = f->fcol[q];
          const double l = w[p] / f->fval[f->fdiag[p]];
          w[p] = l;
          if (l != 0.0)
            for (int u = f->fdiag[p] + 1; u < f->fptr[p + 1]; u++) w[f->fcol[u]] -= l * f->fval[u];
        }
        for (int q = f->fptr[i]; q < f->fptr[i + 1]; q++) f->fval[q] = w[f->fcol[q]];
        if (f->fdiag[i] < 0 || f->fval[f->fdiag[i]] == 0.0) { if (i < mybad) mybad = i; }
      }
    }
    free(w);
#pragma omp critical
    if (mybad < bad) bad = mybad;
  }
  free(blk_of);
  f->zero_pivot_row = (bad < n) ? bad : -1;
  return (bad < n) ? -1 : 0;
}

int orc_ilu_zero_pivot_row(void) { return g_ilu.zero_pivot_row; }

/* z = (LU)^-1 r (every block at once: blocks share no dependencies) */
static void ilu_apply(const double *r, double *z)
{
  const orc_ilu_t *f = &g_ilu;
#pragma omp parallel
  {
    for (int k = 0; k < f->nlev_l; k++) {
#pragma omp for schedule(static)
      for (int t = f->lptr[k]; t < f->lptr[k + 1]; t++) {
        const int i = f->lrows[t];
        double s = r[i];
        for (int q = f->fptr[i]; q < f->fdiag[i]; q++) s -= f->fval[q] * z[f->fcol[q]];
        z[i] = s;
      }
    }
    for (int k = 0; k < f->nlev_u; k++) {
#pragma omp for schedule(static)
      for (int t = f->uptr[k]; t < f->uptr[k + 1]; t++) {
        const int i = f->urows[t];
        double s = z[i];
        for (int q = f->fdiag[i] + 1; q < f->fptr[i + 1]; q++) s -= f->fval[q] * z[f->fcol[q]];
        z[i] = s / f->fval[f->fdiag[i]];
      }
    }
  }
}

void orc_ilu_apply(const double *r, double *z, int nthreads)
{
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  ilu_apply(r, z);
}

/* export the factor values (nnz) */
void orc_ilu_values(double *v)
{
  memcpy(v, g_ilu.fval, sizeof(double) * g_ilu.nnz);
}

/* PETSc KSPConvergedReason values used here */
#define R_ITERATING 0
#define R_RTOL 2
#define R_ATOL 3
#define R_DIV_NULL (-2)
#define R_DIV_ITS (-3)
#define R_DIV_DTOL (-4)
#define R_DIV_BREAKDOWN (-5)
#define R_DIV_NANORINF (-9)

static void pc_apply(int n, int pc, const double *dinv, const double *binv, const double *r, double *z)
{
  if (pc == 3) { ilu_apply(r, z); return; }
  if (pc != 2) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) z[i] = dinv[i] * r[i];
    return;
  }
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g_nblk; k++) {
    int r0 = g_blk_ptr[k], bs = g_blk_ptr[k + 1] - r0;
    const double *B = binv + (size_t)k * 16;
    for (int i = 0; i < bs; i++) {
      double s = 0.0;
      for (int j = 0; j < bs; j++) s += B[i * bs + j] * r[r0 + j];
      z[r0 + i] = s;
    }
  }
}

typedef struct {
  double rnorm0, ttol;
  double rtol, atol, dtol;
} conv_ctx;

static int converged(conv_ctx *c, int n_its, double rnorm)
{
  if (n_its == 0) { c->rnorm0 = rnorm; c->ttol = fmax(c->rtol * rnorm, c->atol); }
  if (rnorm != rnorm || isinf(rnorm)) return R_DIV_NANORINF;
  if (rnorm <= c->ttol) return (rnorm < c->atol) ? R_ATOL : R_RTOL;
  if (rnorm >= c->dtol * c->rnorm0) return R_DIV_DTOL;
  return R_ITERATING;
}

/*
 * GMRES(restart) with left preconditioning (pc: 0 none, 1 jacobi, 2 point-block
 * jacobi over the blocks set by orc_set_blocks), x0 = 0.
 * Follows PETSc 3.10 KSPSolve_GMRES / KSPGMRESCycle /
 * KSPGMRESClassicalGramSchmidtOrthogonalization / KSPGMRESUpdateHessenberg /
 * KSPGMRESBuildSoln.  Returns the KSPConvergedReason; *its_out the iteration
 * count, *rnorm_out the last preconditioned residual norm.
 */
int orc_gmres(int n, const int *rowptr, const int *colidx, const double *vals, int pc,
              const double *b, double *x, int restart, double rtol, double atol, double dtol,
              int maxit, int *its_out, double *rnorm_out, int nthreads)
{
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  const int m = restart;
  const double haptol = 1.0e-30;
  double *dinv = malloc(sizeof(double) * n);
  for (int r = 0; r < n; r++) {
    double d = 0.0;
    for (int k = rowptr[r]; k < rowptr[r + 1]; k++)
      if (colidx[k] == r) d = vals[k];
    dinv[r] = (pc == 1) ? ((d != 0.0) ? 1.0 / d : 1.0) : 1.0;
  }
  double *binv = NULL;
  if (pc == 2) {
    binv = calloc((size_t)g_nblk * 16, sizeof(double));
    for (int k = 0; k < g_nblk; k++) {
      int r0 = g_blk_ptr[k], bs = g_blk_ptr[k + 1] - r0;
      double *B = binv + (size_t)k * 16;
      for (int i = 0; i < bs; i++)
        for (int p = rowptr[r0 + i]; p < rowptr[r0 + i + 1]; p++) {
          int c = colidx[p];
          if (c >= r0 && c < r0 + bs) B[i * bs + (c - r0)] = vals[p];
        }
      small_inverse(bs, B);
    }
  }
  double *V = malloc(sizeof(double) * (size_t)n * (m + 1));
  double *tmp = malloc(sizeof(double) * n);
  double *H = calloc((size_t)(m + 1) * m, sizeof(double));   /* H[row*m + col] */
  double *cc = calloc(m, sizeof(double)), *ss = calloc(m, sizeof(double));
  double *grs = calloc(m + 1, sizeof(double)), *nrs = calloc(m, sizeof(double));
  double *hh = calloc(m + 1, sizeof(double));
  conv_ctx cv = {0, 0, rtol, atol, dtol};
  memset(x, 0, sizeof(double) * n);
  int its = 0, reason = R_ITERATING, first = 1;
  double res = 0.0;

  while (reason == R_ITERATING) {
    /* KSPInitialResidual: r = b - A x (b when x0 = 0), then v0 = M^-1 r */
    if (first) {
#pragma omp parallel for schedule(static)
      for (int i = 0; i < n; i++) tmp[i] = b[i];
    } else {
      spmv(n, rowptr, colidx, vals, x, tmp);
#pragma omp parallel for schedule(static)
      for (int i = 0; i < n; i++) tmp[i] = b[i] - tmp[i];
    }
    pc_apply(n, pc, dinv, binv, tmp, V);
    first = 0;
    /* KSPGMRESCycle */
    res = sqrt(vdot(n, V, V));
    if (res != 0.0) {
      double sc = 1.0 / res;
#pragma omp parallel for schedule(static)
      for (int i = 0; i < n; i++) V[i] *= sc;
    }
    grs[0] = res;
    int it = 0;
    if (res == 0.0) { if (its == 0) { cv.rnorm0 = 0; } reason = R_ATOL; break; }
    reason = converged(&cv, its, res);
    while (reason == R_ITERATING && it < m && its < maxit) {
      double *vi = V + (size_t)n * it, *w = V + (size_t)n * (it + 1);
      spmv(n, rowptr, colidx, vals, vi, tmp);
      pc_apply(n, pc, dinv, binv, tmp, w);
      /* classical Gram-Schmidt */
      for (int j = 0; j <= it; j++) hh[j] = vdot(n, w, V + (size_t)n * j);
#pragma omp parallel for schedule(static)
      for (int i = 0; i < n; i++) {
        double s = w[i];
        for (int j = 0; j <= it; j++) s += (-hh[j]) * V[(size_t)n * j + i];
        w[i] = s;
      }
      for (int j = 0; j <= it; j++) H[j * m + it] = hh[j];
      double tt = sqrt(vdot(n, w, w));
      if (tt != 0.0) {
        double sc = 1.0 / tt;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) w[i] *= sc;
      }
      H[(it + 1) * m + it] = tt;
      double hapbnd = fabs(tt / grs[it]);
      if (hapbnd > haptol) hapbnd = haptol;
      int hapend = (tt < hapbnd);
      /* KSPGMRESUpdateHessenberg */
      for (int j = 1; j <= it; j++) {
        double t = H[(j - 1) * m + it];
        H[(j - 1) * m + it] = cc[j - 1] * t + ss[j - 1] * H[j * m + it];
        H[j * m + it] = cc[j - 1] * H[j * m + it] - ss[j - 1] * t;
      }
      if (!hapend) {
        double a = H[it * m + it], bq = H[(it + 1) * m + it];
        double t = sqrt(a * a + bq * bq);
        if (t == 0.0) { reason = R_DIV_NULL; break; }
        cc[it] = a / t;
        ss[it] = bq / t;
        grs[it + 1] = -(ss[it] * grs[it]);
        grs[it] = cc[it] * grs[it];
        H[it * m + it] = cc[it] * a + ss[it] * bq;
        res = fabs(grs[it + 1]);
      } else {
        res = 0.0;
      }
      it++;
      its++;
      reason = converged(&cv, its, res);
      if (hapend && reason == R_ITERATING) { reason = R_DIV_BREAKDOWN; break; }
    }
    /* KSPGMRESBuildSoln with it-1 */
    int last = it - 1;
    if (last >= 0) {
      if (H[last * m + last] != 0.0) nrs[last] = grs[last] / H[last * m + last];
      else nrs[last] = 0.0;
      for (int ii = 1; ii <= last; ii++) {
        int k = last - ii;
        double t = grs[k];
        for (int j = k + 1; j <= last; j++) t = t - H[k * m + j] * nrs[j];
        nrs[k] = (H[k * m + k] != 0.0) ? t / H[k * m + k] : 0.0;
      }
#pragma omp parallel for schedule(static)
      for (int i = 0; i < n; i++) {
        double s = 0.0;
        for (int j = 0; j <= last; j++) s += nrs[j] * V[(size_t)n * j + i];
        x[i] += s;
      }
    }
    if (reason != R_ITERATING) break;
    if (its >= maxit) { reason = R_DIV_ITS; break; }
  }
  if (its_out) *its_out = its;
  if (rnorm_out) *rnorm_out = res;
  free(dinv); free(binv); free(V); free(tmp); free(H); free(cc); free(ss); free(grs); free(nrs); free(hh);
  return reason;
}

/*
 * BiCGStab with left preconditioning (pc as in orc_gmres, 3 = the ILU set up
 * by orc_ilu_symbolic/numeric), x0 = 0: PETSc 3.10 KSPSolve_BCGS, the solver
 * of input/petsc_options_bcgs.dat:1 (third-party code, not in the reference
 * tree; published algorithm restated).  The convergence test uses the
 * preconditioned residual norm with KSPConvergedDefault; breakdowns (zero
 * (v, rp), zero rho) end the solve with KSP_DIVERGED_BREAKDOWN.  Returns the
 * KSPConvergedReason.
 */
int orc_bcgs(int n, const int *rowptr, const int *colidx, const double *vals, int pc,
             const double *b, double *x, double rtol, double atol, double dtol,
             int maxit, int *its_out, double *rnorm_out, int nthreads)
{
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  double *dinv = malloc(sizeof(double) * n);
  for (int r = 0; r < n; r++) {
    double d = 0.0;
    for (int k = rowptr[r]; k < rowptr[r + 1]; k++)
      if (colidx[k] == r) d = vals[k];
    dinv[r] = (pc == 1) ? ((d != 0.0) ? 1.0 / d : 1.0) : 1.0;
  }
  double *binv = NULL;
  if (pc == 2) {
    binv = calloc((size_t)g_nblk * 16, sizeof(double));
    for (int k = 0; k < g_nblk; k++) {
      int r0 = g_blk_ptr[k], bs = g_blk_ptr[k + 1] - r0;
      double *B = binv + (size_t)k * 16;
      for (int i = 0; i < bs; i++)
        for (int p = rowptr[r0 + i]; p < rowptr[r0 + i + 1]; p++) {
          int c = colidx[p];
          if (c >= r0 && c < r0 + bs) B[i * bs + (c - r0)] = vals[p];
        }
      small_inverse(bs, B);
    }
  }
  double *R = malloc(sizeof(double) * n), *RP = malloc(sizeof(double) * n), *V = calloc(n, sizeof(double));
  double *T = malloc(sizeof(double) * n), *S = malloc(sizeof(double) * n), *P = calloc(n, sizeof(double));
  conv_ctx cv = {0, 0, rtol, atol, dtol};
  memset(x, 0, sizeof(double) * n);
  /* r = M^-1 b (x0 = 0) */
  pc_apply(n, pc, dinv, binv, b, R);
  double dp = sqrt(vdot(n, R, R));
  int its = 0;
  int reason = converged(&cv, 0, dp);
  if (reason == R_ITERATING) {
    memcpy(RP, R, sizeof(double) * n);
    double rhoold = 1.0, alpha = 1.0, omegaold = 1.0;
    int i = 0;
    do {
      const double rho = vdot(n, R, RP);
      const double beta = (rho / rhoold) * (alpha / omegaold);
#pragma omp parallel for schedule(static)
      for (int k = 0; k < n; k++) P[k] = 1.0 * R[k] + (-omegaold * beta) * V[k] + beta * P[k];
      spmv(n, rowptr, colidx, vals, P, T);
      pc_apply(n, pc, dinv, binv, T, V);
      double d1 = vdot(n, V, RP);
      if (d1 != d1 || isinf(d1)) { reason = R_DIV_NANORINF; break; }
      if (d1 == 0.0) { reason = R_DIV_BREAKDOWN; break; }
      alpha = rho / d1;
#pragma omp parallel for schedule(static)
      for (int k = 0; k < n; k++) S[k] = -alpha * V[k] + R[k];
      spmv(n, rowptr, colidx, vals, S, R);
      pc_apply(n, pc, dinv, binv, R, T);
      d1 = vdot(n, S, T);
      const double d2 = vdot(n, T, T);
      if (d2 == 0.0) {
        if (vdot(n, S, S) != 0.0) { reason = R_DIV_BREAKDOWN; break; }
#pragma omp parallel for schedule(static)
        for (int k = 0; k < n; k++) x[k] += alpha * P[k];
        its++;
        dp = 0.0;
        reason = R_RTOL;
        break;
      }
      const double omega = d1 / d2;
#pragma omp parallel for schedule(static)
      for (int k = 0; k < n; k++) {
        x[k] = alpha * P[k] + omega * S[k] + 1.0 * x[k];
        R[k] = -omega * T[k] + S[k];
      }
      dp = sqrt(vdot(n, R, R));
      rhoold = rho;
      omegaold = omega;
      its++;
      reason = converged(&cv, its, dp);
      if (reason != R_ITERATING) break;
      if (rho == 0.0) { reason = R_DIV_BREAKDOWN; break; }
      i++;
    } while (i < maxit);
    if (reason == R_ITERATING) reason = R_DIV_ITS;
  }
  if (its_out) *its_out = its;
  if (rnorm_out) *rnorm_out = dp;
  free(dinv); free(binv); free(R); free(RP); free(V); free(T); free(S); free(P);
  return reason;
}

/* greedy element colouring: elements that share a node get different
 * colours; elements are visited in id order and take the smallest free
 * colour.  Same rule as the CUDA library's host-side builder. */
int orc_color(int nNode, int nElem, int npe, const int *conn, int *color)
{
  /* node -> elements */
  int *ecount = calloc(nNode + 1, sizeof(int));
  for (int e = 0; e < nElem; e++)
    for (int a = 0; a < npe; a++) ecount[conn[e * npe + a] + 1]++;
  for (int n = 0; n < nNode; n++) ecount[n + 1] += ecount[n];
  int *elist = malloc(sizeof(int) * (size_t)ecount[nNode]);
  int *fill = calloc(nNode, sizeof(int));
  for (int e = 0; e < nElem; e++)
    for (int a = 0; a < npe; a++) {
      int n = conn[e * npe + a];
      elist[ecount[n] + fill[n]++] = e;
    }
  for (int e = 0; e < nElem; e++) color[e] = -1;
  int ncolors = 0;
  uint64_t used;
  for (int e = 0; e < nElem; e++) {
    used = 0;
    for (int a = 0; a < npe; a++) {
      int n = conn[e * npe + a];
      for (int k = ecount[n]; k < ecount[n + 1]; k++) {
        int c = color[elist[k]];
        if (c >= 0 && c < 64) used |= (1ULL << c);
      }
    }
    int c = 0;
    while (c < 64 && (used & (1ULL << c))) c++;
    color[e] = c;
    if (c + 1 > ncolors) ncolors = c + 1;
  }
  free(ecount); free(elist); free(fill);
  return ncolors;
}
