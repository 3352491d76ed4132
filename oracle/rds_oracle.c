/* CPU restatement of pdekit's explicit continuous RDS iteration -- TEST ORACLE ONLY.
 * See rds_oracle.h for scope and the reference files each part follows. Compiled with
 * -ffp-contract=off so that no multiply-add is fused, as in the reference's x86-64 -O2 build.
 */
#include "rds_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NEQ_MAX 5
#define DIM_MAX 3
#define NDOF_MAX 32
#define NR_MAX (NDOF_MAX * NEQ_MAX)
#define NQ_MAX 64
#define NFL_MAX 40
#define NGEO_MAX 32

/* ------------------------------------------------------------------------------------------
 * Physics. Pointwise properties, physical flux, upwind matrices K = R op(Lambda) L and the
 * eigen-structure R, L, Lambda for the direction of a shape-function gradient.
 * ------------------------------------------------------------------------------------------ */

typedef struct
{
  double vars[NEQ_MAX];
  double V[DIM_MAX]; /* advection speed (scalar) or velocity (Euler) */
  double rho, inv_rho, v2, P, E, H, a;
} props_t;

/* RotationAdvection2D::compute_properties (physics/scalar/RotationAdvection2D.hpp:201-225),
 * Burgers2D::compute_properties (physics/scalar/Burgers2D.hpp:154-174),
 * Euler2DCons::compute_properties (physics/euler/Euler2DCons.hpp:159-218),
 * Euler3DCons::compute_properties (physics/euler/Euler3DCons.hpp:160-235). */
static int props(const rdso_model *m, const double *u, props_t *p)
{
  int bad = 0;
  for (int e = 0; e < m->neq; ++e)
    p->vars[e] = u[e];
  if (m->physics == RDSO_ADVECTION_CONST)
  {
    p->V[0] = m->adv[0];
    p->V[1] = m->adv[1];
  }
  else if (m->physics == RDSO_BURGERS2D)
  {
    p->V[0] = u[0];
    p->V[1] = 1.;
  }
  else
  {
    const int D = m->dim;
    const double gm1 = m->gamma - 1.;
    p->rho     = u[0];
    p->inv_rho = 1. / p->rho;
    for (int d = 0; d < D; ++d)
      p->V[d] = u[1 + d] * p->inv_rho;
    p->v2 = p->V[0] * p->V[0] + p->V[1] * p->V[1];
    if (D == 3)
      p->v2 = p->V[0] * p->V[0] + p->V[1] * p->V[1] + p->V[2] * p->V[2];
    const double rhoE = u[D + 1];
    p->P              = gm1 * (rhoE - 0.5 * p->rho * p->v2);
    if (p->P <= 0.)
      bad = 1;
    const double RT = p->P * p->inv_rho;
    p->E            = rhoE * p->inv_rho;
    p->H            = p->E + RT;
    p->a            = sqrt(m->gamma * RT);
  }
  return bad;
}

/* Physical flux F[e][d]: RotationAdvection2D::flux (:230-236), Burgers2D::flux (:186-194),
 * Euler2DCons::flux (:235-249), Euler3DCons::flux (:241-263). */
static void flux(const rdso_model *m, const props_t *p, double F[NEQ_MAX][DIM_MAX])
{
  if (m->physics == RDSO_ADVECTION_CONST)
  {
    F[0][0] = p->V[0] * p->vars[0];
    F[0][1] = p->V[1] * p->vars[0];
  }
  else if (m->physics == RDSO_BURGERS2D)
  {
    F[0][0] = 0.5 * p->V[0] * p->vars[0];
    F[0][1] = p->V[1] * p->vars[0];
  }
  else if (m->physics == RDSO_EULER2D)
  {
    const double rhou = p->vars[1], rhov = p->vars[2];
    F[0][0] = rhou;
    F[1][0] = rhou * p->V[0] + p->P;
    F[2][0] = rhou * p->V[1];
    F[3][0] = rhou * p->H;
    F[0][1] = rhov;
    F[1][1] = rhov * p->V[0];
    F[2][1] = rhov * p->V[1] + p->P;
    F[3][1] = rhov * p->H;
  }
  else
  {
    const double rhou = p->vars[1], rhov = p->vars[2], rhow = p->vars[3];
    F[0][0] = rhou;
    F[1][0] = rhou * p->V[0] + p->P;
    F[2][0] = rhou * p->V[1];
    F[3][0] = rhou * p->V[2];
    F[4][0] = rhou * p->H;
    F[0][1] = rhov;
    F[1][1] = rhov * p->V[0];
    F[2][1] = rhov * p->V[1] + p->P;
    F[3][1] = rhov * p->V[2];
    F[4][1] = rhov * p->H;
    F[0][2] = rhow;
    F[1][2] = rhow * p->V[0];
    F[2][2] = rhow * p->V[1];
    F[3][2] = rhow * p->V[2] + p->P;
    F[4][2] = rhow * p->H;
  }
}

/* Right/left eigenvectors and eigenvalues of the flux Jacobian in direction 'dir':
 * Euler2DCons::flux_jacobian_eigen_structure (physics/euler/Euler2DCons.hpp:316-398),
 * Euler3DCons::flux_jacobian_eigen_structure (physics/euler/Euler3DCons.hpp:332-447),
 * scalar ones (Burgers2D.hpp:249-260, RotationAdvection2D.hpp:305-323).
 * The Euler eigenvalues are those of the normalised direction times |dir|. */
static void eigen_structure(const rdso_model *m, const props_t *p, const double *dir,
                            double R[NEQ_MAX][NEQ_MAX], double L[NEQ_MAX][NEQ_MAX],
                            double lam[NEQ_MAX])
{
  if (m->physics == RDSO_ADVECTION_CONST || m->physics == RDSO_BURGERS2D)
  {
    R[0][0] = 1.;
    L[0][0] = 1.;
    lam[0]  = p->V[0] * dir[0] + p->V[1] * dir[1];
    return;
  }
  const double gm1 = m->gamma - 1.;
  if (m->physics == RDSO_EULER2D)
  {
    const double norm = sqrt(dir[0] * dir[0] + dir[1] * dir[1]);
    const double nx   = (norm < 1.e-9) ? dir[0] : dir[0] / norm;
    const double ny   = (norm < 1.e-9) ? dir[1] : dir[1] / norm;
    const double inv_a = 1. / p->a, inv_a2 = inv_a * inv_a;
    const double um    = p->V[0] * nx + p->V[1] * ny;
    const double ra    = 0.5 * p->rho * inv_a;
    const double coeffM2 = (0.5 * (m->gamma - 1.0) * p->v2) * inv_a2;
    const double uDivA   = gm1 * p->V[0] * inv_a;
    const double vDivA   = gm1 * p->V[1] * inv_a;
    const double rho_a   = p->rho * p->a;
    const double gm1_ov_rhoa = gm1 / rho_a;
    R[0][0] = 1.;
    R[0][1] = 0.;
    R[0][2] = ra;
    R[0][3] = ra;
    R[1][0] = p->V[0];
    R[1][1] = p->rho * ny;
    R[1][2] = ra * (p->V[0] + p->a * nx);
    R[1][3] = ra * (p->V[0] - p->a * nx);
    R[2][0] = p->V[1];
    R[2][1] = -p->rho * nx;
    R[2][2] = ra * (p->V[1] + p->a * ny);
    R[2][3] = ra * (p->V[1] - p->a * ny);
    R[3][0] = 0.5 * p->v2;
    R[3][1] = p->rho * (p->V[0] * ny - p->V[1] * nx);
    R[3][2] = ra * (p->H + p->a * um);
    R[3][3] = ra * (p->H - p->a * um);
    L[0][0] = 1. - coeffM2;
    L[0][1] = uDivA * inv_a;
    L[0][2] = vDivA * inv_a;
    L[0][3] = -gm1 * inv_a2;
    L[1][0] = p->inv_rho * (p->V[1] * nx - p->V[0] * ny);
    L[1][1] = p->inv_rho * ny;
    L[1][2] = -p->inv_rho * nx;
    L[1][3] = 0.0;
    L[2][0] = p->a * p->inv_rho * (coeffM2 - um * inv_a);
    L[2][1] = p->inv_rho * (nx - uDivA);
    L[2][2] = p->inv_rho * (ny - vDivA);
    L[2][3] = gm1_ov_rhoa;
    L[3][0] = p->a * p->inv_rho * (coeffM2 + um * inv_a);
    L[3][1] = -p->inv_rho * (nx + uDivA);
    L[3][2] = -p->inv_rho * (ny + vDivA);
    L[3][3] = gm1_ov_rhoa;
    lam[0]  = norm * um;
    lam[1]  = norm * um;
    lam[2]  = norm * (um + p->a);
    lam[3]  = norm * (um - p->a);
    return;
  }
  /* Euler 3D */
  const double norm = sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
  const double nx   = (norm == 0) ? dir[0] : dir[0] / norm;
  const double ny   = (norm == 0) ? dir[1] : dir[1] / norm;
  const double nz   = (norm == 0) ? dir[2] : dir[2] / norm;
  const double inv_a = 1. / p->a, inv_a2 = inv_a * inv_a;
  const double u = p->V[0], v = p->V[1], w = p->V[2];
  const double um = u * nx + v * ny + w * nz;
  const double ra = 0.5 * p->rho * inv_a;
  const double gu_a = gm1 * u * inv_a, gv_a = gm1 * v * inv_a, gw_a = gm1 * w * inv_a;
  const double rho_a       = p->rho * p->a;
  const double gm1_ov_rhoa = gm1 / rho_a;
  const double ke          = 0.5 * p->v2;
  const double gm2         = (0.5 * gm1 * p->v2) * inv_a2;
  const double k2          = 1.0 - gm2;
  const double k3          = -gm1 * inv_a2;
  const double rho = p->rho, ir = p->inv_rho, a = p->a, H = p->H;
  R[0][0] = nx;
  R[0][1] = ny;
  R[0][2] = nz;
  R[0][3] = ra;
  R[0][4] = ra;
  R[1][0] = u * nx;
  R[1][1] = u * ny - rho * nz;
  R[1][2] = u * nz + rho * ny;
  R[1][3] = ra * (u + a * nx);
  R[1][4] = ra * (u - a * nx);
  R[2][0] = v * nx + rho * nz;
  R[2][1] = v * ny;
  R[2][2] = v * nz - rho * nx;
  R[2][3] = ra * (v + a * ny);
  R[2][4] = ra * (v - a * ny);
  R[3][0] = w * nx - rho * ny;
  R[3][1] = w * ny + rho * nx;
  R[3][2] = w * nz;
  R[3][3] = ra * (w + a * nz);
  R[3][4] = ra * (w - a * nz);
  R[4][0] = ke * nx + rho * (v * nz - w * ny);
  R[4][1] = ke * ny + rho * (w * nx - u * nz);
  R[4][2] = ke * nz + rho * (u * ny - v * nx);
  R[4][3] = ra * (H + a * um);
  R[4][4] = ra * (H - a * um);
  L[0][0] = nx * k2 - ir * (v * nz - w * ny);
  L[0][1] = gu_a * inv_a * nx;
  L[0][2] = gv_a * inv_a * nx + nz * ir;
  L[0][3] = gw_a * inv_a * nx - ny * ir;
  L[0][4] = k3 * nx;
  L[1][0] = ny * k2 - ir * (w * nx - u * nz);
  L[1][1] = gu_a * inv_a * ny - nz * ir;
  L[1][2] = gv_a * inv_a * ny;
  L[1][3] = gw_a * inv_a * ny + nx * ir;
  L[1][4] = k3 * ny;
  L[2][0] = nz * k2 - ir * (u * ny - v * nx);
  L[2][1] = gu_a * inv_a * nz + ny * ir;
  L[2][2] = gv_a * inv_a * nz - nx * ir;
  L[2][3] = gw_a * inv_a * nz;
  L[2][4] = k3 * nz;
  L[3][0] = a * ir * (gm2 - um / a);
  L[3][1] = ir * (nx - gu_a);
  L[3][2] = ir * (ny - gv_a);
  L[3][3] = ir * (nz - gw_a);
  L[3][4] = gm1_ov_rhoa;
  L[4][0] = a * ir * (gm2 + um / a);
  L[4][1] = ir * (-nx - gu_a);
  L[4][2] = ir * (-ny - gv_a);
  L[4][3] = ir * (-nz - gw_a);
  L[4][4] = gm1_ov_rhoa;
  lam[0]  = norm * um;
  lam[1]  = norm * um;
  lam[2]  = norm * um;
  lam[3]  = norm * (um + a);
  lam[4]  = norm * (um - a);
}

/* K = R op(Lambda) L with op = max(0,.) (sign > 0) or min(0,.) (sign < 0); eig receives the
 * unclipped eigenvalues. Summation K_ij = sum_k (R_ik op(l_k)) L_kj in k order, as the
 * closed forms of build_K_mat (Euler2DCons.hpp:402-536, Euler3DCons.hpp:451-) evaluate it. */
static void build_K(const rdso_model *m, const props_t *p, const double *dir, int sign,
                    double *eig, double K[NEQ_MAX][NEQ_MAX])
{
  double R[NEQ_MAX][NEQ_MAX], L[NEQ_MAX][NEQ_MAX];
  const int n = m->neq;
  eigen_structure(m, p, dir, R, L, eig);
  double lo[NEQ_MAX];
  for (int k = 0; k < n; ++k)
    lo[k] = sign > 0 ? (eig[k] > 0.0 ? eig[k] : 0.0)
                     : sign < 0 ? (eig[k] < 0.0 ? eig[k] : 0.0) : eig[k];
  if (n == 1)
  {
    /* scalar build_K_mat: 1. * op(lambda) * 1. */
    K[0][0] = 1. * lo[0] * 1.;
    return;
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
    {
      double s = R[i][0] * lo[0] * L[0][j];
      for (int k = 1; k < n; ++k)
        s = s + R[i][k] * lo[k] * L[k][j];
      K[i][j] = s;
    }
}

/* ------------------------------------------------------------------------------------------
 * Small dense helpers
 * ------------------------------------------------------------------------------------------ */

/* Inverse of an n x n matrix (n <= 5). n = 1: 1/a. Otherwise Gauss-Jordan elimination with
 * row partial pivoting (the reference uses closed-form cofactors up to 4x4,
 * math/unary_ops/matrix_unary_ops/MatrixInverse.hpp:113-300, and LAPACK dgetrf/dgetri for
 * 5x5, :87-97; all agree to rounding on the well-conditioned sum of K+ matrices). */
static void inverse(int n, double A[NEQ_MAX][NEQ_MAX], double X[NEQ_MAX][NEQ_MAX])
{
  if (n == 1)
  {
    X[0][0] = 1.0 / A[0][0];
    return;
  }
  double M[NEQ_MAX][2 * NEQ_MAX];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
    {
      M[i][j]     = A[i][j];
      M[i][n + j] = (i == j) ? 1.0 : 0.0;
    }
  for (int k = 0; k < n; ++k)
  {
    int piv = k;
    for (int i = k + 1; i < n; ++i)
      if (fabs(M[i][k]) > fabs(M[piv][k]))
        piv = i;
    if (piv != k)
      for (int j = 0; j < 2 * n; ++j)
      {
        const double t = M[k][j];
        M[k][j]        = M[piv][j];
        M[piv][j]      = t;
      }
    const double ip = 1.0 / M[k][k];
    for (int j = 0; j < 2 * n; ++j)
      M[k][j] *= ip;
    for (int i = 0; i < n; ++i)
    {
      if (i == k)
        continue;
      const double f = M[i][k];
      for (int j = 0; j < 2 * n; ++j)
        M[i][j] -= f * M[k][j];
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      X[i][j] = M[i][n + j];
}

/* 3x3 determinant and inverse as DenseSMat<3,3>::det / ::inv use them
 * (MatrixInverse.hpp:167-184: cofactors times 1/det). */
static double det3(const double *m)
{
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
         m[2] * (m[3] * m[7] - m[4] * m[6]);
}

static void inv3(const double *m1, double det, double *m2)
{
  const double invDet = 1. / det;
  m2[0] = (m1[4] * m1[8] - m1[5] * m1[7]) * invDet;
  m2[1] = -(m1[1] * m1[8] - m1[2] * m1[7]) * invDet;
  m2[2] = (m1[1] * m1[5] - m1[4] * m1[2]) * invDet;
  m2[3] = -(m1[3] * m1[8] - m1[5] * m1[6]) * invDet;
  m2[4] = (m1[0] * m1[8] - m1[2] * m1[6]) * invDet;
  m2[5] = -(m1[0] * m1[5] - m1[2] * m1[3]) * invDet;
  m2[6] = (m1[3] * m1[7] - m1[4] * m1[6]) * invDet;
  m2[7] = -(m1[0] * m1[7] - m1[1] * m1[6]) * invDet;
  m2[8] = (m1[0] * m1[4] - m1[1] * m1[3]) * invDet;
}

/* Jacobian J(xi,x) = sum_g dVgeo[xi](q,g) X[g][x]; detJ; invJ(x,xi) = d xi / d x.
 * GeometryMetric MetricComputer<2D,2D> (GeometryMetric.hpp:364-440) and <3D,3D> (:485-560). */
static double jacobian(int D, const double *dVgeo, int nq, int ngeo, int q, const double *X,
                       double invJ[DIM_MAX][DIM_MAX])
{
  double J[DIM_MAX][DIM_MAX];
  for (int xi = 0; xi < D; ++xi)
    for (int x = 0; x < D; ++x)
    {
      const double *row = dVgeo + ((size_t)xi * nq + q) * ngeo;
      double s          = row[0] * X[0 * D + x];
      for (int g = 1; g < ngeo; ++g)
        s = s + row[g] * X[g * D + x];
      J[xi][x] = s;
    }
  if (D == 2)
  {
    const double det     = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    const double inv_det = 1.0 / det;
    invJ[0][0]           = inv_det * J[1][1];
    invJ[1][1]           = inv_det * J[0][0];
    invJ[0][1]           = -inv_det * J[0][1];
    invJ[1][0]           = -inv_det * J[1][0];
    return det;
  }
  double Jm[9], Ji[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      Jm[i * 3 + j] = J[i][j];
  const double det = det3(Jm);
  inv3(Jm, det, Ji);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      invJ[i][j] = Ji[i * 3 + j];
  return det;
}

/* ------------------------------------------------------------------------------------------
 * One cell: metrics + scheme
 * ------------------------------------------------------------------------------------------ */

static int cell_residual_theta(const rdso_model *m, const rdso_cells *g, const double *X,
                               const double *un, double *elem_res, double *elem_ws,
                               double *theta_out);

static int cell_residual(const rdso_model *m, const rdso_cells *g, const double *X,
                         const double *un, double *elem_res, double *elem_ws)
{
  return cell_residual_theta(m, g, X, un, elem_res, elem_ws, NULL);
}

/* The cell's scheme residual; for PGB also its blending coefficient (theta_out, may be NULL). */
static int cell_residual_theta(const rdso_model *m, const rdso_cells *g, const double *X,
                               const double *un, double *elem_res, double *elem_ws,
                               double *theta_out)
{
  const int D = m->dim, NEQ = m->neq;
  const int ndof = g->ndof, nq = g->nq, nfl = g->nfl, ngeo = g->ngeo;
  /* PSI distributes with the N scheme first */
  const int nlike = m->scheme == RDSO_N || m->scheme == RDSO_PSI;
  int bad = 0;

  /* geometry at quadrature points */
  double invJ[NQ_MAX][DIM_MAX][DIM_MAX], jdet[NQ_MAX];
  for (int q = 0; q < nq; ++q)
    jdet[q] = jacobian(D, g->dVgeo, nq, ngeo, q, X, invJ[q]);

  /* solution at quadrature points: uq = V u  (SolutionSpaceMetric.hpp:288-327) */
  double uq[NQ_MAX][NEQ_MAX];
  for (int q = 0; q < nq; ++q)
    for (int e = 0; e < NEQ; ++e)
    {
      const double *row = g->V + (size_t)q * ndof;
      double s          = row[0] * un[0 * NEQ + e];
      for (int n = 1; n < ndof; ++n)
        s = s + row[n] * un[n * NEQ + e];
      uq[q][e] = s;
    }

  /* flux nodes: Sf = Vsf u, F(Sf)  (FluxSpaceMetric.hpp:588-661) */
  double Ff[NFL_MAX][NEQ_MAX][DIM_MAX];
  for (int f = 0; f < nfl; ++f)
  {
    double sf[NEQ_MAX];
    for (int e = 0; e < NEQ; ++e)
    {
      const double *row = g->Vsf + (size_t)f * ndof;
      double s          = row[0] * un[0 * NEQ + e];
      for (int n = 1; n < ndof; ++n)
        s = s + row[n] * un[n * NEQ + e];
      sf[e] = s;
    }
    props_t pf;
    bad += props(m, sf, &pf);
    double F[NEQ_MAX][DIM_MAX];
    flux(m, &pf, F);
    for (int e = 0; e < NEQ; ++e)
      for (int d = 0; d < D; ++d)
        Ff[f][e][d] = F[e][d];
  }

  /* divergence of the flux interpolant at quadrature points (FluxSpaceMetric.hpp:680-740):
   * dF_ref[xi] = dVf[xi] F_icomp ; dF_icomp/dx_icomp = sum_xi invJ(icomp,xi) dF_ref[xi] */
  double divF[NQ_MAX][NEQ_MAX][DIM_MAX];
  for (int icomp = 0; icomp < D; ++icomp)
    for (int q = 0; q < nq; ++q)
      for (int e = 0; e < NEQ; ++e)
      {
        double dref[DIM_MAX];
        for (int xi = 0; xi < D; ++xi)
        {
          const double *row = g->dVf + ((size_t)xi * nq + q) * nfl;
          double s          = row[0] * Ff[0][e][icomp];
          for (int f = 1; f < nfl; ++f)
            s = s + row[f] * Ff[f][e][icomp];
          dref[xi] = s;
        }
        double s = invJ[q][icomp][0] * dref[0];
        for (int xi = 1; xi < D; ++xi)
          s = s + invJ[q][icomp][xi] * dref[xi];
        divF[q][e][icomp] = s;
      }

  /* scheme (PGLDA.hpp:111-311, PGN.hpp:98-290, PGB.hpp:314-498) */
  double lda[NDOF_MAX][NEQ_MAX], diss[NDOF_MAX][NEQ_MAX], wsn[NDOF_MAX];
  double phi[NEQ_MAX];
  memset(lda, 0, sizeof(lda));
  memset(diss, 0, sizeof(diss));
  memset(phi, 0, sizeof(phi));
  for (int n = 0; n < ndof; ++n)
    wsn[n] = 0.0;
  double elem_volume = 0.0;

  static double Kp[NDOF_MAX][NEQ_MAX][NEQ_MAX];
  for (int q = 0; q < nq; ++q)
  {
    double sumKp[NEQ_MAX][NEQ_MAX], inv[NEQ_MAX][NEQ_MAX];
    memset(sumKp, 0, sizeof(sumKp));
    const double wj = g->w[q] * jdet[q];
    elem_volume += wj;

    props_t pq;
    bad += props(m, uq[q], &pq);

    for (int n = 0; n < ndof; ++n)
    {
      double gref[DIM_MAX], gphys[DIM_MAX];
      for (int d = 0; d < D; ++d)
        gref[d] = g->dV[((size_t)d * nq + q) * ndof + n];
      for (int x = 0; x < D; ++x)
      {
        double s = invJ[q][x][0] * gref[0];
        for (int xi = 1; xi < D; ++xi)
          s = s + invJ[q][x][xi] * gref[xi];
        gphys[x] = s;
      }
      double eig[NEQ_MAX];
      if (m->scheme == RDSO_LDA)
      {
        /* build_K_mat with op = max(0,.) (PGLDA.hpp:204-214) */
        build_K(m, &pq, gphys, +1, eig, Kp[n]);
      }
      else
      {
        /* eigen structure, clip, K = R D+ L (PGB.hpp:363-382, PGN.hpp:186-205) */
        double R[NEQ_MAX][NEQ_MAX], L[NEQ_MAX][NEQ_MAX];
        eigen_structure(m, &pq, gphys, R, L, eig);
        double dp[NEQ_MAX];
        for (int k = 0; k < NEQ; ++k)
          dp[k] = eig[k] > 0.0 ? eig[k] : 0.0;
        for (int i = 0; i < NEQ; ++i)
          for (int j = 0; j < NEQ; ++j)
          {
            double s = (R[i][0] * dp[0]) * L[0][j];
            for (int k = 1; k < NEQ; ++k)
              s = s + (R[i][k] * dp[k]) * L[k][j];
            Kp[n][i][j] = s;
          }
      }
      double lmax = 1.e-6;
      for (int e = 0; e < NEQ; ++e)
      {
        const double ae = fabs(eig[e]);
        lmax            = lmax > ae ? lmax : ae;
      }
      wsn[n] = wsn[n] > lmax ? wsn[n] : lmax;
      for (int i = 0; i < NEQ; ++i)
        for (int j = 0; j < NEQ; ++j)
          sumKp[i][j] += Kp[n][i][j];
    }

    inverse(NEQ, sumKp, inv);

    /* pointwise residual r_q = sum_d dF_d/dx_d */
    double rq[NEQ_MAX];
    for (int e = 0; e < NEQ; ++e)
    {
      double s = 0.0;
      for (int d = 0; d < D; ++d)
        s += divF[q][e][d];
      rq[e] = s;
    }

    /* Kp[n] * inv: B[n] = Kp[n] inv */
    double B[NDOF_MAX][NEQ_MAX][NEQ_MAX];
    for (int n = 0; n < ndof; ++n)
      for (int i = 0; i < NEQ; ++i)
        for (int j = 0; j < NEQ; ++j)
        {
          double s = Kp[n][i][0] * inv[0][j];
          for (int k = 1; k < NEQ; ++k)
            s = s + Kp[n][i][k] * inv[k][j];
          B[n][i][j] = s;
        }

    if (nlike)
    {
      /* PGN accumulates the LDA part and then the dissipation into the same nodal residual
       * at every quadrature point (PGN.hpp:246-269) */
      for (int n = 0; n < ndof; ++n)
        for (int i = 0; i < NEQ; ++i)
        {
          double s = B[n][i][0] * rq[0];
          for (int k = 1; k < NEQ; ++k)
            s = s + B[n][i][k] * rq[k];
          lda[n][i] += wj * s;
        }
    }

    if (m->scheme == RDSO_B || nlike)
    {
      /* N-type dissipation sum_{m != n} Kp[n] inv Kp[m] (u_n - u_m) */
      double(*acc)[NEQ_MAX] = nlike ? lda : diss;
      for (int n = 0; n < ndof; ++n)
        for (int mm = 0; mm < ndof; ++mm)
        {
          if (mm == n)
            continue;
          double C[NEQ_MAX][NEQ_MAX];
          for (int i = 0; i < NEQ; ++i)
            for (int j = 0; j < NEQ; ++j)
            {
              double s = B[n][i][0] * Kp[mm][0][j];
              for (int k = 1; k < NEQ; ++k)
                s = s + B[n][i][k] * Kp[mm][k][j];
              C[i][j] = s;
            }
          double du[NEQ_MAX];
          for (int e = 0; e < NEQ; ++e)
            du[e] = un[n * NEQ + e] - un[mm * NEQ + e];
          for (int i = 0; i < NEQ; ++i)
          {
            double s = C[i][0] * du[0];
            for (int k = 1; k < NEQ; ++k)
              s = s + C[i][k] * du[k];
            acc[n][i] += wj * s;
          }
        }
    }

    for (int e = 0; e < NEQ; ++e)
      phi[e] += wj * rq[e];

    for (int n = 0; n < ndof && !nlike; ++n)
      for (int i = 0; i < NEQ; ++i)
      {
        double s = B[n][i][0] * rq[0];
        for (int k = 1; k < NEQ; ++k)
          s = s + B[n][i][k] * rq[k];
        lda[n][i] += wj * s;
      }
  }

  if (m->scheme == RDSO_LDA)
  {
    for (int n = 0; n < ndof; ++n)
      for (int e = 0; e < NEQ; ++e)
        elem_res[n * NEQ + e] = lda[n][e];
  }
  else if (m->scheme == RDSO_N)
  {
    for (int n = 0; n < ndof; ++n)
      for (int e = 0; e < NEQ; ++e)
        elem_res[n * NEQ + e] = lda[n][e];
  }
  else if (m->scheme == RDSO_PSI)
  {
    /* the reference's residual limiter on the N residuals, per equation of a scalar problem
     * (LFResidualLimiter.hpp:37-110; for systems it does nothing, :18-30): where the cell
     * residual is above 1e-14 in magnitude, x_n = max(phi_n / phi, 0) + 1e-12 and
     * phi_n = x_n / sum_m x_m * phi */
    for (int e = 0; e < NEQ; ++e)
    {
      double x[NDOF_MAX], sum_xp = 0.0;
      const int lim = NEQ == 1 && fabs(phi[e]) > 1.e-14;
      for (int n = 0; n < ndof; ++n)
      {
        if (lim)
        {
          const double r = lda[n][e] / phi[e];
          x[n]           = (r < 0.0 ? 0.0 : r) + 1.e-12; /* std::max(r, 0.0) */
          sum_xp += x[n];
        }
      }
      for (int n = 0; n < ndof; ++n)
        elem_res[n * NEQ + e] = lim ? x[n] / sum_xp * phi[e] : lda[n][e];
    }
  }
  else
  {
    /* internal blending coefficient from equation 0 (PGB.hpp:437-477) */
    double abs_phiN = 0.0;
    for (int n = 0; n < ndof; ++n)
      abs_phiN += fabs(lda[n][0] + diss[n][0]);
    const double theta = fabs(phi[0]) / (abs_phiN + 1.e-6);
    if (theta_out)
      *theta_out = theta;
    for (int n = 0; n < ndof; ++n)
      for (int e = 0; e < NEQ; ++e)
        elem_res[n * NEQ + e] = lda[n][e] + theta * diss[n][e];
  }

  double wmax = wsn[0];
  for (int n = 1; n < ndof; ++n)
    wmax = wmax > wsn[n] ? wmax : wsn[n];
  for (int n = 0; n < ndof; ++n)
    elem_ws[n] = elem_volume * wmax;
  return bad;
}

void rdso_cell_residual(const rdso_model *m, const rdso_cells *g, const double *X,
                        const double *un, double *elem_res, double *elem_ws)
{
  cell_residual(m, g, X, un, elem_res, elem_ws);
}

/* Element Jacobian of the Picard linearisation, accumulated point by point in the reference's
 * order. PGLDA (PGLDA.hpp:316-536): J_mn += w_q |J_q| (Kp_m (sum Kp)^-1) K_n with Kp from
 * build_K_mat(op = max(0,.)) and K_n from build_K_mat(op = identity). PGN (PGN.hpp:296-440,
 * the plain N scheme): J_mn += w_q |J_q| (delta_mn Kp_m - Kp_m (sum Km)^-1 Km_n) with Kp, Km
 * = R max/min(Lambda, 0) L. */
void rdso_element_jacobian(const rdso_model *m, const rdso_cells *g, const double *X,
                           const double *un, double *jac)
{
  const int D = m->dim, NEQ = m->neq;
  const int ndof = g->ndof, nq = g->nq, ngeo = g->ngeo, NR = ndof * NEQ;
  for (int i = 0; i < NR * NR; ++i)
    jac[i] = 0.0;
  /* PGB (PGB.hpp:505-690): the LDA Jacobian plus theta times the stabilisation Jacobian
   * stab_mn = sum_q w_q |J_q| (delta_mn Kp_m - Kp_m (sum Kp)^-1 Kp_n), theta from the residual */
  const int pgb = m->scheme == RDSO_B;
  static double stab[NR_MAX * NR_MAX];
  double theta = 0.0;
  if (pgb)
  {
    double er[NDOF_MAX * NEQ_MAX], ew[NDOF_MAX];
    cell_residual_theta(m, g, X, un, er, ew, &theta);
    for (int i = 0; i < NR * NR; ++i)
      stab[i] = 0.0;
  }
  static double Kp[NDOF_MAX][NEQ_MAX][NEQ_MAX], Kn[NDOF_MAX][NEQ_MAX][NEQ_MAX];
  for (int q = 0; q < nq; ++q)
  {
    double invJ[DIM_MAX][DIM_MAX];
    const double jd = jacobian(D, g->dVgeo, nq, ngeo, q, X, invJ);
    const double wj = g->w[q] * jd;
    double uq[NEQ_MAX];
    for (int e = 0; e < NEQ; ++e)
    {
      const double *row = g->V + (size_t)q * ndof;
      double s          = row[0] * un[0 * NEQ + e];
      for (int n = 1; n < ndof; ++n)
        s = s + row[n] * un[n * NEQ + e];
      uq[e] = s;
    }
    props_t pq;
    props(m, uq, &pq);
    double sumKp[NEQ_MAX][NEQ_MAX], inv[NEQ_MAX][NEQ_MAX];
    memset(sumKp, 0, sizeof(sumKp));
    for (int n = 0; n < ndof; ++n)
    {
      double gref[DIM_MAX], gphys[DIM_MAX], eig[NEQ_MAX];
      for (int d = 0; d < D; ++d)
        gref[d] = g->dV[((size_t)d * nq + q) * ndof + n];
      for (int x = 0; x < D; ++x)
      {
        double s = invJ[x][0] * gref[0];
        for (int xi = 1; xi < D; ++xi)
          s = s + invJ[x][xi] * gref[xi];
        gphys[x] = s;
      }
      build_K(m, &pq, gphys, +1, eig, Kp[n]);
      build_K(m, &pq, gphys, m->scheme == RDSO_N ? -1 : 0, eig, Kn[n]);
      for (int i = 0; i < NEQ; ++i)
        for (int j = 0; j < NEQ; ++j)
          sumKp[i][j] += (m->scheme == RDSO_N) ? Kn[n][i][j] : Kp[n][i][j];
    }
    inverse(NEQ, sumKp, inv);
    for (int mm = 0; mm < ndof; ++mm)
    {
      double B[NEQ_MAX][NEQ_MAX];
      for (int i = 0; i < NEQ; ++i)
        for (int j = 0; j < NEQ; ++j)
        {
          double s = Kp[mm][i][0] * inv[0][j];
          for (int k = 1; k < NEQ; ++k)
            s = s + Kp[mm][i][k] * inv[k][j];
          B[i][j] = s;
        }
      for (int n = 0; n < ndof; ++n)
        for (int i = 0; i < NEQ; ++i)
          for (int j = 0; j < NEQ; ++j)
          {
            double s = B[i][0] * Kn[n][0][j];
            for (int k = 1; k < NEQ; ++k)
              s = s + B[i][k] * Kn[n][k][j];
            if (m->scheme == RDSO_N)
              s = (n == mm ? Kp[mm][i][j] : 0.0) - s;
            jac[(size_t)(mm * NEQ + i) * NR + n * NEQ + j] += wj * s;
            if (pgb)
            {
              double sp = B[i][0] * Kp[n][0][j];
              for (int k = 1; k < NEQ; ++k)
                sp = sp + B[i][k] * Kp[n][k][j];
              stab[(size_t)(mm * NEQ + i) * NR + n * NEQ + j] +=
                  (n == mm) ? wj * (Kp[mm][i][j] - sp) : -(wj * sp);
            }
          }
    }
  }
  if (pgb)
    for (int i = 0; i < NR * NR; ++i)
      jac[i] += theta * stab[i];
}

/* ------------------------------------------------------------------------------------------ */

void rdso_dual_volume(const rdso_model *m, const rdso_cells *groups, int ngroups, int nnodes,
                      const double *geo_coords, double *vol)
{
  const int D = m->dim;
  for (int i = 0; i < nnodes; ++i)
    vol[i] = 0.0;
  for (int ig = 0; ig < ngroups; ++ig)
  {
    const rdso_cells *g = &groups[ig];
    for (int c = 0; c < g->ncells; ++c)
    {
      double X[NGEO_MAX * DIM_MAX];
      for (int k = 0; k < g->ngeo; ++k)
        for (int d = 0; d < D; ++d)
          X[k * D + d] = geo_coords[(size_t)g->geo_conn[(size_t)c * g->ngeo + k] * D + d];
      double cv = 0.0;
      /* RDTimeUpdate::setup (RDTimeUpdate.hpp:118-177): Gauss rule of the cell's order */
      const int nqv        = g->nqv > 0 ? g->nqv : g->nq;
      const double *wv     = g->nqv > 0 ? g->wv : g->w;
      const double *dvgeo  = g->nqv > 0 ? g->dVgeo_v : g->dVgeo;
      for (int q = 0; q < nqv; ++q)
      {
        double invJ[DIM_MAX][DIM_MAX];
        const double dj = jacobian(D, dvgeo, nqv, g->ngeo, q, X, invJ);
        cv += wv[q] * dj;
      }
      for (int n = 0; n < g->ndof; ++n)
        vol[g->sol_conn[(size_t)c * g->ndof + n]] += cv;
    }
  }
}

/* Euler flux through a direction n (Euler2DCons::flux(p, direction, flux),
 * physics/euler/Euler2DCons.hpp:253-266; Euler3DCons.hpp:267-285). */
static void euler_flux_normal(const rdso_model *m, const props_t *p, const double *n, double *F)
{
  const int D = m->dim;
  double rhoum = p->vars[1] * n[0] + p->vars[2] * n[1];
  if (D == 3)
    rhoum = p->vars[1] * n[0] + p->vars[2] * n[1] + p->vars[3] * n[2];
  F[0] = rhoum;
  for (int d = 0; d < D; ++d)
    F[1 + d] = rhoum * p->V[d] + p->P * n[d];
  F[D + 1] = rhoum * p->H;
}

/* Weak boundary-facet residuals: WeakDirichlet (WeakDirichletBC.hpp:159-265), WeakWall,
 * WeakSubInlet, WeakSubOutlet, WeakFarfield, WeakSuperInlet (WeakSuperInlet.hpp:62-160: no
 * residual, only the wave speed), WeakSymmetry (WeakSymmetry.hpp:100-190), plus the rescaling to
 * the facet total (WeakBC.hpp:786-832) and the nodal accumulation (WeakBC.hpp:315-352). */
static int apply_weak_bc(const rdso_model *m, const rdso_bc *b, const double *geo_coords,
                         const double *vol, const double *u, double *res, double *ws)
{
  const int D = m->dim, NEQ = m->neq;
  int bad = 0;
  for (int f = 0; f < b->nfacets; ++f)
  {
    double X[NGEO_MAX * DIM_MAX];
    for (int k = 0; k < b->nfgeo; ++k)
      for (int d = 0; d < D; ++d)
        X[k * D + d] = geo_coords[(size_t)b->geo_conn[(size_t)f * b->nfgeo + k] * D + d];
    const int *dofs = b->sol_conn + (size_t)f * b->nfdof;
    double bres[NDOF_MAX][NEQ_MAX], coeff[NDOF_MAX], total[NEQ_MAX];
    memset(bres, 0, sizeof(bres));
    memset(total, 0, sizeof(total));
    for (int n = 0; n < b->nfdof; ++n)
      coeff[n] = 0.0;

    for (int q = 0; q < b->nfq; ++q)
    {
      /* facet normal and length (GeometryMetric MetricComputer<2D,1D>, :560-600;
       * <3D,2D>, :610-660) */
      double nrm[DIM_MAX], jd;
      if (D == 2)
      {
        const double *row = b->fdVgeo + (size_t)q * b->nfgeo;
        double tx = row[0] * X[0], ty = row[0] * X[1];
        for (int k = 1; k < b->nfgeo; ++k)
        {
          tx = tx + row[k] * X[k * 2 + 0];
          ty = ty + row[k] * X[k * 2 + 1];
        }
        const double n0 = ty, n1 = -tx;
        const double norm = sqrt(n0 * n0 + n1 * n1);
        const double inv_norm = 1.0 / norm;
        nrm[0] = inv_norm * n0;
        nrm[1] = inv_norm * n1;
        jd     = norm;
      }
      else
      {
        double t[2][3];
        for (int xi = 0; xi < 2; ++xi)
        {
          const double *row = b->fdVgeo + ((size_t)xi * b->nfq + q) * b->nfgeo;
          for (int d = 0; d < 3; ++d)
          {
            double s = row[0] * X[d];
            for (int k = 1; k < b->nfgeo; ++k)
              s = s + row[k] * X[k * 3 + d];
            t[xi][d] = s;
          }
        }
        const double n0 = t[0][1] * t[1][2] - t[0][2] * t[1][1];
        const double n1 = t[0][2] * t[1][0] - t[0][0] * t[1][2];
        const double n2 = t[0][0] * t[1][1] - t[0][1] * t[1][0];
        const double norm = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
        const double inv_norm = 1.0 / norm;
        jd     = norm;
        nrm[0] = inv_norm * n0;
        nrm[1] = inv_norm * n1;
        nrm[2] = inv_norm * n2;
      }
      const double wq = jd * b->fw[q];

      double uqf[NEQ_MAX];
      for (int e = 0; e < NEQ; ++e)
      {
        const double *row = b->fV + (size_t)q * b->nfdof;
        double s          = row[0] * u[(size_t)dofs[0] * NEQ + e];
        for (int n = 1; n < b->nfdof; ++n)
          s = s + row[n] * u[(size_t)dofs[n] * NEQ + e];
        uqf[e] = s;
      }
      props_t p;
      bad += props(m, uqf, &p);
      double eig[NEQ_MAX], Km[NEQ_MAX][NEQ_MAX];
      build_K(m, &p, nrm, -1, eig, Km);

      /* lambda floor 1e-9 (WeakDirichletBC.hpp), 1e-8 for WeakFarfield (WeakFarfield.hpp:149) */
      double eig_max = (b->kind == RDSO_BC_WEAK_FARFIELD) ? 1.e-8 : 1.e-9;
      double ghost[NEQ_MAX], gflux[NEQ_MAX];
      for (int e = 0; e < NEQ; ++e)
      {
        const double ae = fabs(eig[e]);
        eig_max         = eig_max > ae ? eig_max : ae;
      }
      for (int n = 0; n < b->nfdof; ++n)
        coeff[n] = coeff[n] > eig_max ? coeff[n] : eig_max;

      double relax = 1.0;
      if (b->kind == RDSO_BC_WEAK_SUPER_INLET)
      {
        for (int e = 0; e < NEQ; ++e)
          gflux[e] = 0.0;
      }
      else if (b->kind == RDSO_BC_WEAK_WALL)
      {
        /* WeakWall.hpp:93-250 (active branch): mirror state with the normal velocity removed,
         * same density and pressure; residual = relax V w (F(u_ghost).n - F(u).n), relax = 1
         * for P1 facets, 1/(3p) otherwise; total without relax */
        relax = (b->order <= 1) ? 1.0 : 1. / (3. * b->order);
        double Fn[NEQ_MAX], Fg[NEQ_MAX], ug[NEQ_MAX];
        euler_flux_normal(m, &p, nrm, Fn);
        double vn = 0.0, v2_new = 0.0;
        for (int d = 0; d < D; ++d)
          vn += p.V[d] * nrm[d];
        ug[0] = p.rho;
        for (int d = 0; d < D; ++d)
        {
          ug[d + 1] = p.V[d] - vn * nrm[d];
          v2_new += ug[d + 1] * ug[d + 1];
          ug[d + 1] *= p.rho;
        }
        ug[D + 1] = uqf[D + 1] + 0.5 * p.rho * (v2_new - p.v2);
        props_t pg;
        bad += props(m, ug, &pg);
        euler_flux_normal(m, &pg, nrm, Fg);
        for (int e = 0; e < NEQ; ++e)
          gflux[e] = Fg[e] - Fn[e];
      }
      else
      {
        if (b->kind == RDSO_BC_WEAK_DIRICHLET)
        {
          const double *gq = b->gq + ((size_t)f * b->nfq + q) * NEQ;
          for (int e = 0; e < NEQ; ++e)
            ghost[e] = gq[e];
        }
        else if (b->kind == RDSO_BC_WEAK_FARFIELD)
        {
          /* WeakFarfield.hpp:125-240 (active branch): the reference state, K-(n) (u_ref - u) */
          for (int e = 0; e < NEQ; ++e)
            ghost[e] = b->gq[e];
        }
        else if (b->kind == RDSO_BC_WEAK_SYMMETRY)
        {
          /* WeakSymmetry.hpp:120-160: density and energy kept, momentum rho (V - 2 (V.n) n) */
          double vn = 0.0;
          for (int d = 0; d < D; ++d)
            vn += nrm[d] * p.V[d];
          ghost[0]       = uqf[0];
          ghost[NEQ - 1] = uqf[NEQ - 1];
          for (int d = 0; d < D; ++d)
            ghost[d + 1] = uqf[0] * (p.V[d] - 2. * vn * nrm[d]);
        }
        else if (b->kind == RDSO_BC_WEAK_SUB_INLET)
        {
          /* WeakSubInlet.hpp:113-215: total conditions at the local Mach number */
          const double gm1 = m->gamma - 1.;
          const double Ma  = sqrt(p.v2) / p.a;
          const double fac = 1. + 0.5 * gm1 * Ma * Ma;
          const double Tg  = b->params[0] / fac;
          const double pg  = b->params[1] / pow(fac, m->gamma / (m->gamma - 1.));
          ghost[0]         = pg / (287.046 * Tg);
          ghost[1]         = Ma * sqrt(m->gamma * 287.046 * Tg) * ghost[0];
          for (int d = 1; d < D; ++d)
            ghost[d + 1] = 0.0;
          double rho2u2 = 0.0;
          for (int d = 0; d < D; ++d)
            rho2u2 += ghost[d + 1] * ghost[d + 1];
          ghost[NEQ - 1] = pg / gm1 + 0.5 * (rho2u2 / ghost[0]);
        }
        else
        {
          /* WeakSubOutlet.hpp:105-190: interior state with the outlet pressure */
          const double gm1 = m->gamma - 1.;
          for (int i = 0; i < NEQ - 1; ++i)
            ghost[i] = uqf[i];
          double rho2u2 = 0.0;
          for (int d = 0; d < D; ++d)
            rho2u2 += uqf[d + 1] * uqf[d + 1];
          ghost[NEQ - 1] = b->params[0] / gm1 + 0.5 * rho2u2 / uqf[0];
        }
        for (int e = 0; e < NEQ; ++e)
          ghost[e] -= uqf[e];
        for (int i = 0; i < NEQ; ++i)
        {
          double s = Km[i][0] * ghost[0];
          for (int k = 1; k < NEQ; ++k)
            s = s + Km[i][k] * ghost[k];
          gflux[i] = s;
        }
      }
      for (int e = 0; e < NEQ; ++e)
        total[e] += wq * gflux[e];
      for (int n = 0; n < b->nfdof; ++n)
        for (int e = 0; e < NEQ; ++e)
          bres[n][e] += relax * b->fV[(size_t)q * b->nfdof + n] * wq * gflux[e];
    }

    for (int e = 0; e < NEQ; ++e)
    {
      double sum = 0.0;
      for (int n = 0; n < b->nfdof; ++n)
        sum += bres[n][e];
      if (fabs(sum) > 1.e-14)
      {
        const double scale = total[e] / sum;
        for (int n = 0; n < b->nfdof; ++n)
          bres[n][e] *= scale;
      }
    }

    for (int n = 0; n < b->nfdof; ++n)
    {
      const int v   = dofs[n];
      const double V = vol[v];
      ws[v] += V * coeff[n];
      const double iv = 1. / V;
      for (int e = 0; e < NEQ; ++e)
        res[(size_t)v * NEQ + e] += iv * bres[n][e];
    }
  }
  return bad;
}

/* StrongDirichletBC::apply (StrongDirichletBC.hpp:202-233): the facet dofs take the condition's
 * values, facet by facet in order (a dof shared by two facets keeps the later value). */
static void apply_strong_bc(const rdso_model *m, const rdso_bc *b, double *u)
{
  const int NEQ = m->neq;
  for (int f = 0; f < b->nfacets; ++f)
    for (int n = 0; n < b->nfdof; ++n)
    {
      const int v = b->sol_conn[(size_t)f * b->nfdof + n];
      for (int e = 0; e < NEQ; ++e)
        u[(size_t)v * NEQ + e] = b->gq[((size_t)f * b->nfdof + n) * NEQ + e];
    }
}

int rdso_assemble(const rdso_model *m, const rdso_cells *groups, int ngroups, const rdso_bc *bcs,
                  int nbcs, int nnodes, const double *geo_coords, const double *vol,
                  double *u, double cfl, double *res, double *ws, double *dt)
{
  const int D = m->dim, NEQ = m->neq;
  int bad = 0;
  for (size_t i = 0; i < (size_t)nnodes * NEQ; ++i)
    res[i] = 0.0;
  for (int i = 0; i < nnodes; ++i)
    ws[i] = 0.0;

  for (int ig = 0; ig < ngroups; ++ig)
  {
    const rdso_cells *g = &groups[ig];
    for (int c = 0; c < g->ncells; ++c)
    {
      double X[NGEO_MAX * DIM_MAX], un[NDOF_MAX * NEQ_MAX];
      for (int k = 0; k < g->ngeo; ++k)
        for (int d = 0; d < D; ++d)
          X[k * D + d] = geo_coords[(size_t)g->geo_conn[(size_t)c * g->ngeo + k] * D + d];
      const int *dofs = g->sol_conn + (size_t)c * g->ndof;
      for (int n = 0; n < g->ndof; ++n)
        for (int e = 0; e < NEQ; ++e)
          un[n * NEQ + e] = u[(size_t)dofs[n] * NEQ + e];
      double er[NDOF_MAX * NEQ_MAX], ew[NDOF_MAX];
      bad += cell_residual(m, g, X, un, er, ew);
      /* scatter (PGRDMExplicitCellWorker.hpp:549-567) */
      for (int n = 0; n < g->ndof; ++n)
      {
        const int v     = dofs[n];
        const double iv = 1. / vol[v];
        for (int e = 0; e < NEQ; ++e)
          res[(size_t)v * NEQ + e] += iv * er[n * NEQ + e];
        ws[v] += ew[n];
      }
    }
  }

  /* conditions in their (name) order: weak ones add facet residuals, strong ones overwrite
   * the state that the later conditions and the update see */
  for (int ib = 0; ib < nbcs; ++ib)
  {
    if (bcs[ib].kind == RDSO_BC_STRONG_DIRICHLET)
      apply_strong_bc(m, &bcs[ib], u);
    else
      bad += apply_weak_bc(m, &bcs[ib], geo_coords, vol, u, res, ws);
  }

  /* RDTimeUpdate::compute_local_time_step (RDTimeUpdate.cpp:41-53) */
  for (int i = 0; i < nnodes; ++i)
    dt[i] = cfl * vol[i] / ws[i];
  return bad;
}

void rdso_update(int nnodes, int neq, const double *dt, const double *res, double *u)
{
  for (int i = 0; i < nnodes; ++i)
    for (int e = 0; e < neq; ++e)
      u[(size_t)i * neq + e] -= dt[i] * res[(size_t)i * neq + e];
}

void rdso_residual_norm(int nnodes, int neq, const double *res, const double *dt, double *norm)
{
  for (int e = 0; e < neq; ++e)
    norm[e] = 0.0;
  for (int i = 0; i < nnodes; ++i)
    for (int e = 0; e < neq; ++e)
    {
      const double r = res[(size_t)i * neq + e] * dt[i];
      norm[e] += r * r;
    }
  for (int e = 0; e < neq; ++e)
    norm[e] = sqrt(norm[e] / nnodes);
}
