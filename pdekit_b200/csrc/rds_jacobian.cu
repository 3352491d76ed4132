// Element Jacobians of the PGLDA, PGN and PGB schemes, the matrices the reference's
// Picard-linearised implicit solver assembles (src/solver/rdm/cellsplitters/PGLDA.hpp:316-536,
// PGN.hpp:296-440, PGB.hpp:505-690,
// called from src/solver/rdm/assembly/PGRDMPicardJacCellAssemblyWorker.hpp:370):
//
//   PGLDA  J_mn = sum_q w_q |J_q| (K+_m (sum_k K+_k)^-1) K_n
//   PGN    J_mn = sum_q w_q |J_q| (delta_mn K+_m - K+_m (sum_k K-_k)^-1 K-_n)
//   PGB    J_mn = PGLDA + theta sum_q w_q |J_q| (delta_mn K+_m - K+_m (sum_k K+_k)^-1 K+_n)
//          (PGB.hpp:505-690), theta the cell's blending coefficient of the residual (a.theta)
//
// with K+- = R max/min(Lambda, 0) L as in the residual and K_n the unclipped upwind matrix (the
// flux Jacobian in direction grad phi_n); the implicit PGN of the reference is the plain N
// scheme (its explicit PGN adds the N dissipation to LDA instead). One thread per (cell, row
// node m). Scalar physics keep the row in registers; Euler rows (NEQ x NDOF NEQ) are accumulated
// in the thread's own rows of the output, point by point. The output is [cell][ndof * neq][ndof * neq], row-major per cell, the
// element matrix before the division by the dual volumes that the reference applies when it
// assembles the global matrix.

#include "rds_internal.h"
#include "rds_physics.cuh"
#include "rds_tables.cuh"

namespace rds
{

namespace
{

// Inverse of a small matrix by Gauss-Jordan elimination with row partial pivoting (FP64).
template <int N>
__device__ __forceinline__ void gj_inverse(double A[N][N], double R[N][N])
{
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j)
      R[i][j] = (i == j) ? 1.0 : 0.0;
#pragma unroll
  for (int k = 0; k < N; ++k)
  {
    int piv    = k;
    double amx = fabs(A[k][k]);
#pragma unroll
    for (int i = k + 1; i < N; ++i)
      if (fabs(A[i][k]) > amx)
      {
        amx = fabs(A[i][k]);
        piv = i;
      }
#pragma unroll
    for (int i = k + 1; i < N; ++i)
      if (i == piv)
      {
#pragma unroll
        for (int j = 0; j < N; ++j)
        {
          double t = A[k][j];
          A[k][j]  = A[i][j];
          A[i][j]  = t;
          t        = R[k][j];
          R[k][j]  = R[i][j];
          R[i][j]  = t;
        }
      }
    const double inv = 1.0 / A[k][k];
#pragma unroll
    for (int j = 0; j < N; ++j)
    {
      A[k][j] *= inv;
      R[k][j] *= inv;
    }
#pragma unroll
    for (int i = 0; i < N; ++i)
      if (i != k)
      {
        const double f = A[i][k];
#pragma unroll
        for (int j = 0; j < N; ++j)
        {
          A[i][j] -= f * A[k][j];
          R[i][j] -= f * R[k][j];
        }
      }
  }
}

// Inverse Jacobian of the geometry map at point q (ij[x][xi] = d xi / d x) and its determinant.
template <int D, int NDOF, int NQ, int NFL, int NGEO>
__device__ __forceinline__ double inv_jacobian(const Tables<double, D, NDOF, NQ, NFL, NGEO> &tb,
                                               int q, const double (&X)[NGEO][D],
                                               double (&ij)[D][D])
{
  double J[D][D];
#pragma unroll
  for (int xi = 0; xi < D; ++xi)
#pragma unroll
    for (int x = 0; x < D; ++x)
    {
      double s = tb.dVgeo[xi][q][0] * X[0][x];
#pragma unroll
      for (int g = 1; g < NGEO; ++g)
        s = s + tb.dVgeo[xi][q][g] * X[g][x];
      J[xi][x] = s;
    }
  if constexpr (D == 2)
  {
    const double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    const double id  = 1.0 / det;
    ij[0][0]         = id * J[1][1];
    ij[1][1]         = id * J[0][0];
    ij[0][1]         = -id * J[0][1];
    ij[1][0]         = -id * J[1][0];
    return det;
  }
  else
  {
    const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    const double c01 = J[1][0] * J[2][2] - J[1][2] * J[2][0];
    const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    const double det = J[0][0] * c00 - J[0][1] * c01 + J[0][2] * c02;
    const double id  = 1.0 / det;
    ij[0][0]         = c00 * id;
    ij[0][1]         = -(J[0][1] * J[2][2] - J[0][2] * J[2][1]) * id;
    ij[0][2]         = (J[0][1] * J[1][2] - J[1][1] * J[0][2]) * id;
    ij[1][0]         = -c01 * id;
    ij[1][1]         = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
    ij[1][2]         = -(J[0][0] * J[1][2] - J[0][2] * J[1][0]) * id;
    ij[2][0]         = c02 * id;
    ij[2][1]         = -(J[0][0] * J[2][1] - J[0][1] * J[2][0]) * id;
    ij[2][2]         = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
    return det;
  }
}

template <int PHYS, int SCHEME, int D, int NEQ, int NDOF, int NQ, int NFL, int NGEO, bool AFFINE>
__global__ void __launch_bounds__(kBlock)
    cells_jacobian(const CellArgs a, const __grid_constant__ Tables<double, D, NDOF, NQ, NFL, NGEO> tb,
                   double *__restrict__ jac)
{
  constexpr int NR = NDOF * NEQ; // rows (and columns) of one element matrix
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)a.ncells * NDOF)
    return;
  const int c = (int)(t / NDOF), m = (int)(t % NDOF);

  double X[NGEO][D];
#pragma unroll
  for (int g = 0; g < NGEO; ++g)
  {
    const int v = __ldg(a.geo_conn + (size_t)g * a.ncells + c);
#pragma unroll
    for (int d = 0; d < D; ++d)
      X[g][d] = __ldg(a.X + (size_t)d * a.ngeo_nodes + v);
  }
  int dof[NDOF];
#pragma unroll
  for (int n = 0; n < NDOF; ++n)
    dof[n] = __ldg(a.sol_conn + (size_t)n * a.ncells + c);

  double ij[D][D];
  double det = 0.0;
  if (AFFINE)
    det = inv_jacobian(tb, 0, X, ij);

  double *rows = jac + ((size_t)c * NR + (size_t)m * NEQ) * NR; // this thread's NEQ rows

  if constexpr (NEQ == 1)
  {
    double row[NDOF], stab[NDOF];
#pragma unroll
    for (int n = 0; n < NDOF; ++n)
      row[n] = stab[n] = 0.0;
    for (int q = 0; q < NQ; ++q)
    {
      if (!AFFINE)
        det = inv_jacobian(tb, q, X, ij);
      const double wj = tb.w[q] * det;
      double ax = a.adv0, ay = a.adv1;
      if (PHYS == RDS_BURGERS2D)
      {
        double uq = 0.0;
#pragma unroll
        for (int n = 0; n < NDOF; ++n)
          uq += tb.V[q][n] * __ldg(a.u + dof[n]);
        ax = uq;
        ay = 1.0;
      }
      double k[NDOF], sumk = 0.0, kpm = 0.0;
#pragma unroll
      for (int n = 0; n < NDOF; ++n)
      {
        const double gx = ij[0][0] * tb.dV[0][q][n] + ij[0][1] * tb.dV[1][q][n];
        const double gy = ij[1][0] * tb.dV[0][q][n] + ij[1][1] * tb.dV[1][q][n];
        k[n]            = ax * gx + ay * gy;
        const double kp = k[n] > 0.0 ? k[n] : 0.0;
        if (SCHEME == RDS_PGN)
          sumk += k[n] < 0.0 ? k[n] : 0.0; // sum of K-
        else
          sumk += kp; // sum of K+
        if (n == m)
          kpm = kp;
      }
      const double beta = kpm * (1.0 / sumk);
#pragma unroll
      for (int n = 0; n < NDOF; ++n)
      {
        if (SCHEME == RDS_PGN)
        {
          const double km = k[n] < 0.0 ? k[n] : 0.0;
          row[n] += wj * ((n == m ? kpm : 0.0) - beta * km);
        }
        else
        {
          row[n] += wj * (beta * k[n]);
          if (SCHEME == RDS_PGB)
          {
            const double kp = k[n] > 0.0 ? k[n] : 0.0;
            stab[n] += (n == m) ? wj * (kpm - beta * kp) : -(wj * (beta * kp));
          }
        }
      }
    }
    const double theta = (SCHEME == RDS_PGB) ? a.theta[c] : 0.0;
#pragma unroll
    for (int n = 0; n < NDOF; ++n)
      rows[n] = (SCHEME == RDS_PGB) ? row[n] + theta * stab[n] : row[n];
  }
  else
  {
    for (int i = 0; i < NEQ; ++i)
      for (int j = 0; j < NR; ++j)
        rows[(size_t)i * NR + j] = 0.0;
    const double gamma = a.gamma;
    const double theta = (SCHEME == RDS_PGB) ? a.theta[c] : 0.0;
    for (int q = 0; q < NQ; ++q)
    {
      if (!AFFINE)
        det = inv_jacobian(tb, q, X, ij);
      const double wj = tb.w[q] * det;
      double uq[NEQ];
#pragma unroll
      for (int e = 0; e < NEQ; ++e)
      {
        double s = 0.0;
#pragma unroll
        for (int n = 0; n < NDOF; ++n)
          s += tb.V[q][n] * __ldg(a.u + (size_t)e * a.nnodes + dof[n]);
        uq[e] = s;
      }
      EulerProps<double, D> p;
      if (euler_props<double, D>(uq, gamma, p))
        atomicOr(a.status, kFlagNegPressure);
      EulerAcoustic<double, D> ac;
      euler_acoustic<double, D>(p, gamma, ac);
      auto grad = [&](int n, double (&g)[D]) {
#pragma unroll
        for (int x = 0; x < D; ++x)
        {
          double s = ij[x][0] * tb.dV[0][q][n];
#pragma unroll
          for (int xi = 1; xi < D; ++xi)
            s += ij[x][xi] * tb.dV[xi][q][n];
          g[x] = s;
        }
      };
      // sum of K+ over the nodes, and K+ of the row node
      double SK[NEQ][NEQ], Km[NEQ][NEQ];
#pragma unroll
      for (int i = 0; i < NEQ; ++i)
#pragma unroll
        for (int j = 0; j < NEQ; ++j)
          SK[i][j] = Km[i][j] = 0.0;
      for (int n = 0; n < NDOF; ++n)
      {
        double g[D], K[NEQ][NEQ];
        grad(n, g);
        euler_K_split<+1, double, D>(p, ac, g, K);
        if (n == m)
        {
#pragma unroll
          for (int i = 0; i < NEQ; ++i)
#pragma unroll
            for (int j = 0; j < NEQ; ++j)
              Km[i][j] = K[i][j];
        }
        if (SCHEME == RDS_PGN)
          euler_K_split<-1, double, D>(p, ac, g, K);
#pragma unroll
        for (int i = 0; i < NEQ; ++i)
#pragma unroll
          for (int j = 0; j < NEQ; ++j)
            SK[i][j] += K[i][j];
      }
      double inv[NEQ][NEQ];
      gj_inverse<NEQ>(SK, inv);
      double B[NEQ][NEQ]; // K+_m (sum K+)^-1, PGN: K+_m (sum K-)^-1
#pragma unroll
      for (int i = 0; i < NEQ; ++i)
#pragma unroll
        for (int j = 0; j < NEQ; ++j)
        {
          double s = 0.0;
#pragma unroll
          for (int k = 0; k < NEQ; ++k)
            s += Km[i][k] * inv[k][j];
          B[i][j] = s;
        }
      for (int n = 0; n < NDOF; ++n)
      {
        double g[D], K[NEQ][NEQ];
        grad(n, g);
        if (SCHEME == RDS_PGN)
          euler_K_split<-1, double, D>(p, ac, g, K);
        else
          euler_K_split<0, double, D>(p, ac, g, K);
        double Kp[NEQ][NEQ]; // PGB: K+_n for the stabilisation part
        if (SCHEME == RDS_PGB)
          euler_K_split<+1, double, D>(p, ac, g, Kp);
#pragma unroll
        for (int i = 0; i < NEQ; ++i)
#pragma unroll
          for (int j = 0; j < NEQ; ++j)
          {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < NEQ; ++k)
              s += B[i][k] * K[k][j];
            double v = (SCHEME == RDS_PGN) ? ((n == m ? Km[i][j] : 0.0) - s) : s;
            if (SCHEME == RDS_PGB)
            {
              double sp = 0.0;
#pragma unroll
              for (int k = 0; k < NEQ; ++k)
                sp += B[i][k] * Kp[k][j];
              v += theta * ((n == m ? Km[i][j] : 0.0) - sp);
            }
            rows[(size_t)i * NR + n * NEQ + j] += wj * v;
          }
      }
    }
  }
}

template <int PHYS, int SCHEME, int D, int NEQ, int NDOF, int NQ, int NFL, int NGEO>
cudaError_t launch_jac(const HostCellGroup &g, const CellArgs &a, double *jac, cudaStream_t s)
{
  Tables<double, D, NDOF, NQ, NFL, NGEO> tb;
  fill_tables(tb, g.w, g.V, g.dV, g.dVgeo, g.dVf, g.Vsf);
  const long long nt = (long long)a.ncells * NDOF;
  const unsigned grid = (unsigned)((nt + kBlock - 1) / kBlock);
  if (g.affine)
    cells_jacobian<PHYS, SCHEME, D, NEQ, NDOF, NQ, NFL, NGEO, true><<<grid, kBlock, 0, s>>>(a, tb, jac);
  else
    cells_jacobian<PHYS, SCHEME, D, NEQ, NDOF, NQ, NFL, NGEO, false><<<grid, kBlock, 0, s>>>(a, tb, jac);
  return cudaGetLastError();
}

template <int PHYS, int SCHEME, int D, int NEQ>
cudaError_t dispatch_jac(const HostCellGroup &g, const CellArgs &a, double *jac, cudaStream_t s,
                         bool *ok)
{
  const rds_cell_group &d = g.desc;
  *ok                     = true;
#define RDS_JAC(SHAPE, NGEO, NDOF, NQ, NFL)                                                        \
  if (d.shape == SHAPE && d.ngeo == NGEO && d.ndof == NDOF && d.nq == NQ && d.nfl == NFL)         \
    return launch_jac<PHYS, SCHEME, D, NEQ, NDOF, NQ, NFL, NGEO>(g, a, jac, s);
  if constexpr (D == 2)
  {
    RDS_JAC(RDS_TRIAG, 3, 3, 6, 6)
    RDS_JAC(RDS_TRIAG, 3, 3, 7, 6)
    RDS_JAC(RDS_TRIAG, 3, 6, 6, 10)
    RDS_JAC(RDS_TRIAG, 3, 6, 7, 10)
    RDS_JAC(RDS_TRIAG, 3, 10, 12, 15)
    RDS_JAC(RDS_TRIAG, 3, 10, 16, 15)
    if constexpr (NEQ > 1)
    {
      RDS_JAC(RDS_QUAD, 4, 4, 4, 9)
      RDS_JAC(RDS_QUAD, 4, 4, 8, 9)
      RDS_JAC(RDS_QUAD, 4, 9, 8, 16)
      RDS_JAC(RDS_QUAD, 4, 16, 20, 25)
    }
  }
  else
  {
    RDS_JAC(RDS_TETRA, 4, 4, 4, 10)
    RDS_JAC(RDS_TETRA, 4, 10, 11, 20)
    RDS_JAC(RDS_TETRA, 4, 10, 14, 20)
  }
#undef RDS_JAC
  *ok = false;
  return cudaSuccess;
}

// Block-CSR assembly: entry (i, j) of block b (row node v) = sum over the block's contributions
// k (in ascending group and cell order) of jac[off_k + i * nr_k + j] / V_v, each element entry
// scaled by the row node's inverse dual volume before the sum, as the reference hands them to its
// sparse matrix (PGRDMPicardJacCellAssemblyWorker.hpp:392-412).
__global__ void __launch_bounds__(kBlock)
    assemble_bsr(long long nvals, int neq, const int32_t *__restrict__ brow,
                 const int64_t *__restrict__ cptr, const int64_t *__restrict__ coff,
                 const int32_t *__restrict__ cnr, const double *__restrict__ jac,
                 const double *__restrict__ vol, double *__restrict__ values)
{
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nvals)
    return;
  const int bs         = neq * neq;
  const long long b    = t / bs;
  const int r          = (int)(t % bs);
  const int ei = r / neq, ej = r % neq;
  const double iv      = 1. / vol[brow[b]];
  double s             = 0.0;
  for (long long k = cptr[b]; k < cptr[b + 1]; ++k)
    s += iv * jac[coff[k] + (long long)ei * cnr[k] + ej];
  values[t] = s;
}

} // namespace

cudaError_t launch_assemble_bsr(long long nnzb, int neq, const int32_t *brow, const int64_t *cptr,
                                const int64_t *coff, const int32_t *cnr, const double *jac,
                                const double *vol, double *values, cudaStream_t s)
{
  const long long nvals = nnzb * neq * neq;
  if (nvals == 0)
    return cudaSuccess;
  assemble_bsr<<<(unsigned)((nvals + kBlock - 1) / kBlock), kBlock, 0, s>>>(
      nvals, neq, brow, cptr, coff, cnr, jac, vol, values);
  return cudaGetLastError();
}

cudaError_t launch_jacobians(const HostCellGroup &g, const CellArgs &a, int physics, int scheme,
                             int dim, int neq, double *jac, cudaStream_t s)
{
  bool ok         = false;
  cudaError_t err = cudaSuccess;
  auto by_scheme = [&](auto lda, auto n, auto b) {
    return scheme == RDS_PGN ? n() : scheme == RDS_PGB ? b() : lda();
  };
#define RDS_JAC_PHYS(P, D, NEQ)                                                                    \
  by_scheme([&] { return dispatch_jac<P, RDS_PGLDA, D, NEQ>(g, a, jac, s, &ok); },                \
            [&] { return dispatch_jac<P, RDS_PGN, D, NEQ>(g, a, jac, s, &ok); },                  \
            [&] { return dispatch_jac<P, RDS_PGB, D, NEQ>(g, a, jac, s, &ok); })
  if (physics == RDS_ADVECTION_CONST && dim == 2 && neq == 1)
    err = RDS_JAC_PHYS(RDS_ADVECTION_CONST, 2, 1);
  else if (physics == RDS_BURGERS2D && dim == 2 && neq == 1)
    err = RDS_JAC_PHYS(RDS_BURGERS2D, 2, 1);
  else if (physics == RDS_EULER2D && dim == 2 && neq == 4)
    err = RDS_JAC_PHYS(RDS_EULER2D, 2, 4);
  else if (physics == RDS_EULER3D && dim == 3 && neq == 5)
    err = RDS_JAC_PHYS(RDS_EULER3D, 3, 5);
#undef RDS_JAC_PHYS
  if (!ok)
    return cudaErrorNotSupported;
  return err;
}

} // namespace rds
