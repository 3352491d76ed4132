// Weak boundary-condition kernels: one thread per boundary facet.
//
// WeakDirichlet (src/solver/rdm/bc/WeakDirichletBC.hpp:159-265): at each facet quadrature
// point, K- = R min(Lambda,0) L for the facet normal, ghost flux K- (g - u_q), accumulated as
// V(q,n) w_q |J_q| K-(g - u_q) per facet dof and as the facet total; the dof residuals are then
// rescaled so that they sum to the facet total (src/solver/rdm/bc/WeakBC.hpp:786-832). The
// facet's wave speed is max_q max(1e-9, |lambda|) for every dof, entering the nodal wave speed
// multiplied by the dual volume (WeakBC.hpp:315-352).
//
// Facet normals are (dy/dxi, -dx/dxi)/|.| in 2D and the normalised cross product of the two
// tangents in 3D, with |J| the length / area factor (src/interpolation/GeometryMetric.hpp:560-660).

#include "rds_internal.h"
#include "rds_physics.cuh"

namespace rds
{

namespace
{

template <typename T, int D, int NFDOF, int NFQ, int NFGEO>
struct FacetTables
{
  T fw[NFQ];
  T fV[NFQ][NFDOF];
  T fdVgeo[D - 1][NFQ][NFGEO];
};

template <int PHYS, int D, int NEQ, int NFDOF, int NFQ, int NFGEO>
__global__ void __launch_bounds__(kBlock)
    bc_weak_dirichlet(const BCArgs a, const FacetTables<double, D, NFDOF, NFQ, NFGEO> tb)
{
  if (*a.stop)
    return;
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= a.nfacets)
    return;

  double X[NFGEO][D];
#pragma unroll
  for (int g = 0; g < NFGEO; ++g)
  {
    const int v = a.geo_conn[(size_t)g * a.nfacets + f];
#pragma unroll
    for (int d = 0; d < D; ++d)
      X[g][d] = a.X[(size_t)d * a.ngeo_nodes + v];
  }
  int dof[NFDOF];
  double un[NFDOF][NEQ];
#pragma unroll
  for (int n = 0; n < NFDOF; ++n)
  {
    dof[n] = a.sol_conn[(size_t)n * a.nfacets + f];
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
      un[n][e] = a.u[(size_t)e * a.nnodes + dof[n]];
  }

  double bres[NFDOF][NEQ], total[NEQ];
#pragma unroll
  for (int e = 0; e < NEQ; ++e)
  {
    total[e] = 0.0;
#pragma unroll
    for (int n = 0; n < NFDOF; ++n)
      bres[n][e] = 0.0;
  }
  double coeff = 0.0;
  bool bad     = false;

#pragma unroll
  for (int q = 0; q < NFQ; ++q)
  {
    double nrm[D], jd;
    if (D == 2)
    {
      double tx = tb.fdVgeo[0][q][0] * X[0][0], ty = tb.fdVgeo[0][q][0] * X[0][1];
#pragma unroll
      for (int g = 1; g < NFGEO; ++g)
      {
        tx = tx + tb.fdVgeo[0][q][g] * X[g][0];
        ty = ty + tb.fdVgeo[0][q][g] * X[g][1];
      }
      const double n0 = ty, n1 = -tx;
      jd                    = sqrt(n0 * n0 + n1 * n1);
      const double inv_norm = 1.0 / jd;
      nrm[0]                = inv_norm * n0;
      nrm[1]                = inv_norm * n1;
    }
    else
    {
      double t[2][3];
#pragma unroll
      for (int xi = 0; xi < 2; ++xi)
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
          double s = tb.fdVgeo[xi][q][0] * X[0][d];
#pragma unroll
          for (int g = 1; g < NFGEO; ++g)
            s = s + tb.fdVgeo[xi][q][g] * X[g][d];
          t[xi][d] = s;
        }
      const double n0 = t[0][1] * t[1][2] - t[0][2] * t[1][1];
      const double n1 = t[0][2] * t[1][0] - t[0][0] * t[1][2];
      const double n2 = t[0][0] * t[1][1] - t[0][1] * t[1][0];
      jd                    = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
      const double inv_norm = 1.0 / jd;
      nrm[0]                = inv_norm * n0;
      nrm[1]                = inv_norm * n1;
      nrm[D - 1]            = inv_norm * n2;
    }
    const double wq = jd * tb.fw[q];

    double uq[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
    {
      double s = tb.fV[q][0] * un[0][e];
#pragma unroll
      for (int n = 1; n < NFDOF; ++n)
        s = s + tb.fV[q][n] * un[n][e];
      uq[e] = s;
    }

    double eig_max = 1.e-9;
    double gflux[NEQ];
    {
      double K[NEQ][NEQ], lam[NEQ];
      if constexpr (NEQ == 1)
      {
        const double ax = (PHYS == RDS_BURGERS2D) ? uq[0] : a.adv0;
        const double ay = (PHYS == RDS_BURGERS2D) ? 1.0 : a.adv1;
        lam[0]  = ax * nrm[0] + ay * nrm[1];
        K[0][0] = lam[0] < 0.0 ? lam[0] : 0.0;
      }
      else
      {
        EulerProps<double, D> p;
        bad |= euler_props<double, D>(uq, a.gamma, p);
        double Kf[D + 2][D + 2], lamf[D + 2];
        euler_K<-1, double, D>(p, nrm, a.gamma, Kf, lamf);
#pragma unroll
        for (int i = 0; i < NEQ; ++i)
        {
          lam[i] = lamf[i];
#pragma unroll
          for (int j = 0; j < NEQ; ++j)
            K[i][j] = Kf[i][j];
        }
      }
      double ghost[NEQ];
#pragma unroll
      for (int e = 0; e < NEQ; ++e)
      {
        eig_max  = fmax(eig_max, fabs(lam[e]));
        ghost[e] = a.gq[((size_t)e * NFQ + q) * a.nfacets + f] - uq[e];
      }
#pragma unroll
      for (int i = 0; i < NEQ; ++i)
      {
        double s = K[i][0] * ghost[0];
#pragma unroll
        for (int k = 1; k < NEQ; ++k)
          s = s + K[i][k] * ghost[k];
        gflux[i] = s;
      }
    }
    coeff = fmax(coeff, eig_max);
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
    {
      total[e] += wq * gflux[e];
#pragma unroll
      for (int n = 0; n < NFDOF; ++n)
        bres[n][e] += tb.fV[q][n] * wq * gflux[e];
    }
  }

#pragma unroll
  for (int e = 0; e < NEQ; ++e)
  {
    double sum = 0.0;
#pragma unroll
    for (int n = 0; n < NFDOF; ++n)
      sum += bres[n][e];
    if (fabs(sum) > 1.e-14)
    {
      const double scale = total[e] / sum;
#pragma unroll
      for (int n = 0; n < NFDOF; ++n)
        bres[n][e] *= scale;
    }
  }

#pragma unroll
  for (int n = 0; n < NFDOF; ++n)
  {
    const long long slot = a.slot_base + (long long)n * a.nfacets + f;
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
      a.contrib[e * a.S + slot] = bres[n][e];
    a.wsc[a.ws_base + (long long)n * a.nfacets + f] = a.vol[dof[n]] * coeff;
  }
  if (bad)
    atomicOr(a.status, kFlagNegPressure);
}

template <int PHYS, int D, int NEQ, int NFDOF, int NFQ, int NFGEO>
cudaError_t launch_wd(const HostBC &b, const BCArgs &a, cudaStream_t s)
{
  FacetTables<double, D, NFDOF, NFQ, NFGEO> tb;
  for (int q = 0; q < NFQ; ++q)
  {
    tb.fw[q] = b.fw[q];
    for (int n = 0; n < NFDOF; ++n)
      tb.fV[q][n] = b.fV[q * NFDOF + n];
    for (int xi = 0; xi < D - 1; ++xi)
      for (int g = 0; g < NFGEO; ++g)
        tb.fdVgeo[xi][q][g] = b.fdVgeo[(xi * NFQ + q) * NFGEO + g];
  }
  const int grid = (a.nfacets + kBlock - 1) / kBlock;
  bc_weak_dirichlet<PHYS, D, NEQ, NFDOF, NFQ, NFGEO><<<grid, kBlock, 0, s>>>(a, tb);
  return cudaGetLastError();
}

template <int PHYS, int D, int NEQ>
cudaError_t dispatch_wd(const HostBC &b, const BCArgs &a, cudaStream_t s, bool *ok)
{
  const rds_bc_group &d = b.desc;
  *ok                   = true;
  if (D == 2 && d.nfgeo == 2)
  {
#define RDS_WD(NFDOF, NFQ)                                                                         \
  if (d.nfdof == NFDOF && d.nfq == NFQ)                                                            \
    return launch_wd<PHYS, D, NEQ, NFDOF, NFQ, 2>(b, a, s);
    RDS_WD(2, 3)
    RDS_WD(2, 4)
    RDS_WD(3, 3)
    RDS_WD(3, 4)
    RDS_WD(4, 5)
    RDS_WD(4, 4)
#undef RDS_WD
  }
  *ok = false;
  return cudaSuccess;
}

} // namespace

cudaError_t launch_bc(const HostBC &b, const BCArgs &a, int physics, int dim, int neq,
                      cudaStream_t s, const char **name)
{
  bool ok = false;
  cudaError_t err = cudaSuccess;
  *name = "bc_weak_dirichlet";
  if (b.desc.kind == RDS_BC_WEAK_DIRICHLET)
  {
    if (physics == RDS_ADVECTION_CONST && dim == 2 && neq == 1)
      err = dispatch_wd<RDS_ADVECTION_CONST, 2, 1>(b, a, s, &ok);
    else if (physics == RDS_BURGERS2D && dim == 2 && neq == 1)
      err = dispatch_wd<RDS_BURGERS2D, 2, 1>(b, a, s, &ok);
    else if (physics == RDS_EULER2D && dim == 2 && neq == 4)
      err = dispatch_wd<RDS_EULER2D, 2, 4>(b, a, s, &ok);
  }
  if (!ok)
    return cudaErrorNotSupported;
  return err;
}

} // namespace rds
