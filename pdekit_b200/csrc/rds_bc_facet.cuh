// One weak boundary facet (the body of rds_bc.cu's kernels), shared with the fused correction
// sweeps of the defect-correction loop (rds_cells_scalar_dc.cu). COHERENT: the state is read
// through L2 (ld.global.cg), as a kernel must that reads a state other blocks of the same
// launch have written.
#pragma once

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

template <int KIND, int PHYS, int D, int NEQ, int NFDOF, int NFQ, int NFGEO, bool COHERENT = false>
__device__ __forceinline__ void bc_weak_facet(const BCArgs &a,
                                              const FacetTables<double, D, NFDOF, NFQ, NFGEO> &tb,
                                              const int f)
{
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
      un[n][e] = COHERENT ? __ldcg(a.u + (size_t)e * a.nnodes + dof[n])
                          : a.u[(size_t)e * a.nnodes + dof[n]];
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
  double coeff       = 0.0;
  bool bad           = false;
  const double relax = (KIND == RDS_BC_WEAK_WALL) ? a.relax : 1.0;

#pragma unroll
  for (int q = 0; q < NFQ; ++q)
  {
    double nrm[D], jd;
    if constexpr (D == 2)
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

    double eig_max = (KIND == RDS_BC_WEAK_FARFIELD) ? 1.e-8 : 1.e-9;
    double gflux[NEQ];
    if constexpr (NEQ == 1)
    {
      // scalar: K = 1 * op(V . n) * 1
      const double ax  = (PHYS == RDS_BURGERS2D) ? uq[0] : a.adv0;
      const double ay  = (PHYS == RDS_BURGERS2D) ? 1.0 : a.adv1;
      const double lam = ax * nrm[0] + ay * nrm[1];
      const double km  = lam < 0.0 ? lam : 0.0;
      eig_max          = fmax(eig_max, fabs(lam));
      gflux[0]         = km * (a.gq[(size_t)q * a.nfacets + f] - uq[0]);
    }
    else
    {
      EulerProps<double, D> p;
      bad |= euler_props<double, D>(uq, a.gamma, p);
      double K[NEQ][NEQ], lam[NEQ];
      euler_K<-1, double, D>(p, nrm, a.gamma, K, lam);
#pragma unroll
      for (int e = 0; e < NEQ; ++e)
        eig_max = fmax(eig_max, fabs(lam[e]));
      if constexpr (KIND == RDS_BC_WEAK_SUPER_INLET)
      {
#pragma unroll
        for (int e = 0; e < NEQ; ++e)
          gflux[e] = 0.0;
      }
      else if constexpr (KIND == RDS_BC_WEAK_WALL)
      {
        double Fn[NEQ], Fg[NEQ], ug[NEQ];
        euler_flux_n<double, D>(uq, p, nrm, Fn);
        double vn = 0.0, v2_new = 0.0;
#pragma unroll
        for (int d = 0; d < D; ++d)
          vn += p.V[d] * nrm[d];
        ug[0] = p.rho;
#pragma unroll
        for (int d = 0; d < D; ++d)
        {
          ug[d + 1] = p.V[d] - vn * nrm[d];
          v2_new += ug[d + 1] * ug[d + 1];
          ug[d + 1] *= p.rho;
        }
        ug[D + 1] = uq[D + 1] + 0.5 * p.rho * (v2_new - p.v2);
        EulerProps<double, D> pg;
        bad |= euler_props<double, D>(ug, a.gamma, pg);
        euler_flux_n<double, D>(ug, pg, nrm, Fg);
#pragma unroll
        for (int e = 0; e < NEQ; ++e)
          gflux[e] = Fg[e] - Fn[e];
      }
      else
      {
        double ghost[NEQ];
        const double gm1 = a.gamma - 1.0;
        if constexpr (KIND == RDS_BC_WEAK_SUB_INLET)
        {
          const double Ma  = sqrt(p.v2) / p.a;
          const double fac = 1. + 0.5 * gm1 * Ma * Ma;
          const double Tg  = a.params[0] / fac;
          const double pg  = a.params[1] / pow(fac, a.gamma / (a.gamma - 1.));
          ghost[0]         = pg / (287.046 * Tg);
          ghost[1]         = Ma * sqrt(a.gamma * 287.046 * Tg) * ghost[0];
#pragma unroll
          for (int d = 1; d < D; ++d)
            ghost[d + 1] = 0.0;
          double rho2u2 = 0.0;
#pragma unroll
          for (int d = 0; d < D; ++d)
            rho2u2 += ghost[d + 1] * ghost[d + 1];
          ghost[NEQ - 1] = pg / gm1 + 0.5 * (rho2u2 / ghost[0]);
        }
        else if constexpr (KIND == RDS_BC_WEAK_SUB_OUTLET)
        {
#pragma unroll
          for (int i = 0; i < NEQ - 1; ++i)
            ghost[i] = uq[i];
          double rho2u2 = 0.0;
#pragma unroll
          for (int d = 0; d < D; ++d)
            rho2u2 += uq[d + 1] * uq[d + 1];
          ghost[NEQ - 1] = a.params[0] / gm1 + 0.5 * rho2u2 / uq[0];
        }
        else if constexpr (KIND == RDS_BC_WEAK_FARFIELD)
        {
#pragma unroll
          for (int e = 0; e < NEQ; ++e)
            ghost[e] = a.gq[e];
        }
        else if constexpr (KIND == RDS_BC_WEAK_SYMMETRY)
        {
          double vn = 0.0;
#pragma unroll
          for (int d = 0; d < D; ++d)
            vn += nrm[d] * p.V[d];
          ghost[0]       = uq[0];
          ghost[NEQ - 1] = uq[NEQ - 1];
#pragma unroll
          for (int d = 0; d < D; ++d)
            ghost[d + 1] = uq[0] * (p.V[d] - 2. * vn * nrm[d]);
        }
        else
        {
#pragma unroll
          for (int e = 0; e < NEQ; ++e)
            ghost[e] = a.gq[((size_t)e * NFQ + q) * a.nfacets + f];
        }
#pragma unroll
        for (int e = 0; e < NEQ; ++e)
          ghost[e] -= uq[e];
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
    }
    coeff = fmax(coeff, eig_max);
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
    {
      total[e] += wq * gflux[e];
#pragma unroll
      for (int n = 0; n < NFDOF; ++n)
        bres[n][e] += relax * tb.fV[q][n] * wq * gflux[e];
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

  if (NEQ == 1 && a.c32)
  {
    // correction sweep of the defect-correction loop: the change since the exact sweep, whose
    // contribution is still in contrib (FP64 difference, then FP32: relative to the change)
#pragma unroll
    for (int n = 0; n < NFDOF; ++n)
    {
      const long long slot = a.slot_base + (long long)n * a.nfacets + f;
      a.c32[slot]          = float(bres[n][0] - a.contrib[slot]);
    }
  }
  else
  {
#pragma unroll
    for (int n = 0; n < NFDOF; ++n)
    {
      const long long slot = a.slot_base + (long long)n * a.nfacets + f;
#pragma unroll
      for (int e = 0; e < NEQ; ++e)
        a.contrib[e * a.S + slot] = bres[n][e];
      a.wsc[a.ws_base + (long long)n * a.nfacets + f] = a.vol[dof[n]] * coeff;
    }
  }
  if (bad)
    atomicOr(a.status, kFlagNegPressure);
}

} // namespace

} // namespace rds
