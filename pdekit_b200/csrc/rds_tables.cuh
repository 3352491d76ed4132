// Reference-element tables carried to the kernels by value.
//
// A kernel's by-value parameters live in the constant bank. With the loops over quadrature
// points, dofs and flux nodes fully unrolled, every table index is a compile-time constant, so
// each table entry is consumed directly as a constant-bank operand of the FMA that needs it: no
// load instruction, no shared-memory traffic, and the same entry is broadcast to all threads of
// a warp (every thread works on a different cell of the same element type). The tables of the
// largest element type used here (P3 quadrilateral, 20 quadrature points, P4 flux basis) take
// 20 KB in FP64, inside the 32 KB parameter limit of CUDA 12.1+ on sm_70 and newer.
#pragma once

#include <cstring>
#include <vector>

namespace rds
{

template <typename T, int D, int NDOF, int NQ, int NFL, int NGEO>
struct Tables
{
  T w[NQ];
  T V[NQ][NDOF];
  T dV[D][NQ][NDOF];
  T dVgeo[D][NQ][NGEO];
  T dVf[D][NQ][NFL];
  T Vsf[NFL][NDOF];
};

template <typename T, int D, int NDOF, int NQ, int NFL, int NGEO>
inline void fill_tables(Tables<T, D, NDOF, NQ, NFL, NGEO> &t, const std::vector<double> &w,
                        const std::vector<double> &V, const std::vector<double> &dV,
                        const std::vector<double> &dVgeo, const std::vector<double> &dVf,
                        const std::vector<double> &Vsf)
{
  for (int q = 0; q < NQ; ++q)
    t.w[q] = T(w[q]);
  for (int q = 0; q < NQ; ++q)
    for (int n = 0; n < NDOF; ++n)
      t.V[q][n] = T(V[q * NDOF + n]);
  for (int d = 0; d < D; ++d)
    for (int q = 0; q < NQ; ++q)
    {
      for (int n = 0; n < NDOF; ++n)
        t.dV[d][q][n] = T(dV[(d * NQ + q) * NDOF + n]);
      for (int g = 0; g < NGEO; ++g)
        t.dVgeo[d][q][g] = T(dVgeo[(d * NQ + q) * NGEO + g]);
      for (int f = 0; f < NFL; ++f)
        t.dVf[d][q][f] = T(dVf[(d * NQ + q) * NFL + f]);
    }
  for (int f = 0; f < NFL; ++f)
    for (int n = 0; n < NDOF; ++n)
      t.Vsf[f][n] = T(Vsf[f * NDOF + n]);
}

} // namespace rds
