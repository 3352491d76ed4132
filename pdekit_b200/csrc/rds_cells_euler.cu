// Cell residual kernels for the 2D / 3D Euler equations (PGLDA / PGN / PGB): a group of G
// lanes of one warp works on one cell.
//
// The reference's per-cell work (src/solver/rdm/cellsplitters/PGLDA.hpp:171-310,
// PGN.hpp:154-289, PGB.hpp:314-498 with the metrics of src/interpolation/*Metric.hpp) is split
// over the group as follows:
//   A  stage the cell's nodal states (ndof x neq, FP64) in shared memory;
//   B  flux nodes f = lane, lane + G, ...: S_f = Vsf u, F(S_f)            -> shared memory;
//   C  quadrature points q = lane, lane + G, ...: u_q = V u and the flux divergence
//      r_q = sum_d (invJ dVf F_d)_d                                       -> shared memory;
//   D1 quadrature points q = lane, lane + G, ...: the upwind matrices of all nodes in the split
//      form K+_n = oc I + rp lp^T + rm lm^T (Euler2DCons.hpp:316-536 / Euler3DCons.hpp:332-560;
//      euler_K_factors), summed into sum K+ (and sum K+ (u - u_0) for N / B) without storing
//      any K+_n; one solve per point with sum K+ (2D: closed-form adjugate, as the reference's
//      4 x 4 inverse; 3D: FP64 LU with partial pivoting) for v = (sum K+)^-1 r_q and
//      u_bar - u_0 = (sum K+)^-1 sum_m K+_m (u_m - u_0)                   -> shared memory;
//   D2 nodes n = lane, lane + G, ...: for every point the factors of K+_n again, applied in
//      factored form:  lda_n += w_q |J_q| K+_n v  and  diss_n += w_q |J_q| K+_n (u_n - u_bar)
//      (= sum_{m != n} K+_n (sum K+)^-1 K+_m (u_n - u_m), the reference's N dissipation);
//   E  PGB blending theta = |Phi_0| / (sum_n |lda_n0 + diss_n0| + 1e-6) with a group sum,
//      nodal residuals to the contribution slots, cell wave speed |K| max lambda.
// T is the arithmetic type of B, C and the upwind matrices; the LU, the solves and all
// accumulations are FP64 in both precisions.

#include "rds_internal.h"
#include "rds_physics.cuh"
#include "rds_tables.cuh"

namespace rds
{

namespace
{

template <int G>
__device__ __forceinline__ double group_sum(double v)
{
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int G>
__device__ __forceinline__ double group_max(double v)
{
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1)
    v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Solve A x = b for two right-hand sides (LU with row partial pivoting, FP64).
// TWO = false: b2 is left alone (PGLDA needs only the first right-hand side; the first is
// computed with the same operations either way).
template <int N, bool TWO = true>
__device__ __forceinline__ void lu_solve2(double A[N][N], double b1[N], double b2[N])
{
  double rdiag[N]; // 1 / U_kk, reused by the back substitution
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
    if (piv != k)
    {
#pragma unroll
      for (int j = 0; j < N; ++j)
      {
        // swap rows k and piv without dynamic register indexing
#pragma unroll
        for (int i = k + 1; i < N; ++i)
          if (i == piv)
          {
            const double t = A[k][j];
            A[k][j]        = A[i][j];
            A[i][j]        = t;
          }
      }
#pragma unroll
      for (int i = k + 1; i < N; ++i)
        if (i == piv)
        {
          double t = b1[k];
          b1[k]    = b1[i];
          b1[i]    = t;
          if (TWO)
          {
            t     = b2[k];
            b2[k] = b2[i];
            b2[i] = t;
          }
        }
    }
    const double inv = 1.0 / A[k][k];
    rdiag[k]         = inv;
#pragma unroll
    for (int i = k + 1; i < N; ++i)
    {
      const double f = A[i][k] * inv;
#pragma unroll
      for (int j = k + 1; j < N; ++j)
        A[i][j] -= f * A[k][j];
      b1[i] -= f * b1[k];
      if (TWO)
        b2[i] -= f * b2[k];
    }
  }
#pragma unroll
  for (int i = N - 1; i >= 0; --i)
  {
#pragma unroll
    for (int j = i + 1; j < N; ++j)
    {
      b1[i] -= A[i][j] * b1[j];
      if (TWO)
        b2[i] -= A[i][j] * b2[j];
    }
    b1[i] *= rdiag[i];
    if (TWO)
      b2[i] *= rdiag[i];
  }
}

// Solve A x = b for two right-hand sides, 4 x 4: x = adj(A) b / det(A), the adjugate from the
// 2 x 2 minors of rows (0, 1) and of rows (2, 3) (Laplace expansion by complementary minors).
// The reference inverts these matrices by a closed-form adjugate too
// (src/math/unary_ops/matrix_unary_ops/MatrixInverse.hpp:187-290).
template <bool TWO = true>
__device__ __forceinline__ void adj_solve4(const double A[4][4], double b1[4], double b2[4])
{
  const double s0 = A[0][0] * A[1][1] - A[1][0] * A[0][1];
  const double s1 = A[0][0] * A[1][2] - A[1][0] * A[0][2];
  const double s2 = A[0][0] * A[1][3] - A[1][0] * A[0][3];
  const double s3 = A[0][1] * A[1][2] - A[1][1] * A[0][2];
  const double s4 = A[0][1] * A[1][3] - A[1][1] * A[0][3];
  const double s5 = A[0][2] * A[1][3] - A[1][2] * A[0][3];
  const double c5 = A[2][2] * A[3][3] - A[3][2] * A[2][3];
  const double c4 = A[2][1] * A[3][3] - A[3][1] * A[2][3];
  const double c3 = A[2][1] * A[3][2] - A[3][1] * A[2][2];
  const double c2 = A[2][0] * A[3][3] - A[3][0] * A[2][3];
  const double c1 = A[2][0] * A[3][2] - A[3][0] * A[2][2];
  const double c0 = A[2][0] * A[3][1] - A[3][0] * A[2][1];
  const double det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
  const double id  = 1.0 / det;
  const double B[4][4] = {
      {A[1][1] * c5 - A[1][2] * c4 + A[1][3] * c3, -A[0][1] * c5 + A[0][2] * c4 - A[0][3] * c3,
       A[3][1] * s5 - A[3][2] * s4 + A[3][3] * s3, -A[2][1] * s5 + A[2][2] * s4 - A[2][3] * s3},
      {-A[1][0] * c5 + A[1][2] * c2 - A[1][3] * c1, A[0][0] * c5 - A[0][2] * c2 + A[0][3] * c1,
       -A[3][0] * s5 + A[3][2] * s2 - A[3][3] * s1, A[2][0] * s5 - A[2][2] * s2 + A[2][3] * s1},
      {A[1][0] * c4 - A[1][1] * c2 + A[1][3] * c0, -A[0][0] * c4 + A[0][1] * c2 - A[0][3] * c0,
       A[3][0] * s4 - A[3][1] * s2 + A[3][3] * s0, -A[2][0] * s4 + A[2][1] * s2 - A[2][3] * s0},
      {-A[1][0] * c3 + A[1][1] * c1 - A[1][2] * c0, A[0][0] * c3 - A[0][1] * c1 + A[0][2] * c0,
       -A[3][0] * s3 + A[3][1] * s1 - A[3][2] * s0, A[2][0] * s3 - A[2][1] * s1 + A[2][2] * s0}};
  double x1[4], x2[4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
  {
    x1[i] = (B[i][0] * b1[0] + B[i][1] * b1[1] + B[i][2] * b1[2] + B[i][3] * b1[3]) * id;
    if (TWO)
      x2[i] = (B[i][0] * b2[0] + B[i][1] * b2[1] + B[i][2] * b2[2] + B[i][3] * b2[3]) * id;
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
  {
    b1[i] = x1[i];
    if (TWO)
      b2[i] = x2[i];
  }
}

// Inverse Jacobian and determinant at quadrature point q from the geometry nodes.
template <typename T, int D, int NDOF, int NQ, int NFL, int NGEO>
__device__ __forceinline__ T jacobian_at(const Tables<T, D, NDOF, NQ, NFL, NGEO> &tb, int q,
                                         const T (&X)[NGEO][D], T (&ij)[D][D])
{
  T J[D][D];
#pragma unroll
  for (int xi = 0; xi < D; ++xi)
#pragma unroll
    for (int x = 0; x < D; ++x)
    {
      T s = tb.dVgeo[xi][q][0] * X[0][x];
#pragma unroll
      for (int g = 1; g < NGEO; ++g)
        s = s + tb.dVgeo[xi][q][g] * X[g][x];
      J[xi][x] = s;
    }
  if constexpr (D == 2)
  {
    const T det     = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    const T inv_det = T(1) / det;
    ij[0][0]        = inv_det * J[1][1];
    ij[1][1]        = inv_det * J[0][0];
    ij[0][1]        = -inv_det * J[0][1];
    ij[1][0]        = -inv_det * J[1][0];
    return det;
  }
  else
  {
    const T c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    const T c01 = J[1][0] * J[2][2] - J[1][2] * J[2][0];
    const T c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    const T det = J[0][0] * c00 - J[0][1] * c01 + J[0][2] * c02;
    const T inv = T(1) / det;
    ij[0][0]    = c00 * inv;
    ij[0][1]    = -(J[0][1] * J[2][2] - J[0][2] * J[2][1]) * inv;
    ij[0][2]    = (J[0][1] * J[1][2] - J[1][1] * J[0][2]) * inv;
    ij[1][0]    = -c01 * inv;
    ij[1][1]    = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * inv;
    ij[1][2]    = -(J[0][0] * J[1][2] - J[0][2] * J[1][0]) * inv;
    ij[2][0]    = c02 * inv;
    ij[2][1]    = -(J[0][0] * J[2][1] - J[0][1] * J[2][0]) * inv;
    ij[2][2]    = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * inv;
    return det;
  }
}

// The same from a lane-indexed geometry table dvg [D][NGEO][NQ] (global memory).
template <typename T, int D, int NQ, int NGEO>
__device__ __forceinline__ T jacobian_lt(const T *__restrict__ dvg, int q, const T (&X)[NGEO][D],
                                         T (&ij)[D][D])
{
  Tables<T, D, 1, 1, 1, NGEO> t1; // only dVgeo[.][0][.] is read
#pragma unroll
  for (int xi = 0; xi < D; ++xi)
#pragma unroll
    for (int g = 0; g < NGEO; ++g)
      t1.dVgeo[xi][0][g] = __ldg(dvg + (xi * NGEO + g) * NQ + q);
  return jacobian_at(t1, 0, X, ij);
}

template <typename T>
__device__ __forceinline__ T ldt(const T *p)
{
  return __ldg(p);
}

// Lane-indexed copies of a cell group's tables in global memory (read through L1): the entries
// that the lanes of a warp read at different points (phases C, D1), flux nodes (B) or nodes (D2),
// each laid out with that index fastest, so that a warp's reads fall in one or two sectors. The
// kernel-parameter copy (constant bank, whose reads at different addresses are serialised) keeps
// the reads that are uniform across the warp. Offsets in elements; euler_lane_tables fills it.
template <int D, int NDOF, int NQ, int NFL, int NGEO>
struct LaneTab
{
  static constexpr int VSF  = 0;                   // Vsf [NDOF][NFL]
  static constexpr int V    = VSF + NDOF * NFL;    // V [NDOF][NQ]
  static constexpr int DVF  = V + NDOF * NQ;       // dVf [D][NFL][NQ]
  static constexpr int DVG  = DVF + D * NFL * NQ;  // dVgeo [D][NGEO][NQ]
  static constexpr int DVQ  = DVG + D * NGEO * NQ; // dV [D][NDOF][NQ] (lanes over points)
  static constexpr int DVN  = DVQ + D * NDOF * NQ; // dV [D][NQ][NDOF] (lanes over nodes)
  static constexpr int W    = DVN + D * NQ * NDOF; // w [NQ]
  static constexpr int SIZE = W + NQ;
};

// Shared-memory footprint per cell (bytes): nodal states (FP64), the flux values of one chunk of
// NFC flux nodes in phases B-C aliased with the per-point solutions of D1 (FP64, 8-byte
// aligned: u_bar - u_0, and for T = float also v, which otherwise overwrites r_q), u_q and r_q.
// Strides are odd numbers of elements so that the lanes of a warp, which work on different
// cells, fall on different banks.
template <typename T, int D, int NDOF, int NQ, int NFL, int NFC>
struct EulerSmem
{
  static constexpr int odd(int n) { return n | 1; }
  static constexpr int NEQ   = D + 2;
  static constexpr int U     = odd(NDOF * NEQ); // doubles per cell
  static constexpr int FK_F  = NFC * NEQ * D;   // T (phases B-C)
  static constexpr int FK_S  = sizeof(T) == 8 ? NQ * NEQ : (2 * NQ * NEQ + 1) * 2; // T (D1-D2)
  static constexpr int FK    = odd(FK_F > FK_S ? FK_F : FK_S);
  static constexpr int QV    = NQ * NEQ;        // T, u_q then r_q
  static constexpr int QV2   = odd(2 * QV);
  static constexpr int BYTES = U * 8 + FK * (int)sizeof(T) + QV2 * (int)sizeof(T);
};

template <int PHYS, int SCHEME, typename T, int NDOF, int NQ, int NFL, int NGEO, bool AFFINE,
          int G, int NT, int NCH, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    cells_euler(const CellArgs a, const Tables<T, (PHYS == RDS_EULER3D ? 3 : 2), NDOF, NQ, NFL,
                                                NGEO> tb)
{
  constexpr int D   = (PHYS == RDS_EULER3D) ? 3 : 2;
  constexpr int NEQ = D + 2;
  constexpr int NPT = (NDOF + G - 1) / G; // nodes per lane
  constexpr int NFC = (NFL + NCH - 1) / NCH; // flux nodes per chunk
  using SM          = EulerSmem<T, D, NDOF, NQ, NFL, NFC>;
  using LT          = LaneTab<D, NDOF, NQ, NFL, NGEO>;
  // 2D: divergent table reads from the lane-indexed copy; 3D keeps the kernel-parameter tables
  // (its 96-cell blocks leave too little L1 next to their shared memory)
  constexpr bool LTB       = (D == 2);
  const T *__restrict__ lt = static_cast<const T *>(a.lt);
  auto tVsf = [&](int f, int n) -> T {
    if constexpr (LTB)
      return ldt(lt + LT::VSF + n * NFL + f);
    else
      return tb.Vsf[f][n];
  };
  auto tV = [&](int q, int n) -> T {
    if constexpr (LTB)
      return ldt(lt + LT::V + n * NQ + q);
    else
      return tb.V[q][n];
  };
  auto tdVf = [&](int xi, int q, int f) -> T {
    if constexpr (LTB)
      return ldt(lt + LT::DVF + (xi * NFL + f) * NQ + q);
    else
      return tb.dVf[xi][q][f];
  };
  auto tdVq = [&](int xi, int q, int n) -> T { // lanes over points
    if constexpr (LTB)
      return ldt(lt + LT::DVQ + (xi * NDOF + n) * NQ + q);
    else
      return tb.dV[xi][q][n];
  };
  auto tdVn = [&](int xi, int q, int n) -> T { // lanes over nodes
    if constexpr (LTB)
      return ldt(lt + LT::DVN + (xi * NQ + q) * NDOF + n);
    else
      return tb.dV[xi][q][n];
  };
  auto tw = [&](int q) -> T {
    if constexpr (LTB)
      return ldt(lt + LT::W + q);
    else
      return tb.w[q];
  };
  constexpr int CPB = NT / G; // cells per block

  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (*a.stop)
    return;

  const int lane  = threadIdx.x % G;
  const int slot  = threadIdx.x / G; // cell within the block
  const int c     = blockIdx.x * CPB + slot;
  const bool live = c < a.ncells;
  const int cc    = live ? c : a.ncells - 1; // dead groups shadow the last cell, write nothing

  // per-cell shared-memory regions
  double *su = reinterpret_cast<double *>(smem_raw) + (size_t)slot * SM::U;
  T *sfk = reinterpret_cast<T *>(reinterpret_cast<double *>(smem_raw) + (size_t)CPB * SM::U) +
           (size_t)slot * SM::FK;
  T *suq = reinterpret_cast<T *>(reinterpret_cast<double *>(smem_raw) + (size_t)CPB * SM::U) +
           (size_t)CPB * SM::FK + (size_t)slot * SM::QV2;
  T *srq = suq + SM::QV;

  // ---- A: nodal states
  for (int i = lane; i < NDOF * NEQ; i += G)
  {
    const int n = i / NEQ, e = i % NEQ;
    const int v = __ldg(a.sol_conn + (size_t)n * a.ncells + cc);
    su[i]       = __ldg(a.u + (size_t)e * a.nnodes + v);
  }
  T X[NGEO][D];
#pragma unroll
  for (int g = 0; g < NGEO; ++g)
  {
    const int v = __ldg(a.geo_conn + (size_t)g * a.ncells + cc);
#pragma unroll
    for (int d = 0; d < D; ++d)
      X[g][d] = T(__ldg(a.X + (size_t)d * a.ngeo_nodes + v));
  }
  __syncwarp();

  auto jac_q = [&](int q, T(&ij)[D][D]) -> T { // lanes over points
    if constexpr (LTB)
      return jacobian_lt<T, D, NQ, NGEO>(lt + LT::DVG, q, X, ij);
    else
      return jacobian_at(tb, q, X, ij);
  };

  const T gamma = T(a.gamma);
  bool bad      = false;

  // constant-Jacobian cells (simplices, parallelogram quadrilaterals): one Jacobian for all points
  T ijc[D][D];
  T detc = T(0);
  if (AFFINE)
    detc = jacobian_at(tb, 0, X, ijc);

  if constexpr (NCH == 1)
  {
    // ---- B: flux at the flux nodes; affine cells store it contracted with invJ,
    // G[f][e][xi] = sum_x invJ[x][xi] F[f][e][x], so that C needs D instead of D^2 products
    // per flux node and point. Table entries are read once each and applied to all equations
    // (every sum keeps its order over the nodes).
    for (int f = lane; f < NFL; f += G)
    {
      T s[NEQ];
      {
        const T c = tVsf(f, 0);
#pragma unroll
        for (int e = 0; e < NEQ; ++e)
          s[e] = c * T(su[e]);
      }
#pragma unroll
      for (int n = 1; n < NDOF; ++n)
      {
        const T c = tVsf(f, n);
#pragma unroll
        for (int e = 0; e < NEQ; ++e)
          s[e] = s[e] + c * T(su[n * NEQ + e]);
      }
      EulerProps<T, D> p;
      bad |= euler_props<T, D>(s, gamma, p);
      T F[NEQ][D];
      euler_flux<T, D>(s, p, F);
#pragma unroll
      for (int e = 0; e < NEQ; ++e)
#pragma unroll
        for (int d = 0; d < D; ++d)
        {
          T v = F[e][d];
          if (AFFINE)
          {
            v = ijc[0][d] * F[e][0];
#pragma unroll
            for (int x = 1; x < D; ++x)
              v = v + ijc[x][d] * F[e][x];
          }
          sfk[(f * NEQ + e) * D + d] = v;
        }
    }
    __syncwarp();

    // ---- C: u_q and flux divergence r_q (table entries read once each, as in B)
    for (int q = lane; q < NQ; q += G)
    {
      T uq[NEQ];
      {
        const T c = tV(q, 0);
#pragma unroll
        for (int e = 0; e < NEQ; ++e)
          uq[e] = c * T(su[e]);
      }
#pragma unroll
      for (int n = 1; n < NDOF; ++n)
      {
        const T c = tV(q, n);
#pragma unroll
        for (int e = 0; e < NEQ; ++e)
          uq[e] = uq[e] + c * T(su[n * NEQ + e]);
      }
#pragma unroll
      for (int e = 0; e < NEQ; ++e)
        suq[q * NEQ + e] = uq[e];
      if (AFFINE)
      {
        // r_e = sum_xi sum_f dVf[xi][q][f] G[f][e][xi]
        T r[NEQ];
#pragma unroll
        for (int e = 0; e < NEQ; ++e)
          r[e] = T(0);
#pragma unroll
        for (int xi = 0; xi < D; ++xi)
#pragma unroll
          for (int f = 0; f < NFL; ++f)
          {
            const T c = tdVf(xi, q, f);
#pragma unroll
            for (int e = 0; e < NEQ; ++e)
              r[e] = r[e] + c * sfk[(f * NEQ + e) * D + xi];
          }
#pragma unroll
        for (int e = 0; e < NEQ; ++e)
          srq[q * NEQ + e] = r[e];
      }
      else
      {
        // r_e = sum_ic sum_xi invJ[ic][xi] (sum_f dVf[xi][q][f] F[f][e][ic])
        T ij[D][D];
        jac_q(q, ij);
        T dref[NEQ][D][D]; // [e][ic][xi]
#pragma unroll
        for (int xi = 0; xi < D; ++xi)
        {
          {
            const T c = tdVf(xi, q, 0);
#pragma unroll
            for (int e = 0; e < NEQ; ++e)
#pragma unroll
              for (int ic = 0; ic < D; ++ic)
                dref[e][ic][xi] = c * sfk[(0 * NEQ + e) * D + ic];
          }
#pragma unroll
          for (int f = 1; f < NFL; ++f)
          {
            const T c = tdVf(xi, q, f);
#pragma unroll
            for (int e = 0; e < NEQ; ++e)
#pragma unroll
              for (int ic = 0; ic < D; ++ic)
                dref[e][ic][xi] = dref[e][ic][xi] + c * sfk[(f * NEQ + e) * D + ic];
          }
        }
#pragma unroll
        for (int e = 0; e < NEQ; ++e)
        {
          T r = T(0);
#pragma unroll
          for (int ic = 0; ic < D; ++ic)
          {
            T dphys = ij[ic][0] * dref[e][ic][0];
#pragma unroll
            for (int xi = 1; xi < D; ++xi)
              dphys = dphys + ij[ic][xi] * dref[e][ic][xi];
            r = r + dphys;
          }
          srq[q * NEQ + e] = r;
        }
      }
    }
    __syncwarp();
  }
  else
  {
    // ---- B and C, NCH chunks of NFC flux nodes (the flux region holds one chunk): the flux at
    // the chunk's nodes, then its part of every point's flux divergence r_q (and with the first
    // chunk u_q = V u). Affine cells store the flux contracted with invJ,
    // G[f][e][xi] = sum_x invJ[x][xi] F[f][e][x], so that C needs D instead of D^2 products per
    // flux node and point. Table entries are read once each and applied to all equations (every
    // sum keeps its order over the nodes).
#pragma unroll 1
    for (int ch = 0; ch < NCH; ++ch)
    {
      const int c0 = ch * NFC;
      for (int fl = lane; fl < NFC && c0 + fl < NFL; fl += G)
      {
        const int f = c0 + fl;
        T s[NEQ];
        {
          const T c = tVsf(f, 0);
#pragma unroll
          for (int e = 0; e < NEQ; ++e)
            s[e] = c * T(su[e]);
        }
#pragma unroll
        for (int n = 1; n < NDOF; ++n)
        {
          const T c = tVsf(f, n);
#pragma unroll
          for (int e = 0; e < NEQ; ++e)
            s[e] = s[e] + c * T(su[n * NEQ + e]);
        }
        EulerProps<T, D> p;
        bad |= euler_props<T, D>(s, gamma, p);
        T F[NEQ][D];
        euler_flux<T, D>(s, p, F);
#pragma unroll
        for (int e = 0; e < NEQ; ++e)
#pragma unroll
          for (int d = 0; d < D; ++d)
          {
            T v = F[e][d];
            if (AFFINE)
            {
              v = ijc[0][d] * F[e][0];
#pragma unroll
              for (int x = 1; x < D; ++x)
                v = v + ijc[x][d] * F[e][x];
            }
            sfk[(fl * NEQ + e) * D + d] = v;
          }
      }
      __syncwarp();

      for (int q = lane; q < NQ; q += G)
      {
        if (ch == 0)
        {
          T uq[NEQ];
          {
            const T c = tV(q, 0);
#pragma unroll
            for (int e = 0; e < NEQ; ++e)
              uq[e] = c * T(su[e]);
          }
#pragma unroll
          for (int n = 1; n < NDOF; ++n)
          {
            const T c = tV(q, n);
#pragma unroll
            for (int e = 0; e < NEQ; ++e)
              uq[e] = uq[e] + c * T(su[n * NEQ + e]);
          }
#pragma unroll
          for (int e = 0; e < NEQ; ++e)
            suq[q * NEQ + e] = uq[e];
        }
        T r[NEQ];
#pragma unroll
        for (int e = 0; e < NEQ; ++e)
          r[e] = ch == 0 ? T(0) : srq[q * NEQ + e];
        if (AFFINE)
        {
          // r_e += sum_xi sum_f dVf[xi][q][f] G[f][e][xi]
#pragma unroll
          for (int xi = 0; xi < D; ++xi)
#pragma unroll
            for (int fl = 0; fl < NFC; ++fl)
              if (c0 + fl < NFL)
              {
                const T c = tdVf(xi, q, c0 + fl);
#pragma unroll
                for (int e = 0; e < NEQ; ++e)
                  r[e] = r[e] + c * sfk[(fl * NEQ + e) * D + xi];
              }
        }
        else
        {
          // r_e += sum_ic sum_xi invJ[ic][xi] (sum_f dVf[xi][q][f] F[f][e][ic])
          T ij[D][D];
          jac_q(q, ij);
          T dref[NEQ][D][D]; // [e][ic][xi]
#pragma unroll
          for (int xi = 0; xi < D; ++xi)
          {
            {
              const T c = tdVf(xi, q, c0);
#pragma unroll
              for (int e = 0; e < NEQ; ++e)
#pragma unroll
                for (int ic = 0; ic < D; ++ic)
                  dref[e][ic][xi] = c * sfk[(0 * NEQ + e) * D + ic];
            }
#pragma unroll
            for (int fl = 1; fl < NFC; ++fl)
              if (c0 + fl < NFL)
              {
                const T c = tdVf(xi, q, c0 + fl);
#pragma unroll
                for (int e = 0; e < NEQ; ++e)
#pragma unroll
                  for (int ic = 0; ic < D; ++ic)
                    dref[e][ic][xi] = dref[e][ic][xi] + c * sfk[(fl * NEQ + e) * D + ic];
              }
          }
#pragma unroll
          for (int e = 0; e < NEQ; ++e)
          {
            T rr = T(0);
#pragma unroll
            for (int ic = 0; ic < D; ++ic)
            {
              T dphys = ij[ic][0] * dref[e][ic][0];
#pragma unroll
              for (int xi = 1; xi < D; ++xi)
                dphys = dphys + ij[ic][xi] * dref[e][ic][xi];
              rr = rr + dphys;
            }
            r[e] = ch == 0 ? rr : r[e] + rr;
          }
        }
#pragma unroll
        for (int e = 0; e < NEQ; ++e)
          srq[q * NEQ + e] = r[e];
      }
      __syncwarp();
    }
  }

  // ---- D1: quadrature points over the lanes; per point v = (sum K+)^-1 r_q and, for N / B,
  // u_bar - u_0 = (sum K+)^-1 sum_m K+_m (u_m - u_0), both FP64 in the flux region
  double *sfd = reinterpret_cast<double *>((reinterpret_cast<uintptr_t>(sfk) + 7) & ~uintptr_t(7));
  double *sv  = sizeof(T) == 8 ? reinterpret_cast<double *>(srq) : sfd + NQ * NEQ;
  double *sub = sfd;
  double phi0_l = 0.0; // this lane's points' part of Phi_0 = sum_q w_q |J_q| r_q0
  T wsmax       = T(0);
  for (int q = lane; q < NQ; q += G)
  {
    T ij[D][D];
    T det;
    if (AFFINE)
    {
      det = detc;
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j)
          ij[i][j] = ijc[i][j];
    }
    else
      det = jac_q(q, ij);
    T uq[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
      uq[e] = suq[q * NEQ + e];
    EulerProps<T, D> p;
    bad |= euler_props<T, D>(uq, gamma, p);
    EulerAcoustic<T, D> ac;
    euler_acoustic<T, D>(p, gamma, ac);

    double SK[NEQ][NEQ], SKu[NEQ];
#pragma unroll
    for (int i = 0; i < NEQ; ++i)
    {
      SKu[i] = 0.0;
#pragma unroll
      for (int j = 0; j < NEQ; ++j)
        SK[i][j] = 0.0;
    }
#pragma unroll 1
    for (int n = 0; n < NDOF; ++n)
    {
      T gphys[D];
#pragma unroll
      for (int x = 0; x < D; ++x)
      {
        T acc = ij[x][0] * tdVq(0, q, n);
#pragma unroll
        for (int xi = 1; xi < D; ++xi)
          acc = acc + ij[x][xi] * tdVq(xi, q, n);
        gphys[x] = acc;
      }
      EulerKFactors<T, D> f;
      wsmax = fmax(wsmax, euler_K_factors<+1, T, D>(p, ac, gphys, f));
      double rp[NEQ], rm[NEQ], lp[NEQ], lm[NEQ];
#pragma unroll
      for (int i = 0; i < NEQ; ++i)
      {
        rp[i] = double(f.rp[i]);
        rm[i] = double(f.rm[i]);
        lp[i] = double(f.lp[i]);
        lm[i] = double(f.lm[i]);
      }
#pragma unroll
      for (int i = 0; i < NEQ; ++i)
      {
#pragma unroll
        for (int j = 0; j < NEQ; ++j)
          SK[i][j] += rp[i] * lp[j] + rm[i] * lm[j];
        SK[i][i] += double(f.oc);
      }
      if (SCHEME != RDS_PGLDA)
      {
        // sum K+ (u - u_0): the solve then acts on the differences of the states (a nearly
        // uniform flow has them 100x smaller than the states), as the reference's
        // K+_m (u_n - u_m)
        double du[NEQ], pd = 0.0, md = 0.0;
#pragma unroll
        for (int j = 0; j < NEQ; ++j)
        {
          du[j] = su[n * NEQ + j] - su[j];
          pd += lp[j] * du[j];
          md += lm[j] * du[j];
        }
#pragma unroll
        for (int i = 0; i < NEQ; ++i)
          SKu[i] += double(f.oc) * du[i] + rp[i] * pd + rm[i] * md;
      }
    }
    double v[NEQ], ub[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
    {
      v[e]  = double(srq[q * NEQ + e]);
      ub[e] = SKu[e];
    }
    phi0_l += double(tw(q) * det) * v[0];
    if constexpr (NEQ == 4)
      adj_solve4<SCHEME != RDS_PGLDA>(SK, v, ub);
    else
      lu_solve2<NEQ, SCHEME != RDS_PGLDA>(SK, v, ub);
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
    {
      sv[q * NEQ + e] = v[e];
      if (SCHEME != RDS_PGLDA)
        sub[q * NEQ + e] = ub[e];
    }
  }
  __syncwarp();

  // ---- D2: nodes over the lanes, every point: K+_n v and K+_n (u_n - u_bar) in factored form
  double lda[NPT][NEQ], diss[NPT][NEQ];
#pragma unroll
  for (int s = 0; s < NPT; ++s)
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
    {
      lda[s][e]  = 0.0;
      diss[s][e] = 0.0;
    }
  double vol = 0.0;
#pragma unroll 1
  for (int q = 0; q < NQ; ++q)
  {
    T ij[D][D];
    T det;
    if (AFFINE)
    {
      det = detc;
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j)
          ij[i][j] = ijc[i][j];
    }
    else
      det = jacobian_at(tb, q, X, ij);
    const double wj = double(tb.w[q] * det);
    vol += wj;
    T uq[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
      uq[e] = suq[q * NEQ + e];
    EulerProps<T, D> p;
    euler_props<T, D>(uq, gamma, p);
    EulerAcoustic<T, D> ac;
    euler_acoustic<T, D>(p, gamma, ac);
    double v[NEQ], ub[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
    {
      v[e]  = sv[q * NEQ + e];
      ub[e] = (SCHEME != RDS_PGLDA) ? sub[q * NEQ + e] : 0.0;
    }
#pragma unroll
    for (int s = 0; s < NPT; ++s)
    {
      const int n = lane + s * G;
      if (n < NDOF)
      {
        T gphys[D];
#pragma unroll
        for (int x = 0; x < D; ++x)
        {
          T acc = ij[x][0] * tdVn(0, q, n);
#pragma unroll
          for (int xi = 1; xi < D; ++xi)
            acc = acc + ij[x][xi] * tdVn(xi, q, n);
          gphys[x] = acc;
        }
        EulerKFactors<T, D> f;
        euler_K_factors<+1, T, D>(p, ac, gphys, f);
        const double oc = double(f.oc);
        double pv = 0.0, mv = 0.0;
#pragma unroll
        for (int j = 0; j < NEQ; ++j)
        {
          pv += double(f.lp[j]) * v[j];
          mv += double(f.lm[j]) * v[j];
        }
#pragma unroll
        for (int i = 0; i < NEQ; ++i)
          lda[s][i] += wj * (oc * v[i] + double(f.rp[i]) * pv + double(f.rm[i]) * mv);
        if (SCHEME != RDS_PGLDA)
        {
          double du[NEQ], pd = 0.0, md = 0.0; // u_n - u_bar = (u_n - u_0) - (u_bar - u_0)
#pragma unroll
          for (int j = 0; j < NEQ; ++j)
          {
            du[j] = (su[n * NEQ + j] - su[j]) - ub[j];
            pd += double(f.lp[j]) * du[j];
            md += double(f.lm[j]) * du[j];
          }
#pragma unroll
          for (int i = 0; i < NEQ; ++i)
            diss[s][i] += wj * (oc * du[i] + double(f.rp[i]) * pd + double(f.rm[i]) * md);
        }
      }
    }
  }
  const double phi0 = group_sum<G>(phi0_l);

  // ---- E: blending, outputs
  double theta = 1.0;
  if (SCHEME == RDS_PGB)
  {
    double part = 0.0;
#pragma unroll
    for (int s = 0; s < NPT; ++s)
      if (lane + s * G < NDOF)
        part += fabs(lda[s][0] + diss[s][0]);
    const double abs_phiN = group_sum<G>(part);
    theta                 = fabs(phi0) / (abs_phiN + 1.e-6);
  }
  const double wmax = group_max<G>(double(wsmax));
  // external nodal blending coefficient: theta_n of the lane's nodes, the N part dropped when
  // all of the cell's are below 1e-6 (PGRDMExplicitCellWorker.hpp:508-517,
  // PGB.hpp:141-148,467-477); the group max runs in every lane of the warp
  double tn[NPT];
  bool skip = false;
  if (SCHEME == RDS_PGB && a.blend)
  {
    double tmax = 0.0;
#pragma unroll
    for (int s = 0; s < NPT; ++s)
    {
      const int n = lane + s * G;
      tn[s]       = (live && n < NDOF) ? __ldg(a.blend + __ldg(a.sol_conn + (size_t)n * a.ncells + c))
                                       : 0.0;
      tmax        = fmax(tmax, tn[s]);
    }
    skip = group_max<G>(tmax) < 1.e-6;
  }
  if (live)
  {
#pragma unroll
    for (int s = 0; s < NPT; ++s)
    {
      const int n = lane + s * G;
      if (n < NDOF)
      {
        const long long slot0 = a.slot_base + (long long)n * a.ncells + c;
#pragma unroll
        for (int e = 0; e < NEQ; ++e)
        {
          double r = (SCHEME == RDS_PGLDA) ? lda[s][e] : lda[s][e] + theta * diss[s][e];
          if (SCHEME == RDS_PGB && a.blend)
            r = skip ? lda[s][e] : lda[s][e] + tn[s] * diss[s][e];
          a.contrib[e * a.S + slot0] = r; // write-back: the gather reads it from L2
        }
      }
    }
    if (lane == 0)
    {
      a.wsc[a.ws_base + c] = vol * wmax;
      if (SCHEME == RDS_PGB && a.theta)
        a.theta[c] = theta;
    }
    if (bad)
      atomicOr(a.status, kFlagNegPressure);
  }
}

// NT: threads per block; NCH: chunks of the flux nodes (shared memory per cell), MINB: blocks
// per SM the register allocation must allow (0: the compiler's own choice, which for blocks of
// 128 threads is usually 3; an explicit 1 lets it take all 255 registers). Euler 3D FP64 runs 96 cells in a block of 384
// threads with the flux in 3 chunks (2.3 KB per cell instead of 3.9 KB: 12 warps per SM instead
// of 7); the FP64 P3 triangles and quadrilaterals (25 points) take 3 blocks of 128 threads per
// SM (12 warps).
template <int PHYS, int SCHEME, typename T, int NDOF, int NQ, int NFL, int NGEO, int G,
          int NT = kBlock, int NCH = 1, int MINB = 0>
cudaError_t launch_euler(const HostCellGroup &g, const CellArgs &a, cudaStream_t s)
{
  constexpr int D = (PHYS == RDS_EULER3D) ? 3 : 2;
  Tables<T, D, NDOF, NQ, NFL, NGEO> tb;
  fill_tables(tb, g.w, g.V, g.dV, g.dVgeo, g.dVf, g.Vsf);
  constexpr int CPB = NT / G;
  constexpr int NFC = (NFL + NCH - 1) / NCH;
  static_assert((NCH - 1) * NFC < NFL, "every chunk of flux nodes must be non-empty");
  using SM = EulerSmem<T, D, NDOF, NQ, NFL, NFC>;
  static_assert(CPB * SM::BYTES <= 227 * 1024, "per-block shared memory above the sm_100 limit");
  const int smem = CPB * SM::BYTES;
  const int grid = (a.ncells + CPB - 1) / CPB;
  // the shared-memory opt-in is set once per instantiation (not a stream operation, so it
  // also stays out of captured graphs)
  static bool attr_set = false;
  auto k_aff = cells_euler<PHYS, SCHEME, T, NDOF, NQ, NFL, NGEO, true, G, NT, NCH, MINB>;
  auto k_gen = cells_euler<PHYS, SCHEME, T, NDOF, NQ, NFL, NGEO, false, G, NT, NCH, MINB>;
  if (!attr_set)
  {
    cudaError_t e = cudaFuncSetAttribute(k_aff, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_gen, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess)
      return e;
    attr_set = true;
  }
  CellArgs al = a;
  if constexpr (sizeof(T) == 8)
    al.lt = g.d_lt64;
  else
    al.lt = g.d_lt32;
  if (D == 2 && !al.lt)
    return cudaErrorInvalidValue;
  if (g.const_jac)
    k_aff<<<grid, NT, smem, s>>>(al, tb);
  else
    k_gen<<<grid, NT, smem, s>>>(al, tb);
  return cudaGetLastError();
}

template <int PHYS, int SCHEME, typename T>
cudaError_t dispatch_euler(const HostCellGroup &g, const CellArgs &a, cudaStream_t s, bool *ok)
{
  const rds_cell_group &d = g.desc;
  *ok                     = true;
  if constexpr (PHYS == RDS_EULER2D)
  {
    if (d.shape == RDS_TRIAG && d.ngeo == 3)
    {
      if (d.ndof == 3 && d.nq == 6 && d.nfl == 6)
        return launch_euler<PHYS, SCHEME, T, 3, 6, 6, 3, 4>(g, a, s);
      if (d.ndof == 6 && d.nq == 6 && d.nfl == 10)
        return launch_euler<PHYS, SCHEME, T, 6, 6, 10, 3, 4>(g, a, s);
      if (d.ndof == 6 && d.nq == 7 && d.nfl == 10)
        return launch_euler<PHYS, SCHEME, T, 6, 7, 10, 3, 4>(g, a, s);
      if (d.ndof == 10 && d.nq == 12 && d.nfl == 15)
        return launch_euler<PHYS, SCHEME, T, 10, 12, 15, 3, 4>(g, a, s);
      if (d.ndof == 10 && d.nq == 16 && d.nfl == 15)
        return launch_euler<PHYS, SCHEME, T, 10, 16, 15, 3, 4, kBlock, 1, (sizeof(T) == 8 ? 3 : 0)>(
            g, a, s);
    }
    if (d.shape == RDS_QUAD && d.ngeo == 4)
    {
      // P1 with the 2x2 Gauss rule (orders 2-3), P1 and P2 with the reference's 8-point rule of
      // orders 4-5 or a 3x3 Gauss rule, P3 with the reference's 20-point rule of order 8 or a 5x5
      // Gauss rule
      if (d.ndof == 4 && d.nq == 4 && d.nfl == 9)
        return launch_euler<PHYS, SCHEME, T, 4, 4, 9, 4, 4>(g, a, s);
      if (d.ndof == 4 && d.nq == 8 && d.nfl == 9)
        return launch_euler<PHYS, SCHEME, T, 4, 8, 9, 4, 4>(g, a, s);
      if (d.ndof == 4 && d.nq == 9 && d.nfl == 9)
        return launch_euler<PHYS, SCHEME, T, 4, 9, 9, 4, 4>(g, a, s);
      if (d.ndof == 9 && d.nq == 8 && d.nfl == 16)
        return launch_euler<PHYS, SCHEME, T, 9, 8, 16, 4, 4>(g, a, s);
      if (d.ndof == 9 && d.nq == 9 && d.nfl == 16)
        return launch_euler<PHYS, SCHEME, T, 9, 9, 16, 4, 4>(g, a, s);
      if (d.ndof == 16 && d.nq == 20 && d.nfl == 25)
        return launch_euler<PHYS, SCHEME, T, 16, 20, 25, 4, 8>(g, a, s);
      if (d.ndof == 16 && d.nq == 25 && d.nfl == 25)
        return launch_euler<PHYS, SCHEME, T, 16, 25, 25, 4, 8, kBlock, 1, (sizeof(T) == 8 ? 3 : 0)>(
            g, a, s);
    }
  }
  else
  {
    if (d.shape == RDS_TETRA && d.ngeo == 4)
    {
      // P1 with the order-2 rule (4 points), P2 with the order-4 (11) and order-5 (14) rules
      if (d.ndof == 4 && d.nq == 4 && d.nfl == 10)
        return launch_euler<PHYS, SCHEME, T, 4, 4, 10, 4, 4>(g, a, s);
      if (d.ndof == 10 && d.nq == 11 && d.nfl == 20)
        return launch_euler<PHYS, SCHEME, T, 10, 11, 20, 4, 4>(g, a, s);
      if (d.ndof == 10 && d.nq == 14 && d.nfl == 20)
      {
        if constexpr (sizeof(T) == 8)
          return launch_euler<PHYS, SCHEME, T, 10, 14, 20, 4, 4, 384, 3>(g, a, s);
        else
          return launch_euler<PHYS, SCHEME, T, 10, 14, 20, 4, 4>(g, a, s);
      }
    }
  }
  *ok = false;
  return cudaSuccess;
}

const char *euler_name(int physics, int scheme)
{
  static const char *names[2][3] = {{"cells_euler2d_lda", "cells_euler2d_n", "cells_euler2d_b"},
                                    {"cells_euler3d_lda", "cells_euler3d_n", "cells_euler3d_b"}};
  return names[physics == RDS_EULER3D ? 1 : 0][scheme];
}

} // namespace

void euler_lane_tables(const HostCellGroup &g, int dim, std::vector<double> &out)
{
  // the layout of LaneTab, with run-time sizes
  const int D = dim, NDOF = g.desc.ndof, NQ = g.desc.nq, NFL = g.desc.nfl, NGEO = g.desc.ngeo;
  out.assign((size_t)NDOF * NFL + (size_t)NDOF * NQ + (size_t)D * NFL * NQ + (size_t)D * NGEO * NQ +
                 2 * (size_t)D * NDOF * NQ + NQ,
             0.0);
  size_t o = 0;
  for (int n = 0; n < NDOF; ++n)
    for (int f = 0; f < NFL; ++f)
      out[o++] = g.Vsf[(size_t)f * NDOF + n];
  for (int n = 0; n < NDOF; ++n)
    for (int q = 0; q < NQ; ++q)
      out[o++] = g.V[(size_t)q * NDOF + n];
  for (int d = 0; d < D; ++d)
    for (int f = 0; f < NFL; ++f)
      for (int q = 0; q < NQ; ++q)
        out[o++] = g.dVf[((size_t)d * NQ + q) * NFL + f];
  for (int d = 0; d < D; ++d)
    for (int k = 0; k < NGEO; ++k)
      for (int q = 0; q < NQ; ++q)
        out[o++] = g.dVgeo[((size_t)d * NQ + q) * NGEO + k];
  for (int d = 0; d < D; ++d)
    for (int n = 0; n < NDOF; ++n)
      for (int q = 0; q < NQ; ++q)
        out[o++] = g.dV[((size_t)d * NQ + q) * NDOF + n];
  for (int d = 0; d < D; ++d)
    for (int q = 0; q < NQ; ++q)
      for (int n = 0; n < NDOF; ++n)
        out[o++] = g.dV[((size_t)d * NQ + q) * NDOF + n];
  for (int q = 0; q < NQ; ++q)
    out[o++] = g.w[q];
}

cudaError_t launch_cells_euler(const HostCellGroup &g, const CellArgs &a, int physics, int scheme,
                               int precision, cudaStream_t s, const char **name, bool *ok)
{
  *name = euler_name(physics, scheme);
#define RDS_EULER_CASE(PH, SC)                                                                     \
  if (physics == PH && scheme == SC)                                                               \
    return precision == RDS_MIXED ? dispatch_euler<PH, SC, float>(g, a, s, ok)                     \
                                  : dispatch_euler<PH, SC, double>(g, a, s, ok);
  RDS_EULER_CASE(RDS_EULER2D, RDS_PGLDA)
  RDS_EULER_CASE(RDS_EULER2D, RDS_PGN)
  RDS_EULER_CASE(RDS_EULER2D, RDS_PGB)
  RDS_EULER_CASE(RDS_EULER3D, RDS_PGLDA)
  RDS_EULER_CASE(RDS_EULER3D, RDS_PGN)
  RDS_EULER_CASE(RDS_EULER3D, RDS_PGB)
#undef RDS_EULER_CASE
  *ok = false;
  return cudaSuccess;
}

} // namespace rds
