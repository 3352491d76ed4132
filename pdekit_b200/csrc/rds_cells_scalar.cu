// Cell residual kernels for the scalar 2D physics (constant-direction advection, Burgers) with
// the PGLDA / PGN / PGB distribution schemes. One thread per cell.
//
// Per cell this fuses what the reference does in three batched metric passes and one per-cell
// scheme call (src/solver/rdm/assembly/PGRDMExplicitCellWorker.hpp:406-545):
//   geometry   J = dVgeo X, detJ, invJ          (src/interpolation/GeometryMetric.hpp:364-440)
//   solution   u_q = V u                        (src/interpolation/SolutionSpaceMetric.hpp:288-327)
//   flux       F(Vsf u) at the p+1 flux nodes, d F_d / d x_d at q via invJ dVf F
//                                               (src/interpolation/FluxSpaceMetric.hpp:545-746)
//   scheme     k_n = a(u_q) . grad phi_n, K+ = max(k_n, 0), beta_n = K+_n / sum K+,
//              LDA part  sum_q w_q detJ_q beta_n r_q,
//              N part    sum_q w_q detJ_q beta_n sum_{m != n} K+_m (u_n - u_m)
//              PGB blends with theta = |Phi| / (sum_n |lda_n + diss_n| + 1e-6)
//                                               (src/solver/rdm/cellsplitters/PGLDA.hpp:171-310,
//                                                PGN.hpp:154-289, PGB.hpp:314-498)
//   wave speed |K| max_{q,n} max(1e-6, |k_n|)   (PGLDA.hpp:207-214,301-310)
// and writes the cell's nodal residuals and wave speed to its contribution slots; the node
// gather (rds_gather.cu) sums them in ascending cell order.
//
// Precision: T = double is the plain path. T = float evaluates interpolation, flux, upwind
// coefficients in FP32 and keeps the sum of K+ inverse, the accumulation over quadrature points
// and the nodal residual in FP64.

#include "rds_internal.h"
#include "rds_tables.cuh"

namespace rds
{

namespace
{

// EXT: the external nodal blending coefficient may be set (single contexts; batched contexts
// never hold one, and the branch costs their kernels registers)
template <int PHYS, int SCHEME, typename T, int NDOF, int NQ, int NFL, int NGEO, bool EXT = true>
__device__ __forceinline__ void scalar_cell(const CellArgs &a,
                                            const Tables<T, 2, NDOF, NQ, NFL, NGEO> &tb,
                                            const int c)
{
  // FP32 form: states and coordinates enter as deviations from the cell's first node, taken in
  // FP64 (u_n - u_0, X_g - X_0); interpolants and fluxes are written in those deviations
  // (the bases sum to one and their derivatives to zero), so FP32 round-off acts on terms of the
  // size of the variation across the cell instead of the size of the state, which keeps the
  // FP32 residual floor low. The FP64 form evaluates the reference's expressions as they are.
  constexpr bool DEV = sizeof(T) == 4;

  // ---- gather nodal state and geometry (SoA connectivity: coalesced index loads)
  double ud[NDOF];
  T un[NDOF];
#pragma unroll
  for (int n = 0; n < NDOF; ++n)
  {
    const int v = __ldg(a.sol_conn + (size_t)n * a.ncells + c);
    ud[n]       = __ldg(a.u + v);
    un[n]       = DEV ? T(ud[n] - ud[0]) : T(ud[n]);
  }
  const T u0 = T(ud[0]);

  // ---- straight-sided triangle: one Jacobian for all points
  T ij00, ij01, ij10, ij11, detj;
  {
    T X0[NGEO], X1[NGEO];
    double xg0 = 0.0, yg0 = 0.0;
#pragma unroll
    for (int g = 0; g < NGEO; ++g)
    {
      const int v     = __ldg(a.geo_conn + (size_t)g * a.ncells + c);
      const double xg = __ldg(a.X + v), yg = __ldg(a.X + a.ngeo_nodes + v);
      if (g == 0)
      {
        xg0 = xg;
        yg0 = yg;
      }
      X0[g] = DEV ? T(xg - xg0) : T(xg);
      X1[g] = DEV ? T(yg - yg0) : T(yg);
    }
    T J00 = tb.dVgeo[0][0][0] * X0[0], J01 = tb.dVgeo[0][0][0] * X1[0];
    T J10 = tb.dVgeo[1][0][0] * X0[0], J11 = tb.dVgeo[1][0][0] * X1[0];
#pragma unroll
    for (int g = 1; g < NGEO; ++g)
    {
      J00 = J00 + tb.dVgeo[0][0][g] * X0[g];
      J01 = J01 + tb.dVgeo[0][0][g] * X1[g];
      J10 = J10 + tb.dVgeo[1][0][g] * X0[g];
      J11 = J11 + tb.dVgeo[1][0][g] * X1[g];
    }
    detj            = J00 * J11 - J01 * J10;
    const T inv_det = T(1) / detj;
    ij00            = inv_det * J11;
    ij11            = inv_det * J00;
    ij01            = -inv_det * J01;
    ij10            = -inv_det * J10;
  }

  // ---- flux divergence at the points. F is the order p+1 Lagrange interpolant through the
  // flux nodes, F = (s^2/2, s) for Burgers and (a0 s, a1 s) for advection with s the state at
  // the node (FP32 form: s - u_0 and F(s) - F(u_0)). With invJ constant over the cell,
  //   r_q = sum_f dVf[0][q][f] G0_f + dVf[1][q][f] G1_f,
  //   G0_f = invJ00 F0_f + invJ10 F1_f,  G1_f = invJ01 F0_f + invJ11 F1_f,
  // i.e. the flux is contracted with invJ once per node instead of once per node and point.
  // The values r_q (and Phi = sum_q w_q detJ r_q) are formed first, so the contracted flux is
  // dead before the upwind loop; the rolled FP64 loop keeps them in shared memory.
  constexpr int QUNROLL = sizeof(T) == 8 ? 1 : NQ;
  constexpr bool RQ_SHARED = QUNROLL == 1;
  __shared__ T s_rq[RQ_SHARED ? NQ * kBlock : 1];
  T rq_reg[RQ_SHARED ? 1 : NQ];
  double phi = 0.0, vol = 0.0;
  {
    T G0[NFL], G1[NFL];
#pragma unroll
    for (int f = 0; f < NFL; ++f)
    {
      T s = DEV ? T(0) : tb.Vsf[f][0] * un[0];
#pragma unroll
      for (int n = 1; n < NDOF; ++n)
        s = s + tb.Vsf[f][n] * un[n];
      T F0, F1;
      if (PHYS == RDS_BURGERS2D)
      {
        F0 = DEV ? s * (u0 + T(0.5) * s) : T(0.5) * s * s;
        F1 = s;
      }
      else
      {
        F0 = T(a.adv0) * s;
        F1 = T(a.adv1) * s;
      }
      G0[f] = ij00 * F0 + ij10 * F1;
      G1[f] = ij01 * F0 + ij11 * F1;
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q)
    {
      T r = tb.dVf[0][q][0] * G0[0] + tb.dVf[1][q][0] * G1[0];
#pragma unroll
      for (int f = 1; f < NFL; ++f)
        r = r + tb.dVf[0][q][f] * G0[f] + tb.dVf[1][q][f] * G1[f];
      const double wj = double(tb.w[q] * detj);
      vol += wj;
      phi += wj * double(r);
      if constexpr (RQ_SHARED)
        s_rq[q * kBlock + threadIdx.x] = r;
      else
        rq_reg[q] = r;
    }
  }

  double lda[NDOF], diss[NDOF];
#pragma unroll
  for (int n = 0; n < NDOF; ++n)
  {
    lda[n]  = 0.0;
    diss[n] = 0.0;
  }
  T kmax = T(0);

  // FP64: the quadrature loop stays rolled (the unrolled P3 body overflows the instruction
  // cache); table entries are then indexed constant-bank loads. FP32: unrolled.
#pragma unroll QUNROLL
  for (int q = 0; q < NQ; ++q)
  {
    const double wj = double(tb.w[q] * detj);
    double rq;
    if constexpr (RQ_SHARED)
      rq = double(s_rq[q * kBlock + threadIdx.x]);
    else
      rq = double(rq_reg[q]);

    // advection speed at q
    T ax, ay;
    if (PHYS == RDS_BURGERS2D)
    {
      T uq = DEV ? T(0) : tb.V[q][0] * un[0];
#pragma unroll
      for (int n = 1; n < NDOF; ++n)
        uq = uq + tb.V[q][n] * un[n];
      if (DEV)
        uq = u0 + uq;
      ax = uq;
      ay = T(1);
    }
    else
    {
      ax = T(a.adv0);
      ay = T(a.adv1);
    }

    // upwind coefficients k_n = a . invJ^T grad_xi phi_n = dV[0][q][n] A + dV[1][q][n] B
    const T A = ax * ij00 + ay * ij10;
    const T B = ax * ij01 + ay * ij11;
    T kp[NDOF];
    T sumkp = T(0);
#pragma unroll
    for (int n = 0; n < NDOF; ++n)
    {
      const T k = tb.dV[0][q][n] * A + tb.dV[1][q][n] * B;
      kp[n]     = k > T(0) ? k : T(0);
      kmax      = fmax(kmax, fabs(k));
      sumkp     = sumkp + kp[n];
    }
    // beta_n = K+_n / sum K+ (FP64 inverse in both precisions); w_q detJ beta_n is e K+_n
    const double e = wj * (1.0 / double(sumkp));

    const double erq = e * rq;
#pragma unroll
    for (int n = 0; n < NDOF; ++n)
      lda[n] += erq * double(kp[n]);
    if (SCHEME != RDS_PGLDA)
    {
      // sum_{m != n} K+_m (u_n - u_m) = u_n sum_m K+_m - sum_m K+_m u_m (the m = n terms
      // cancel), so the N dissipation costs O(ndof) per point instead of O(ndof^2)
      double tku = 0.0;
#pragma unroll
      for (int m = 0; m < NDOF; ++m)
        tku += double(kp[m]) * ud[m];
      const double sk = double(sumkp);
#pragma unroll
      for (int n = 0; n < NDOF; ++n)
        diss[n] += (e * double(kp[n])) * (ud[n] * sk - tku);
    }
  }
  // wave speed |K| max_{q,n} max(1e-6, |k_n|)
  const T wsmax = fmax(T(1.e-6), kmax);

  double theta = 1.0;
  if (SCHEME == RDS_PGB)
  {
    double abs_phiN = 0.0;
#pragma unroll
    for (int n = 0; n < NDOF; ++n)
      abs_phiN += fabs(lda[n] + diss[n]);
    theta = fabs(phi) / (abs_phiN + 1.e-6);
    if (a.theta)
      a.theta[c] = theta;
  }

  double *out = a.contrib + a.slot_base + c;
  if (EXT && SCHEME == RDS_PGB && a.blend)
  {
    // external nodal blending coefficient: theta_n of the cell's nodes, the N part dropped
    // when all are below 1e-6 (PGRDMExplicitCellWorker.hpp:508-517, PGB.hpp:141-148,467-477)
    double tn[NDOF], tmax = 0.0;
#pragma unroll
    for (int n = 0; n < NDOF; ++n)
    {
      tn[n] = __ldg(a.blend + __ldg(a.sol_conn + (size_t)n * a.ncells + c));
      tmax  = fmax(tmax, tn[n]);
    }
    const bool skip = tmax < 1.e-6;
#pragma unroll
    for (int n = 0; n < NDOF; ++n)
      out[(size_t)n * a.ncells] = skip ? lda[n] : lda[n] + tn[n] * diss[n];
  }
  else if (SCHEME == RDS_PGPSI && fabs(phi) > 1.e-14)
  {
    // PSI: the N residuals limited with the reference's residual limiter
    // (LFResidualLimiter.hpp:37-110): x_n = max(phi_n / phi, 0) + 1e-12 (std::max's NaN
    // rule), phi_n = x_n / sum x * phi; cells with |phi| <= 1e-14 keep the N residuals
    double x[NDOF], sx = 0.0;
#pragma unroll
    for (int n = 0; n < NDOF; ++n)
    {
      const double r = (lda[n] + diss[n]) / phi;
      x[n]           = (r < 0.0 ? 0.0 : r) + 1.e-12;
      sx += x[n];
    }
#pragma unroll
    for (int n = 0; n < NDOF; ++n)
      out[(size_t)n * a.ncells] = x[n] / sx * phi;
  }
  else
  {
#pragma unroll
    for (int n = 0; n < NDOF; ++n)
    {
      const double r = (SCHEME == RDS_PGLDA) ? lda[n] : lda[n] + theta * diss[n];
      out[(size_t)n * a.ncells] = r; // write-back: the gather reads it from L2
    }
  }
  a.wsc[a.ws_base + c] = vol * double(wsmax);
}

// FP64 P3 Burgers cells: capped at 128 registers (4 blocks per SM instead of 3; 11 % faster,
// measured); 0 (no minimum) keeps the compiler's choice elsewhere (the cap slowed P3 advection)
template <int PHYS, typename T, int NDOF>
constexpr int kMinBlocks = (PHYS == RDS_BURGERS2D && NDOF >= 10 && sizeof(T) == 8) ? 4 : 0;

template <int PHYS, int SCHEME, typename T, int NDOF, int NQ, int NFL, int NGEO>
__global__ void __launch_bounds__(kBlock, kMinBlocks<PHYS, T, NDOF>)
    cells_scalar2d(const __grid_constant__ CellArgs a,
                   const __grid_constant__ Tables<T, 2, NDOF, NQ, NFL, NGEO> tb)
{
  pdl_wait_and_release();
  if (*a.stop)
    return;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncells)
    return;
  scalar_cell<PHYS, SCHEME, T, NDOF, NQ, NFL, NGEO>(a, tb, c);
}

// Batch form: a persistent grid walks the group's active tiles (the problems still iterating
// at this precision); a tile is blockDim.x consecutive cells of one problem, so every thread of
// a block maps to the same problem. Results per cell are those of cells_scalar2d.
template <int PHYS, int SCHEME, typename T, int NDOF, int NQ, int NFL, int NGEO>
__global__ void __launch_bounds__(128, kMinBlocks<PHYS, T, NDOF>)
    cells_scalar2d_batch(const __grid_constant__ CellArgs a,
                         const __grid_constant__ Tables<T, 2, NDOF, NQ, NFL, NGEO> tb)
{
  if (*a.stop)
    return;
  const int32_t *prefix = a.bt.prefix;
  const int np          = a.bt.nprob;
  const int total       = prefix[np];
  for (int t = blockIdx.x; t < total; t += gridDim.x)
  {
    // problem p with prefix[p] <= t < prefix[p+1] (prefix[0] = 0 <= t < prefix[np])
    int lo = 0, hi = np;
    while (hi - lo > 1)
    {
      const int mid = (lo + hi) >> 1;
      if (prefix[mid] <= t)
        lo = mid;
      else
        hi = mid;
    }
    const int c = a.bt.cbeg[lo] + (t - prefix[lo]) * (int)blockDim.x + (int)threadIdx.x;
    if (c < a.bt.cend[lo])
      scalar_cell<PHYS, SCHEME, T, NDOF, NQ, NFL, NGEO, false>(a, tb, c);
  }
}

template <int PHYS, int SCHEME, typename T, int NDOF, int NQ, int NFL, int NGEO>
cudaError_t launch_one(const HostCellGroup &g, const CellArgs &a, cudaStream_t s)
{
  Tables<T, 2, NDOF, NQ, NFL, NGEO> tb;
  fill_tables(tb, g.w, g.V, g.dV, g.dVgeo, g.dVf, g.Vsf);
  const int grid = (a.ncells + kBlock - 1) / kBlock;
  return launch_kernel(cells_scalar2d<PHYS, SCHEME, T, NDOF, NQ, NFL, NGEO>, dim3(grid),
                       dim3(kBlock), 0, s, a.pdl != 0, a, tb);
}

template <int PHYS, int SCHEME, typename T>
cudaError_t dispatch_shape(const HostCellGroup &g, const CellArgs &a, cudaStream_t s, bool *ok)
{
  const rds_cell_group &d = g.desc;
  *ok                     = true;
  if (d.shape == RDS_TRIAG && d.ngeo == 3)
  {
    // (order, quadrature points, flux nodes): P1/P4-rule, P1/P5, P2/P4, P2/P5, P3/P6, P3/P8
    if (d.ndof == 3 && d.nq == 6 && d.nfl == 6)
      return launch_one<PHYS, SCHEME, T, 3, 6, 6, 3>(g, a, s);
    if (d.ndof == 3 && d.nq == 7 && d.nfl == 6)
      return launch_one<PHYS, SCHEME, T, 3, 7, 6, 3>(g, a, s);
    if (d.ndof == 6 && d.nq == 6 && d.nfl == 10)
      return launch_one<PHYS, SCHEME, T, 6, 6, 10, 3>(g, a, s);
    if (d.ndof == 6 && d.nq == 7 && d.nfl == 10)
      return launch_one<PHYS, SCHEME, T, 6, 7, 10, 3>(g, a, s);
    if (d.ndof == 10 && d.nq == 12 && d.nfl == 15)
      return launch_one<PHYS, SCHEME, T, 10, 12, 15, 3>(g, a, s);
    if (d.ndof == 10 && d.nq == 16 && d.nfl == 15)
      return launch_one<PHYS, SCHEME, T, 10, 16, 15, 3>(g, a, s);
  }
  *ok = false;
  return cudaSuccess;
}

template <int PHYS, int SCHEME, typename T, int NDOF, int NQ, int NFL>
cudaError_t launch_batch_one(const HostCellGroup &g, const CellArgs &a, int grid, int tile,
                             cudaStream_t s)
{
  Tables<T, 2, NDOF, NQ, NFL, 3> tb;
  fill_tables(tb, g.w, g.V, g.dV, g.dVgeo, g.dVf, g.Vsf);
  auto k = cells_scalar2d_batch<PHYS, SCHEME, T, NDOF, NQ, NFL, 3>;
  // a persistent grid only balances if all its CTAs are resident at once: cap it at the
  // occupancy of this kernel and tile (computed once per tile size)
  static int per_sm[2] = {0, 0}, nsm = 0;
  const int ti = tile > 64 ? 1 : 0;
  if (per_sm[ti] == 0)
  {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[ti], k, tile, 0);
    if (per_sm[ti] < 1)
      per_sm[ti] = 1;
  }
  const int cap = per_sm[ti] * nsm;
  k<<<grid < cap ? grid : cap, tile, 0, s>>>(a, tb);
  return cudaGetLastError();
}

template <int PHYS, int SCHEME, typename T>
cudaError_t dispatch_batch(const HostCellGroup &g, const CellArgs &a, int grid, int tile,
                           cudaStream_t s, bool *ok)
{
  const rds_cell_group &d = g.desc;
  *ok                     = true;
  if (d.shape == RDS_TRIAG && d.ngeo == 3)
  {
    // straight-sided triangles, P1 / P4 rule, P2 / P5 rule, P3 / P6 and P8 rules
    if (d.ndof == 3 && d.nq == 6 && d.nfl == 6)
      return launch_batch_one<PHYS, SCHEME, T, 3, 6, 6>(g, a, grid, tile, s);
    if (d.ndof == 6 && d.nq == 7 && d.nfl == 10)
      return launch_batch_one<PHYS, SCHEME, T, 6, 7, 10>(g, a, grid, tile, s);
    if (d.ndof == 10 && d.nq == 12 && d.nfl == 15)
      return launch_batch_one<PHYS, SCHEME, T, 10, 12, 15>(g, a, grid, tile, s);
    if (d.ndof == 10 && d.nq == 16 && d.nfl == 15)
      return launch_batch_one<PHYS, SCHEME, T, 10, 16, 15>(g, a, grid, tile, s);
  }
  *ok = false;
  return cudaSuccess;
}

const char *kernel_name(int physics, int scheme)
{
  static const char *names[2][4] = {
      {"cells_adv_lda", "cells_adv_n", "cells_adv_b", "cells_adv_psi"},
      {"cells_burgers_lda", "cells_burgers_n", "cells_burgers_b", "cells_burgers_psi"}};
  return names[physics == RDS_BURGERS2D ? 1 : 0][scheme];
}

} // namespace

// Scalar-physics part of launch_cells (the Euler kernels live in rds_cells_euler.cu).
cudaError_t launch_cells_scalar(const HostCellGroup &g, const CellArgs &a, int physics,
                                int scheme, int precision, cudaStream_t s, const char **name,
                                bool *ok)
{
  *name = kernel_name(physics, scheme);
#define RDS_SCALAR_CASE(PH, SC)                                                                    \
  if (physics == PH && scheme == SC)                                                               \
    return precision == RDS_MIXED ? dispatch_shape<PH, SC, float>(g, a, s, ok)                     \
                                  : dispatch_shape<PH, SC, double>(g, a, s, ok);
  RDS_SCALAR_CASE(RDS_ADVECTION_CONST, RDS_PGLDA)
  RDS_SCALAR_CASE(RDS_ADVECTION_CONST, RDS_PGN)
  RDS_SCALAR_CASE(RDS_ADVECTION_CONST, RDS_PGB)
  RDS_SCALAR_CASE(RDS_BURGERS2D, RDS_PGLDA)
  RDS_SCALAR_CASE(RDS_BURGERS2D, RDS_PGN)
  RDS_SCALAR_CASE(RDS_BURGERS2D, RDS_PGB)
#undef RDS_SCALAR_CASE
  // PSI: FP64 contexts only
  if (scheme == RDS_PGPSI && precision != RDS_MIXED)
  {
    if (physics == RDS_ADVECTION_CONST)
      return dispatch_shape<RDS_ADVECTION_CONST, RDS_PGPSI, double>(g, a, s, ok);
    if (physics == RDS_BURGERS2D)
      return dispatch_shape<RDS_BURGERS2D, RDS_PGPSI, double>(g, a, s, ok);
  }
  *ok = false;
  return cudaSuccess;
}

cudaError_t launch_cells_scalar_batch(const HostCellGroup &g, const CellArgs &a, int precision,
                                      int grid, int tile, cudaStream_t s, const char **name,
                                      bool *ok)
{
  static const char *names[2][4][2] = {
      {{"cells_adv_lda_batch", "cells_adv_lda_batch_f32"},
       {"cells_adv_n_batch", "cells_adv_n_batch_f32"},
       {"cells_adv_b_batch", "cells_adv_b_batch_f32"},
       {"cells_adv_psi_batch", "cells_adv_psi_batch_f32"}},
      {{"cells_burgers_lda_batch", "cells_burgers_lda_batch_f32"},
       {"cells_burgers_n_batch", "cells_burgers_n_batch_f32"},
       {"cells_burgers_b_batch", "cells_burgers_b_batch_f32"},
       {"cells_burgers_psi_batch", "cells_burgers_psi_batch_f32"}}};
  const int physics = g.physics, scheme = g.scheme;
  *ok               = false;
  if ((physics != RDS_ADVECTION_CONST && physics != RDS_BURGERS2D) || scheme < 0 || scheme > 3 ||
      tile <= 0 || tile > 128 || grid <= 0)
    return cudaSuccess;
  *name = names[physics == RDS_BURGERS2D][scheme][precision == RDS_MIXED];
#define RDS_BATCH_CASE(PH, SC)                                                                     \
  if (physics == PH && scheme == SC)                                                               \
    return precision == RDS_MIXED ? dispatch_batch<PH, SC, float>(g, a, grid, tile, s, ok)         \
                                  : dispatch_batch<PH, SC, double>(g, a, grid, tile, s, ok);
  RDS_BATCH_CASE(RDS_ADVECTION_CONST, RDS_PGLDA)
  RDS_BATCH_CASE(RDS_ADVECTION_CONST, RDS_PGN)
  RDS_BATCH_CASE(RDS_ADVECTION_CONST, RDS_PGB)
  RDS_BATCH_CASE(RDS_BURGERS2D, RDS_PGLDA)
  RDS_BATCH_CASE(RDS_BURGERS2D, RDS_PGN)
  RDS_BATCH_CASE(RDS_BURGERS2D, RDS_PGB)
#undef RDS_BATCH_CASE
  if (scheme == RDS_PGPSI && precision != RDS_MIXED)
  {
    if (physics == RDS_ADVECTION_CONST)
      return dispatch_batch<RDS_ADVECTION_CONST, RDS_PGPSI, double>(g, a, grid, tile, s, ok);
    return dispatch_batch<RDS_BURGERS2D, RDS_PGPSI, double>(g, a, grid, tile, s, ok);
  }
  return cudaSuccess;
}

} // namespace rds
