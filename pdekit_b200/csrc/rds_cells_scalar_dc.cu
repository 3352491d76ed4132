// Mixed form, scalar physics: cell kernels of the FP32 correction sweeps of the defect-correction
// loop (rds_api.cu, run_loop_dc).
//
// Every m sweeps the loop evaluates the exact FP64 residual R64(u_r) at the current state u_r
// (the plain cell kernels, rds_cells_scalar.cu) and keeps its update dt R64(u_r). The m - 1
// sweeps in between advance u = u_r + d with the increment
//     R64(u_r) + dR_cells(d) + [R64_bc(u) - R64_bc(u_r)],
// where the boundary part is evaluated in FP64 at u (facets are few; rds_bc.cu writes the
// difference) and dR_cells(d) is the change of the cell residual computed HERE, in FP32, from
// d = u - u_r directly:
//   * the flux change is exact in d: Burgers F(s_r + ds) - F(s_r) = (ds (s_r + ds/2), ds),
//     advection a ds, at the p+1 flux nodes, contracted like the plain kernel;
//   * the distribution coefficients (K+_n, beta_n = K+_n / sum K+, the blending coefficient
//     theta of PGB) are those of u_r (Picard linearisation; for advection they do not depend
//     on u, so dR is then exact);
//   * LDA part  sum_q w_q detJ beta_n dr_q,
//     N part    sum_q w_q detJ beta_n sum_m K+_m (d_n - d_m).
// Every term is a product of a coefficient and a d-sized quantity, so FP32 round-off is relative
// to the correction itself and shrinks with it: the loop keeps converging past the FP32 floor
// of a plain FP32 residual, to the FP64 scheme's own fixed point (at a fixed point d = 0 and
// R64(u_r) = 0). No FP64 arithmetic is left in the cell loop; the changes are stored as FP32
// and summed by the node gather in FP64.
//
// Schemes follow src/solver/rdm/cellsplitters/PGLDA.hpp:171-310, PGN.hpp:154-289 and
// PGB.hpp:314-498 (the plain kernels restate them; this is their linearisation at u_r).

#include "rds_bc_facet.cuh"
#include "rds_gather_dc.cuh"
#include "rds_internal.h"
#include "rds_tables.cuh"

namespace rds
{

namespace
{

// What a cell's correction reads that stays the same within a cycle: its nodes, the reference
// state there (in deviation form too), its inverse Jacobian and the frozen blending coefficient.
template <int NDOF>
struct DcCellState
{
  int v[NDOF];
  double r[NDOF];
  float ut[NDOF], u0;
  float ij00, ij01, ij10, ij11, detj;
  float theta;
};

template <int SCHEME, int NDOF, int NQ, int NFL, int NGEO>
__device__ __forceinline__ void dc_cell_state(const DcCellArgs &a,
                                              const Tables<float, 2, NDOF, NQ, NFL, NGEO> &tb,
                                              const int c, DcCellState<NDOF> &st)
{
  using T = float;
  // reference state in deviation form (coefficients)
  double ur0 = 0.0;
#pragma unroll
  for (int n = 0; n < NDOF; ++n)
  {
    const int v    = __ldg(a.sol_conn + (size_t)n * a.ncells + c);
    const double r = __ldg(a.ur + v);
    if (n == 0)
      ur0 = r;
    st.v[n]  = v;
    st.r[n]  = r;
    st.ut[n] = T(r - ur0);
  }
  st.u0 = T(ur0);

  // straight-sided triangle (deviation form of the vertex coordinates)
  T &ij00 = st.ij00, &ij01 = st.ij01, &ij10 = st.ij10, &ij11 = st.ij11, &detj = st.detj;
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
      X0[g] = T(xg - xg0);
      X1[g] = T(yg - yg0);
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
  st.theta = (SCHEME == RDS_PGB) ? T(__ldg(a.theta + c)) : T(1);
}

// The cell's FP32 change from the correction d = u - u_r (the state is read each sweep).
// COHERENT: the state is read through L2 (ld.global.cg), as the fused sweeps must (other blocks
// of the same launch write it between sweeps)
template <int PHYS, int SCHEME, int NDOF, int NQ, int NFL, int NGEO, bool COHERENT>
__device__ __forceinline__ void dc_cell_sweep(const DcCellArgs &a,
                                              const Tables<float, 2, NDOF, NQ, NFL, NGEO> &tb,
                                              const int c, const DcCellState<NDOF> &st)
{
  using T = float;
  T dn[NDOF];
#pragma unroll
  for (int n = 0; n < NDOF; ++n)
  {
    const double uu = COHERENT ? __ldcg(a.u + st.v[n]) : __ldg(a.u + st.v[n]);
    dn[n]           = T(uu - st.r[n]);
  }
  const T *ut = st.ut;
  const T u0  = st.u0;
  const T ij00 = st.ij00, ij01 = st.ij01, ij10 = st.ij10, ij11 = st.ij11, detj = st.detj;

  // change of the flux divergence at the points, dr_q = sum_f dVf[.][q][f] dG_f, with the flux
  // change at each flux node contracted with invJ once (constant over the cell)
  T dr[NQ];
  {
    T G0[NFL], G1[NFL];
#pragma unroll
    for (int f = 0; f < NFL; ++f)
    {
      T ds = tb.Vsf[f][0] * dn[0];
#pragma unroll
      for (int n = 1; n < NDOF; ++n)
        ds = ds + tb.Vsf[f][n] * dn[n];
      T F0, F1;
      if (PHYS == RDS_BURGERS2D)
      {
        T sr = T(0); // s_r - u_r0 (the node-0 deviation basis sums to one)
#pragma unroll
        for (int n = 1; n < NDOF; ++n)
          sr = sr + tb.Vsf[f][n] * ut[n];
        F0 = ds * ((u0 + sr) + T(0.5) * ds);
        F1 = ds;
      }
      else
      {
        F0 = T(a.adv0) * ds;
        F1 = T(a.adv1) * ds;
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
      dr[q] = r;
    }
  }

  // d in deviation form for the N dissipation (sum_m K+_m (d_n - d_m) is invariant to a shift)
  T dd[NDOF];
#pragma unroll
  for (int n = 0; n < NDOF; ++n)
    dd[n] = dn[n] - dn[0];

  // With e = w_q detJ / sum K+ (so e sum K+ = w_q detJ), the LDA and blended N parts are
  //   sum_q e K+_n dr_q + theta sum_q e K+_n (d_n sum K+ - sum_m K+_m d_m)
  //   = sum_q K+_n [e (dr_q - theta sum_m K+_m d_m)] + theta d_n sum_q w_q detJ K+_n,
  // two FMAs per point and node (theta = 1 for PGN, the N part absent for PGLDA).
  const T theta = st.theta;
  T racc[NDOF], wacc[NDOF];
#pragma unroll
  for (int n = 0; n < NDOF; ++n)
  {
    racc[n] = T(0);
    wacc[n] = T(0);
  }

#pragma unroll
  for (int q = 0; q < NQ; ++q)
  {
    const T wj = tb.w[q] * detj;
    T ax, ay;
    if (PHYS == RDS_BURGERS2D)
    {
      T uq = T(0);
#pragma unroll
      for (int n = 1; n < NDOF; ++n)
        uq = uq + tb.V[q][n] * ut[n];
      ax = u0 + uq;
      ay = T(1);
    }
    else
    {
      ax = T(a.adv0);
      ay = T(a.adv1);
    }
    const T A = ax * ij00 + ay * ij10;
    const T B = ax * ij01 + ay * ij11;
    T kp[NDOF];
    T sumkp = T(0);
#pragma unroll
    for (int n = 0; n < NDOF; ++n)
    {
      const T k = tb.dV[0][q][n] * A + tb.dV[1][q][n] * B;
      kp[n]     = k > T(0) ? k : T(0);
      sumkp     = sumkp + kp[n];
    }
    const T e = __fdividef(wj, sumkp); // a coefficient: 2-ulp division is enough
    T ec;
    if (SCHEME == RDS_PGLDA)
      ec = e * dr[q];
    else
    {
      T tkd = T(0);
#pragma unroll
      for (int m = 1; m < NDOF; ++m)
        tkd = tkd + kp[m] * dd[m];
      ec = e * (dr[q] - theta * tkd);
    }
#pragma unroll
    for (int n = 0; n < NDOF; ++n)
    {
      racc[n] = racc[n] + kp[n] * ec;
      if (SCHEME != RDS_PGLDA)
        wacc[n] = wacc[n] + wj * kp[n];
    }
  }

  float *out = a.c32 + a.slot_base + c;
#pragma unroll
  for (int n = 0; n < NDOF; ++n)
    out[(size_t)n * a.ncells] =
        (SCHEME == RDS_PGLDA) ? racc[n] : racc[n] + (theta * dd[n]) * wacc[n];
}

template <int PHYS, int SCHEME, int NDOF, int NQ, int NFL, int NGEO, bool COHERENT = false>
__device__ __forceinline__ void dc_cell(const DcCellArgs &a,
                                        const Tables<float, 2, NDOF, NQ, NFL, NGEO> &tb,
                                        const int c)
{
  DcCellState<NDOF> st;
  dc_cell_state<SCHEME, NDOF, NQ, NFL, NGEO>(a, tb, c, st);
  dc_cell_sweep<PHYS, SCHEME, NDOF, NQ, NFL, NGEO, COHERENT>(a, tb, c, st);
}

template <int PHYS, int SCHEME, int NDOF, int NQ, int NFL, int NGEO>
__global__ void __launch_bounds__(kBlock)
    cells_scalar2d_dc(const __grid_constant__ DcCellArgs a,
                      const __grid_constant__ Tables<float, 2, NDOF, NQ, NFL, NGEO> tb)
{
  pdl_wait_and_release();
  if (*a.stop)
    return;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncells)
    return;
  dc_cell<PHYS, SCHEME, NDOF, NQ, NFL, NGEO>(a, tb, c);
}

// Batch form: a persistent grid walks the group's active tiles (the problems still iterating);
// a tile is blockDim.x consecutive cells of one problem. Results per cell are those of
// cells_scalar2d_dc.
template <int PHYS, int SCHEME, int NDOF, int NQ, int NFL, int NGEO>
__global__ void __launch_bounds__(128)
    cells_scalar2d_dc_batch(const __grid_constant__ DcCellArgs a,
                            const __grid_constant__ Tables<float, 2, NDOF, NQ, NFL, NGEO> tb)
{
  if (*a.stop)
    return;
  const int32_t *prefix = a.bt.prefix;
  const int np          = a.bt.nprob;
  const int total       = prefix[np];
  for (int t = blockIdx.x; t < total; t += gridDim.x)
  {
    // problem p with prefix[p] <= t < prefix[p+1]
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
      dc_cell<PHYS, SCHEME, NDOF, NQ, NFL, NGEO>(a, tb, c);
  }
}

// ---- fused correction sweeps ------------------------------------------------------------
// A small mesh's correction sweep is a chain of short launches (cells, facets, gather) whose
// cost is mostly their latency. dc_sweeps_fused runs the m - 1 correction sweeps between two
// exact sweeps in one launch: per sweep, phase 1 the cells' and facets' FP32 changes (a
// grid-stride loop over cells, then the facets of each condition), a grid barrier, phase 2 the
// node updates, a grid barrier. The arithmetic is that of the separate kernels (dc_cell,
// bc_weak_facet, dc_correction_node), so the results are theirs bit for bit; only the loads of
// what other blocks wrote in the same launch (the state, the changes) go through L2, and what
// stays the same within the cycle (a thread's first cell's connectivity, reference state and
// inverse Jacobian, its first node's entry slots, dt R64, dt / V and value) is read once into
// registers. Two forms: meshes whose items fit two per thread of one 16-CTA cluster run as a
// single thread-block cluster (co-scheduled by the launch) with the hardware cluster barrier;
// larger ones as a grid of at most what is resident at once (occupancy x SMs) with a barrier
// in global memory whose waits are bounded: a wait that gives up sets kFlagTimeout in the
// status word and the launch returns.

constexpr int kClusterCtas = 16; // the cluster form's CTAs (a non-portable cluster size)
// and threads per CTA: as many as the order's registers allow (P1 <= 102, P2 <= 128 a thread)
constexpr int cluster_threads(int ndof) { return ndof == 3 ? 640 : ndof == 6 ? 512 : 256; }

template <int NFDOF, int NFQ>
struct FusedFacetTables
{
  FacetTables<double, 2, NFDOF, NFQ, 2> t[kFuseMaxBC];
};

// Grid barrier: bar[0] counts arrivals, bar[1] is the generation. Both are zero at launch (the
// host clears them before every launch); the last block to arrive resets the count and
// advances the generation. Returns false when the wait gave up after `limit` polls. `extra`
// (a test option) raises the arrivals awaited beyond the grid, so that no wait completes.
__device__ __forceinline__ bool fused_barrier(unsigned *bar, int limit, int extra)
{
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0)
  {
    int ok           = 1;
    const unsigned g = __ldcg(bar + 1);
    __threadfence();
    if (atomicAdd(bar, 1u) == gridDim.x - 1 + (unsigned)extra)
    {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    }
    else
    {
      int t = 0;
      while (__ldcg(bar + 1) == g)
      {
        if (++t > limit)
        {
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

// Cluster form: the whole grid is one thread-block cluster (at most 16 CTAs, co-scheduled by
// the launch), and the barrier is the cluster's hardware barrier with release / acquire
// semantics at cluster scope (every block of the launch is in the cluster).
__device__ __forceinline__ void cluster_barrier()
{
  __syncwarp(); // the .aligned barrier wants converged warps
  asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
               "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

template <bool CLUSTER>
__device__ __forceinline__ bool sweep_barrier(const DcFusedArgs &a)
{
  if constexpr (CLUSTER)
  {
    cluster_barrier();
    return true;
  }
  else
    return fused_barrier(a.bar, a.wait_limit, a.test_extra);
}

template <int PHYS, int SCHEME, int NDOF, int NQ, int NFL, int NFDOF, int NFQ, int NT,
          bool CLUSTER>
__global__ void __launch_bounds__(NT)
    dc_sweeps_fused(const __grid_constant__ DcFusedArgs a,
                    const __grid_constant__ Tables<float, 2, NDOF, NQ, NFL, 3> tb,
                    const __grid_constant__ FusedFacetTables<NFDOF, NFQ> ft)
{
  if (*a.cell.stop)
    return;
  const int nthreads = gridDim.x * blockDim.x;
  const int tid      = blockIdx.x * blockDim.x + threadIdx.x;
  const int ncells   = a.cell.ncells;
  int nitems         = ncells;
  for (int k = 0; k < a.nbc; ++k)
    nitems += a.bc[k].nfacets;
  // a thread's first cell and first node are the same in every sweep: what they read that
  // does not change within the cycle is read once, into registers
  DcCellState<NDOF> cs;
  if (tid < ncells)
    dc_cell_state<SCHEME, NDOF, NQ, NFL, 3>(a.cell, tb, tid, cs);
  DcNodeState ns;
  if (tid < a.ga.nnodes)
    dc_node_state(a.ga, tid, ns);
  for (int sweep = 0; sweep < a.nsweeps; ++sweep)
  {
    for (int i = tid; i < nitems; i += nthreads)
    {
      if (i == tid && i < ncells)
        dc_cell_sweep<PHYS, SCHEME, NDOF, NQ, NFL, 3, true>(a.cell, tb, i, cs);
      else if (i < ncells)
        dc_cell<PHYS, SCHEME, NDOF, NQ, NFL, 3, true>(a.cell, tb, i);
      else
      {
        int j = i - ncells, k = 0;
        while (j >= a.bc[k].nfacets)
          j -= a.bc[k++].nfacets;
        bc_weak_facet<RDS_BC_WEAK_DIRICHLET, PHYS, 2, 1, NFDOF, NFQ, 2, true>(a.bc[k], ft.t[k], j);
      }
    }
    if (!sweep_barrier<CLUSTER>(a))
    {
      if (threadIdx.x == 0)
        atomicOr(a.status, kFlagTimeout);
      return;
    }
    for (int v = tid; v < a.ga.nnodes; v += nthreads)
    {
      if (v == tid)
        dc_node_sweep(a.ga, v, ns);
      else
        dc_correction_node<true>(a.ga, v);
    }
    if (sweep + 1 < a.nsweeps && !sweep_barrier<CLUSTER>(a))
    {
      if (threadIdx.x == 0)
        atomicOr(a.status, kFlagTimeout);
      return;
    }
  }
}

template <int PHYS, int SCHEME, int NDOF, int NQ, int NFL, int NFDOF, int NFQ>
cudaError_t launch_fused_one(const HostCellGroup &g, const HostBC *const *bcs,
                             const DcFusedArgs &a, cudaStream_t s, bool *cluster)
{
  Tables<float, 2, NDOF, NQ, NFL, 3> tb;
  fill_tables(tb, g.w, g.V, g.dV, g.dVgeo, g.dVf, g.Vsf);
  FusedFacetTables<NFDOF, NFQ> ft{};
  for (int k = 0; k < a.nbc; ++k)
  {
    const HostBC &b = *bcs[k];
    for (int q = 0; q < NFQ; ++q)
    {
      ft.t[k].fw[q] = b.fw[q];
      for (int n = 0; n < NFDOF; ++n)
        ft.t[k].fV[q][n] = b.fV[q * NFDOF + n];
      for (int gg = 0; gg < 2; ++gg)
        ft.t[k].fdVgeo[0][q][gg] = b.fdVgeo[q * 2 + gg];
    }
  }
  int items = a.cell.ncells;
  for (int j = 0; j < a.nbc; ++j)
    items += a.bc[j].nfacets;
  if (a.ga.nnodes > items)
    items = a.ga.nnodes;
  // small meshes (at most two items a thread): one cluster of kClusterCtas CTAs of NTC
  // threads and the hardware cluster barrier (no bounded-wait test there: the launch
  // co-schedules the cluster and the barrier is not a poll)
  constexpr int NTC = cluster_threads(NDOF);
  *cluster           = false;
  if (a.test_extra == 0 && items <= 2 * kClusterCtas * NTC)
  {
    auto kc = dc_sweeps_fused<PHYS, SCHEME, NDOF, NQ, NFL, NFDOF, NFQ, NTC, true>;
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    attr[0].id               = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClusterCtas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim              = dim3(kClusterCtas);
    cfg.blockDim             = dim3(NTC);
    cfg.attrs                = attr;
    cfg.numAttrs             = 1;
    // whether the cluster fits, asked once per kernel and process, on the device current at
    // the first call (one device a process, as the library is used; the first call usually
    // comes during a stream capture: the queries then run in relaxed capture mode and on no
    // stream)
    static int fits = -1;
    if (fits < 0)
    {
      cudaStreamCaptureMode mode = cudaStreamCaptureModeRelaxed;
      cudaThreadExchangeStreamCaptureMode(&mode);
      int nclusters = 0;
      cudaError_t e = cudaFuncSetAttribute(kc, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
      if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveClusters(&nclusters, kc, &cfg);
      fits = (e == cudaSuccess && nclusters >= 1) ? 1 : 0;
      cudaGetLastError();
      cudaThreadExchangeStreamCaptureMode(&mode);
    }
    if (fits == 1)
    {
      *cluster   = true;
      cfg.stream = s;
      return cudaLaunchKernelEx(&cfg, kc, a, tb, ft);
    }
  }
  auto k = dc_sweeps_fused<PHYS, SCHEME, NDOF, NQ, NFL, NFDOF, NFQ, kBlock, false>;
  // every block must be resident at once (the blocks wait for one another at the barriers):
  // the grid is capped at this kernel's occupancy on all SMs
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kBlock, 0);
  if (per_sm < 1)
    return cudaErrorInvalidConfiguration;
  int grid = (items + kBlock - 1) / kBlock;
  if (grid > per_sm * nsm)
    grid = per_sm * nsm;
  cudaError_t e = cudaMemsetAsync(a.bar, 0, 2 * sizeof(unsigned), s);
  if (e != cudaSuccess)
    return e;
  k<<<grid, kBlock, 0, s>>>(a, tb, ft);
  return cudaGetLastError();
}

template <int PHYS, int SCHEME, int NDOF, int NQ, int NFL>
cudaError_t launch_batch_one(const HostCellGroup &g, const DcCellArgs &a, int grid, int tile,
                             cudaStream_t s)
{
  Tables<float, 2, NDOF, NQ, NFL, 3> tb;
  fill_tables(tb, g.w, g.V, g.dV, g.dVgeo, g.dVf, g.Vsf);
  auto k = cells_scalar2d_dc_batch<PHYS, SCHEME, NDOF, NQ, NFL, 3>;
  // a persistent grid only balances if all its CTAs are resident at once: cap it at the
  // occupancy of this kernel and tile
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, tile, 0);
  const int cap = (per_sm < 1 ? 1 : per_sm) * nsm;
  k<<<grid < cap ? grid : cap, tile, 0, s>>>(a, tb);
  return cudaGetLastError();
}

template <int PHYS, int SCHEME, int NDOF, int NQ, int NFL>
cudaError_t launch_one(const HostCellGroup &g, const DcCellArgs &a, cudaStream_t s)
{
  Tables<float, 2, NDOF, NQ, NFL, 3> tb;
  fill_tables(tb, g.w, g.V, g.dV, g.dVgeo, g.dVf, g.Vsf);
  const int grid = (a.ncells + kBlock - 1) / kBlock;
  return launch_kernel(cells_scalar2d_dc<PHYS, SCHEME, NDOF, NQ, NFL, 3>, dim3(grid),
                       dim3(kBlock), 0, s, a.pdl != 0, a, tb);
}

// grid > 0: the batch form (persistent over the active tiles, `tile` cells per CTA)
template <int PHYS, int SCHEME>
cudaError_t dispatch_shape(const HostCellGroup &g, const DcCellArgs &a, int grid, int tile,
                           cudaStream_t s, bool *ok)
{
  const rds_cell_group &d = g.desc;
  *ok                     = true;
#define RDS_DC_SHAPE(ND, NQ_, NF)                                                                  \
  if (d.ndof == ND && d.nq == NQ_ && d.nfl == NF)                                                  \
    return grid > 0 ? launch_batch_one<PHYS, SCHEME, ND, NQ_, NF>(g, a, grid, tile, s)             \
                    : launch_one<PHYS, SCHEME, ND, NQ_, NF>(g, a, s);
  if (d.shape == RDS_TRIAG && d.ngeo == 3)
  {
    // (order, quadrature points, flux nodes): P1/P4-rule, P1/P5, P2/P4, P2/P5, P3/P6, P3/P8
    RDS_DC_SHAPE(3, 6, 6)
    RDS_DC_SHAPE(3, 7, 6)
    RDS_DC_SHAPE(6, 6, 10)
    RDS_DC_SHAPE(6, 7, 10)
    RDS_DC_SHAPE(10, 12, 15)
    RDS_DC_SHAPE(10, 16, 15)
  }
#undef RDS_DC_SHAPE
  *ok = false;
  return cudaSuccess;
}

} // namespace

bool dc_supported(const HostCellGroup &g)
{
  const rds_cell_group &d = g.desc;
  if ((g.physics != RDS_ADVECTION_CONST && g.physics != RDS_BURGERS2D) || d.shape != RDS_TRIAG ||
      d.ngeo != 3)
    return false;
  return (d.ndof == 3 && (d.nq == 6 || d.nq == 7) && d.nfl == 6) ||
         (d.ndof == 6 && (d.nq == 6 || d.nq == 7) && d.nfl == 10) ||
         (d.ndof == 10 && (d.nq == 12 || d.nq == 16) && d.nfl == 15);
}

cudaError_t launch_cells_scalar_dc(const HostCellGroup &g, const DcCellArgs &a, int grid,
                                   int tile, cudaStream_t s, const char **name, bool *ok)
{
  static const char *names[2][2][3] = {
      {{"cells_adv_lda_dc", "cells_adv_n_dc", "cells_adv_b_dc"},
       {"cells_burgers_lda_dc", "cells_burgers_n_dc", "cells_burgers_b_dc"}},
      {{"cells_adv_lda_dc_batch", "cells_adv_n_dc_batch", "cells_adv_b_dc_batch"},
       {"cells_burgers_lda_dc_batch", "cells_burgers_n_dc_batch", "cells_burgers_b_dc_batch"}}};
  *ok = false;
  if (!dc_supported(g) || g.scheme < 0 || g.scheme > 2 ||
      (grid > 0 && (tile <= 0 || tile > 128 || tile % 32 != 0)))
    return cudaSuccess;
  *name = names[grid > 0][g.physics == RDS_BURGERS2D][g.scheme];
#define RDS_DC_CASE(PH, SC)                                                                        \
  if (g.physics == PH && g.scheme == SC)                                                           \
    return dispatch_shape<PH, SC>(g, a, grid, tile, s, ok);
  RDS_DC_CASE(RDS_ADVECTION_CONST, RDS_PGLDA)
  RDS_DC_CASE(RDS_ADVECTION_CONST, RDS_PGN)
  RDS_DC_CASE(RDS_ADVECTION_CONST, RDS_PGB)
  RDS_DC_CASE(RDS_BURGERS2D, RDS_PGLDA)
  RDS_DC_CASE(RDS_BURGERS2D, RDS_PGN)
  RDS_DC_CASE(RDS_BURGERS2D, RDS_PGB)
#undef RDS_DC_CASE
  return cudaSuccess;
}

// The fused correction sweeps cover one straight-sided triangle group with the facet rule of
// its order's usual cell rule (P1: 2 dofs / 3 points, P2: 3 / 4, P3: 4 / 5, P3 with the order-6
// cell rule: 4 / 4) and up to
// kFuseMaxBC weak Dirichlet conditions.
namespace
{
bool fused_facets(int ndof, int nq, const rds_bc_group &d)
{
  const int nfdof = ndof == 3 ? 2 : ndof == 6 ? 3 : 4;
  const int nfq   = (ndof == 10 && nq == 12) ? 4 : nfdof + 1; // P3 / P6 rule: facets of order 7
  return d.nfgeo == 2 && d.nfdof == nfdof && d.nfq == nfq;
}
} // namespace

bool dc_fused_supported(const HostCellGroup &g, const HostBC *const *bcs, int nbc)
{
  if (!dc_supported(g) || g.scheme < 0 || g.scheme > 2 || nbc > kFuseMaxBC)
    return false;
  for (int k = 0; k < nbc; ++k)
    if (bcs[k]->desc.kind != RDS_BC_WEAK_DIRICHLET ||
        !fused_facets(g.desc.ndof, g.desc.nq, bcs[k]->desc))
      return false;
  return true;
}

cudaError_t launch_dc_fused(const HostCellGroup &g, const HostBC *const *bcs,
                            const DcFusedArgs &a, cudaStream_t s, const char **name, bool *ok)
{
  // [cluster form][physics][scheme]
  static const char *names[2][2][3] = {
      {{"dc_sweeps_fused_adv_lda", "dc_sweeps_fused_adv_n", "dc_sweeps_fused_adv_b"},
       {"dc_sweeps_fused_burgers_lda", "dc_sweeps_fused_burgers_n", "dc_sweeps_fused_burgers_b"}},
      {{"dc_sweeps_cluster_adv_lda", "dc_sweeps_cluster_adv_n", "dc_sweeps_cluster_adv_b"},
       {"dc_sweeps_cluster_burgers_lda", "dc_sweeps_cluster_burgers_n",
        "dc_sweeps_cluster_burgers_b"}}};
  *ok = false;
  if (!dc_fused_supported(g, bcs, a.nbc))
    return cudaSuccess;
  const rds_cell_group &d = g.desc;
  *ok                     = true;
  bool cl                 = false;
  const int ip = g.physics == RDS_BURGERS2D ? 1 : 0, is = g.scheme;
  *name                   = names[0][ip][is];
  // the launch name tells the two forms apart
  auto named = [&](cudaError_t e) {
    *name = names[cl ? 1 : 0][ip][is];
    return e;
  };
#define RDS_FUSED(PH, SC)                                                                          \
  if (g.physics == PH && g.scheme == SC)                                                           \
  {                                                                                                \
    if (d.ndof == 3 && d.nq == 6)                                                                  \
      return named(launch_fused_one<PH, SC, 3, 6, 6, 2, 3>(g, bcs, a, s, &cl));                    \
    if (d.ndof == 3 && d.nq == 7)                                                                  \
      return named(launch_fused_one<PH, SC, 3, 7, 6, 2, 3>(g, bcs, a, s, &cl));                    \
    if (d.ndof == 6 && d.nq == 6)                                                                  \
      return named(launch_fused_one<PH, SC, 6, 6, 10, 3, 4>(g, bcs, a, s, &cl));                   \
    if (d.ndof == 6 && d.nq == 7)                                                                  \
      return named(launch_fused_one<PH, SC, 6, 7, 10, 3, 4>(g, bcs, a, s, &cl));                   \
    if (d.ndof == 10 && d.nq == 16)                                                                \
      return named(launch_fused_one<PH, SC, 10, 16, 15, 4, 5>(g, bcs, a, s, &cl));                 \
    if (d.ndof == 10 && d.nq == 12)                                                                \
      return named(launch_fused_one<PH, SC, 10, 12, 15, 4, 4>(g, bcs, a, s, &cl));                 \
  }
  RDS_FUSED(RDS_ADVECTION_CONST, RDS_PGLDA)
  RDS_FUSED(RDS_ADVECTION_CONST, RDS_PGN)
  RDS_FUSED(RDS_ADVECTION_CONST, RDS_PGB)
  RDS_FUSED(RDS_BURGERS2D, RDS_PGLDA)
  RDS_FUSED(RDS_BURGERS2D, RDS_PGN)
  RDS_FUSED(RDS_BURGERS2D, RDS_PGB)
#undef RDS_FUSED
  *ok = false;
  return cudaSuccess;
}

} // namespace rds
