// Node-centred kernels: the deterministic gather that replaces the reference's scatter, the
// local time step and explicit update, the residual norm, and the dual volumes.
//
// The reference accumulates, with one thread, node_res[v] += (1/V_v) elem_res[n] over the
// active cells in ascending order and then over the weak-BC facets in BC order
// (src/solver/rdm/assembly/PGRDMExplicitCellWorker.hpp:549-567, bc/WeakBC.hpp:315-352), and the
// nodal wave speed likewise (src/solver/rdm/RDTimeUpdate.cpp:64-67). Here every node owns the
// list of its contribution slots in exactly that order (CSR built at set-up), so one thread per
// node reproduces the same sequence of IEEE roundings: no atomics, bit-identical across runs.
// Multiplies and adds are issued as separate round-to-nearest operations (no fused
// multiply-add) so the sums match the reference's x86-64 arithmetic.

#include "rds_internal.h"

namespace rds
{

namespace
{

// Deterministic block sum: fixed shuffle tree inside warps, warp results added in order.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *smem)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0)
    smem[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
  {
    for (int w = 0; w < NT / 32; ++w)
      s += smem[w];
  }
  return s; // valid in thread 0
}

__device__ void reduce_final(const double *part, int nblocks, int neq, int nnodes, double *norm,
                             double *norm0, double *hist, int *iter, int max_iter, double drop,
                             int *stop, unsigned *status, double *smem, double *nv);

template <int NEQ, bool DT, bool UPDATE, bool NORM, bool FINAL>
__global__ void __launch_bounds__(kGBlock) gather_nodes(const GatherArgs a)
{
  __shared__ double smem[kGBlock / 32];
  if (*a.stop)
    return;
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  double sq[NEQ];
#pragma unroll
  for (int e = 0; e < NEQ; ++e)
    sq[e] = 0.0;
  if (v < a.nnodes)
  {
    double acc[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
      acc[e] = 0.0;
    double ws     = 0.0;
    const double iv = a.inv_vol[v];
    const int i0 = a.row[v], i1 = a.row[v + 1];
    for (int i = i0; i < i1; ++i)
    {
      const long long s = __ldg(a.ent_slot + i);
      const int w       = __ldg(a.ent_ws + i);
#pragma unroll
      for (int e = 0; e < NEQ; ++e)
        acc[e] = __dadd_rn(acc[e], __dmul_rn(iv, __ldcs(a.contrib + e * a.S + s)));
      ws = __dadd_rn(ws, __ldcs(a.wsc + w));
    }
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
      a.res[(size_t)e * a.nnodes + v] = acc[e];
    a.ws[v] = ws;
    if (DT)
    {
      const double dtv = __ddiv_rn(__dmul_rn(a.cfl, a.vol[v]), ws);
      a.dt[v]          = dtv;
#pragma unroll
      for (int e = 0; e < NEQ; ++e)
      {
        if (UPDATE)
        {
          double *pu = a.u + (size_t)e * a.nnodes + v;
          *pu        = __dsub_rn(*pu, __dmul_rn(dtv, acc[e]));
        }
        if (NORM)
        {
          const double r = __dmul_rn(acc[e], dtv);
          sq[e]          = __dmul_rn(r, r);
        }
      }
    }
  }
  if (NORM)
  {
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
    {
      const double s = block_sum<kGBlock>(sq[e], smem);
      if (threadIdx.x == 0)
        a.part[(size_t)blockIdx.x * NEQ + e] = s;
    }
    if (FINAL)
    {
      // last-block-done: the block that finishes last reduces all partials (fixed order), so
      // the norm needs no separate launch; no block ever waits for another
      __shared__ bool last;
      __shared__ double nv[kMaxNeq];
      if (threadIdx.x == 0)
      {
        __threadfence();
        const unsigned done = atomicAdd(a.counter, 1u);
        last                = (done == gridDim.x - 1);
      }
      __syncthreads();
      if (last)
      {
        __threadfence();
        reduce_final(a.part, gridDim.x, NEQ, a.nnodes, a.norm, a.norm0, a.hist, a.iter,
                     a.max_iter, a.drop, a.stop_w, a.status, smem, nv);
        if (threadIdx.x == 0)
          *a.counter = 0u;
      }
    }
  }
}

// Sum of (res * dt)^2 per block (compute_residual_norm outside the fused loop).
template <int NEQ>
__global__ void __launch_bounds__(kGBlock)
    norm_partials(int nnodes, const double *res, const double *dt, double *part)
{
  __shared__ double smem[kGBlock / 32];
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
  for (int e = 0; e < NEQ; ++e)
  {
    double sq = 0.0;
    if (v < nnodes)
    {
      const double r = __dmul_rn(res[(size_t)e * nnodes + v], dt[v]);
      sq             = __dmul_rn(r, r);
    }
    const double s = block_sum<kGBlock>(sq, smem);
    if (threadIdx.x == 0)
      part[(size_t)blockIdx.x * NEQ + e] = s;
  }
}

// Final reduction of the block partials in a fixed order, norm = sqrt(sum / N), the
// iteration counter, the history and the device-side residual-drop / finiteness test.
// Executed by one whole block (norm_final, or the last block of a fused gather).
__device__ void reduce_final(const double *part, int nblocks, int neq, int nnodes, double *norm,
                             double *norm0, double *hist, int *iter, int max_iter, double drop,
                             int *stop, unsigned *status, double *smem, double *nv)
{
  for (int e = 0; e < neq; ++e)
  {
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
      s += __ldcg(part + (size_t)b * neq + e);
    s = block_sum<kGBlock>(s, smem);
    if (threadIdx.x == 0)
      nv[e] = sqrt(s / nnodes);
  }
  if (threadIdx.x != 0)
    return;
  if (iter == nullptr)
  {
    for (int e = 0; e < neq; ++e)
      norm[e] = nv[e];
    return;
  }
  const int it = *iter;
  double rel   = 0.0;
  bool finite  = true;
  for (int e = 0; e < neq; ++e)
  {
    const double n = nv[e];
    norm[e]        = n;
    if (it == 0)
      norm0[e] = n;
    if (it < max_iter)
      hist[(size_t)it * neq + e] = n;
    if (!isfinite(n))
      finite = false;
    const double n0 = (it == 0) ? n : norm0[e];
    const double r  = n0 > 0.0 ? n / n0 : 0.0;
    rel             = r > rel ? r : rel;
  }
  *iter = it + 1;
  if (!finite)
  {
    atomicOr(status, kFlagNonFinite);
    *stop = 1;
  }
  else if ((drop > 0.0 && rel <= drop) || it + 1 >= max_iter)
  {
    *stop = 1;
  }
}

__global__ void __launch_bounds__(kGBlock)
    norm_final(const double *part, int nblocks, int neq, int nnodes, double *norm, double *norm0,
               double *hist, int *iter, int max_iter, double drop, int *stop, unsigned *status)
{
  __shared__ double smem[kGBlock / 32];
  __shared__ double nv[kMaxNeq];
  if (stop != nullptr && *stop)
    return;
  reduce_final(part, nblocks, neq, nnodes, norm, norm0, hist, iter, max_iter, drop, stop, status,
               smem, nv);
}

__global__ void update_kernel(int n, const double *dt, const double *res, double *u, int neq)
{
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n)
    return;
  const double d = dt[v];
  for (int e = 0; e < neq; ++e)
  {
    double *pu = u + (size_t)e * n + v;
    *pu        = __dsub_rn(*pu, __dmul_rn(d, res[(size_t)e * n + v]));
  }
}

// Cell volume sum_q w_q detJ_q (set-up only; tables read from global memory).
__global__ void cell_volume_kernel(int ncells, int dim, int nq, int ngeo,
                                   const int32_t *geo_conn, const double *X, int ngeo_nodes,
                                   const double *w, const double *dVgeo, double *cvol)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells)
    return;
  double Xc[32][3];
  for (int g = 0; g < ngeo; ++g)
  {
    const int v = geo_conn[(size_t)g * ncells + c];
    for (int d = 0; d < dim; ++d)
      Xc[g][d] = X[(size_t)d * ngeo_nodes + v];
  }
  double vol = 0.0;
  for (int q = 0; q < nq; ++q)
  {
    double J[3][3];
    for (int xi = 0; xi < dim; ++xi)
      for (int x = 0; x < dim; ++x)
      {
        const double *row = dVgeo + ((size_t)xi * nq + q) * ngeo;
        double s          = row[0] * Xc[0][x];
        for (int g = 1; g < ngeo; ++g)
          s = s + row[g] * Xc[g][x];
        J[xi][x] = s;
      }
    double det;
    if (dim == 2)
      det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    else
      det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
            J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
            J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    vol += w[q] * det;
  }
  cvol[c] = vol;
}

__global__ void dual_volume_kernel(int nnodes, const int32_t *row, const int32_t *ent_ws,
                                   const double *cvol, double *vol, double *inv_vol)
{
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nnodes)
    return;
  double s = 0.0;
  for (int i = row[v]; i < row[v + 1]; ++i)
    s = __dadd_rn(s, cvol[ent_ws[i]]);
  vol[v]     = s;
  inv_vol[v] = 1. / s;
}

template <int NEQ>
cudaError_t launch_gather_neq(const GatherArgs &a, int mode, int nblocks, cudaStream_t s)
{
  switch (mode)
  {
  case 0:
    gather_nodes<NEQ, false, false, false, false><<<nblocks, kGBlock, 0, s>>>(a);
    break;
  case 1:
    gather_nodes<NEQ, true, false, false, false><<<nblocks, kGBlock, 0, s>>>(a);
    break;
  case 7:
    gather_nodes<NEQ, true, true, true, false><<<nblocks, kGBlock, 0, s>>>(a);
    break;
  case 15:
    gather_nodes<NEQ, true, true, true, true><<<nblocks, kGBlock, 0, s>>>(a);
    break;
  default:
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

} // namespace

cudaError_t launch_gather(const GatherArgs &a, int mode, int nblocks, cudaStream_t s,
                          const char **name)
{
  *name = (mode == 15) ? "gather_update_norm_final" : (mode == 7) ? "gather_update_norm"
                                                                   : "gather_nodes";
  switch (a.neq)
  {
  case 1:
    return launch_gather_neq<1>(a, mode, nblocks, s);
  case 4:
    return launch_gather_neq<4>(a, mode, nblocks, s);
  case 5:
    return launch_gather_neq<5>(a, mode, nblocks, s);
  default:
    return cudaErrorInvalidValue;
  }
}

cudaError_t launch_norm_partials(int nnodes, int neq, const double *res, const double *dt,
                                 double *part, int nblocks, cudaStream_t s)
{
  switch (neq)
  {
  case 1:
    norm_partials<1><<<nblocks, kGBlock, 0, s>>>(nnodes, res, dt, part);
    break;
  case 4:
    norm_partials<4><<<nblocks, kGBlock, 0, s>>>(nnodes, res, dt, part);
    break;
  case 5:
    norm_partials<5><<<nblocks, kGBlock, 0, s>>>(nnodes, res, dt, part);
    break;
  default:
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_norm_final(const double *part, int nblocks, int neq, int nnodes,
                              double *norm, double *norm0, double *hist, int *iter,
                              int max_hist, double drop, int *stop, unsigned *status,
                              cudaStream_t s, const char **name)
{
  *name = "norm_final";
  norm_final<<<1, kGBlock, 0, s>>>(part, nblocks, neq, nnodes, norm, norm0, hist, iter, max_hist,
                                   drop, stop, status);
  return cudaGetLastError();
}

cudaError_t launch_update(int nnodes, int neq, const double *dt, const double *res, double *u,
                          cudaStream_t s, const char **name)
{
  *name = "update";
  update_kernel<<<(nnodes + kGBlock - 1) / kGBlock, kGBlock, 0, s>>>(nnodes, dt, res, u, neq);
  return cudaGetLastError();
}

cudaError_t launch_cell_volume_raw(int ncells, int dim, int nq, int ngeo, const int32_t *geo_conn,
                                   const double *X, int ngeo_nodes, const double *w,
                                   const double *dVgeo, double *cvol, cudaStream_t s)
{
  cell_volume_kernel<<<(ncells + kBlock - 1) / kBlock, kBlock, 0, s>>>(
      ncells, dim, nq, ngeo, geo_conn, X, ngeo_nodes, w, dVgeo, cvol);
  return cudaGetLastError();
}

cudaError_t launch_dual_volume(int nnodes, const int32_t *row, const int32_t *ent_ws,
                               const double *cvol, double *vol, double *inv_vol, cudaStream_t s)
{
  dual_volume_kernel<<<(nnodes + kGBlock - 1) / kGBlock, kGBlock, 0, s>>>(nnodes, row, ent_ws,
                                                                          cvol, vol, inv_vol);
  return cudaGetLastError();
}

} // namespace rds
