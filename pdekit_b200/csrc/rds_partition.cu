// Kernels of the partitioned single-mesh form: one context per rank holds a part of the cells
// (and the nodes they touch); the ranks' partial nodal sums of residual and wave speed at the
// nodes they share are added through an exchange buffer, then every rank finishes the
// iteration on its nodes (src/solver/rdm/PGRDMethodExplicit.hpp:417-514 with the nodal sums of
// PGRDMExplicitCellWorker.hpp:549-567 split over the ranks).
//
//   pack     buf[slot][0..neq-1] = res[.][v], buf[slot][neq] = ws[v] for the shared nodes v
//            (the buffer is zeroed first, so a sum over the ranks' buffers is the full sum)
//   unpack   res[.][v], ws[v] = buf[slot] (after the sum over the ranks)
//   combine  a Runge-Kutta stage of nodes whose sums came through the exchange (partitioned
//            RK3TVD), with the arithmetic of the gather's stage branch
//   finish   dt = CFL V / ws, u -= dt res, and per block the sum over the nodes this rank owns
//            of (res dt)^2 (for a node range, after the block sums of the other nodes that
//            rds_gather_finish wrote); the block that finishes last adds the block sums in a
//            fixed order.

#include <algorithm>

#include "rds_internal.h"

namespace rds
{

namespace
{

__global__ void __launch_bounds__(kGBlock)
    pack_interface(int n, int neq, int nnodes, const int32_t *__restrict__ nodes,
                   const int32_t *__restrict__ slots, const double *__restrict__ res,
                   const double *__restrict__ ws, double *__restrict__ buf)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const int v = nodes[i];
  double *b   = buf + (size_t)slots[i] * (neq + 1);
  for (int e = 0; e < neq; ++e)
    b[e] = res[(size_t)e * nnodes + v];
  b[neq] = ws[v];
}

__global__ void __launch_bounds__(kGBlock)
    unpack_interface(int n, int neq, int nnodes, const int32_t *__restrict__ nodes,
                     const int32_t *__restrict__ slots, const double *__restrict__ buf,
                     double *__restrict__ res, double *__restrict__ ws)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const int v     = nodes[i];
  const double *b = buf + (size_t)slots[i] * (neq + 1);
  for (int e = 0; e < neq; ++e)
    res[(size_t)e * nnodes + v] = b[e];
  ws[v] = b[neq];
}

// Sum over the block (the result is valid in thread 0); blockDim.x is a multiple of 32.
__device__ __forceinline__ double sum_over_block(double v, double *smem)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0)
    smem[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k)
      s += smem[k];
  return s;
}

__global__ void __launch_bounds__(kGBlock)
    finish_nodes(int v0, int v1, int nnodes, int neq, double cfl, int update,
                 const double *__restrict__ vol, const double *__restrict__ ws,
                 const double *__restrict__ res, double *__restrict__ dt, double *__restrict__ u,
                 const uint8_t *__restrict__ owned, double *__restrict__ part, int part_off,
                 unsigned *counter, double *__restrict__ sq_out)
{
  __shared__ double smem[kGBlock / 32];
  __shared__ bool last;
  const int v   = v0 + blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = v < v1;
  double dtv    = 0.0;
  if (in)
  {
    dtv   = __ddiv_rn(__dmul_rn(cfl, vol[v]), ws[v]);
    dt[v] = dtv;
  }
  for (int e = 0; e < neq; ++e)
  {
    double sq = 0.0;
    if (in)
    {
      const double r = res[(size_t)e * nnodes + v];
      if (owned[v])
      {
        const double rd = __dmul_rn(r, dtv);
        sq              = __dmul_rn(rd, rd);
      }
      if (update)
      {
        double *pu = u + (size_t)e * nnodes + v;
        *pu        = __dsub_rn(*pu, __dmul_rn(dtv, r));
      }
    }
    const double s = sum_over_block(sq, smem);
    if (threadIdx.x == 0)
      part[(size_t)(part_off + blockIdx.x) * neq + e] = s;
  }
  // last-block-done: the block that finishes last adds all block sums in a fixed order (those
  // of a preceding rds_gather_finish first); no block waits for another
  if (!sq_out)
    return;
  if (threadIdx.x == 0)
  {
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last)
    return;
  __threadfence();
  const int nb = part_off + (int)gridDim.x;
  for (int e = 0; e < neq; ++e)
  {
    double t = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
      t += part[(size_t)b * neq + e];
    t = sum_over_block(t, smem);
    if (threadIdx.x == 0)
      sq_out[e] = t;
  }
  if (threadIdx.x == 0)
    *counter = 0u;
}


// Runge-Kutta stage combination of nodes [v0, v1) from their summed residual and wave speed
// (after the exchange): the arithmetic of gather_node's stage branch (rds_gather.cu).
__global__ void __launch_bounds__(kGBlock)
    rk_combine(int v0, int v1, int nnodes, int neq, int first, double cfl, double ca, double cb,
               double cc, const double *__restrict__ vol, const double *__restrict__ ws,
               const double *__restrict__ res, double *__restrict__ dt,
               const double *__restrict__ un, const double *__restrict__ us,
               double *__restrict__ out)
{
  const int v = v0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= v1)
    return;
  double d;
  if (first)
  {
    d     = __ddiv_rn(__dmul_rn(cfl, vol[v]), ws[v]);
    dt[v] = d;
  }
  else
    d = dt[v];
  for (int e = 0; e < neq; ++e)
  {
    const size_t k = (size_t)e * nnodes + v;
    const double r = __dmul_rn(d, res[k]);
    out[k]         = first ? __dsub_rn(un[k], r)
                           : __dsub_rn(__dadd_rn(__dmul_rn(ca, un[k]), __dmul_rn(cb, us[k])),
                                       __dmul_rn(cc, r));
  }
}

} // namespace

cudaError_t launch_pack_interface(int n, int neq, int nnodes, const int32_t *nodes,
                                  const int32_t *slots, const double *res, const double *ws,
                                  double *buf, size_t buf_len, cudaStream_t s)
{
  cudaError_t e = cudaMemsetAsync(buf, 0, buf_len * sizeof(double), s);
  if (e != cudaSuccess || n == 0)
    return e;
  pack_interface<<<(n + kGBlock - 1) / kGBlock, kGBlock, 0, s>>>(n, neq, nnodes, nodes, slots,
                                                                  res, ws, buf);
  return cudaGetLastError();
}

cudaError_t launch_unpack_interface(int n, int neq, int nnodes, const int32_t *nodes,
                                    const int32_t *slots, const double *buf, double *res,
                                    double *ws, cudaStream_t s)
{
  if (n == 0)
    return cudaSuccess;
  unpack_interface<<<(n + kGBlock - 1) / kGBlock, kGBlock, 0, s>>>(n, neq, nnodes, nodes, slots,
                                                                    buf, res, ws);
  return cudaGetLastError();
}

cudaError_t launch_finish(int v0, int v1, int nnodes, int neq, double cfl, int update,
                          const double *vol, const double *ws, const double *res, double *dt,
                          double *u, const uint8_t *owned, double *part, int part_off,
                          unsigned *counter, double *sq, cudaStream_t s)
{
  // at least one block: with an empty range it only adds the preceding block sums
  const int nb = std::max(1, (v1 - v0 + kGBlock - 1) / kGBlock);
  finish_nodes<<<nb, kGBlock, 0, s>>>(v0, v1, nnodes, neq, cfl, update, vol, ws, res, dt, u,
                                      owned, part, part_off, counter, sq);
  return cudaGetLastError();
}

cudaError_t launch_rk_combine(int v0, int v1, int nnodes, int neq, int first, double cfl, double ca,
                              double cb, double cc, const double *vol, const double *ws,
                              const double *res, double *dt, const double *un, const double *us,
                              double *out, cudaStream_t s)
{
  if (v1 <= v0)
    return cudaSuccess;
  rk_combine<<<(v1 - v0 + kGBlock - 1) / kGBlock, kGBlock, 0, s>>>(v0, v1, nnodes, neq, first, cfl,
                                                                  ca, cb, cc, vol, ws, res, dt, un,
                                                                  us, out);
  return cudaGetLastError();
}

} // namespace rds
