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

#include "rds_gather_dc.cuh"
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
                             int *stop, unsigned *status, double *smem, double *nv,
                             StallRec *stall = nullptr, const LoopParams *loop = nullptr);

// Progress test of the FP32 phase of the mixed loop: a halving of the best drop so far is
// progress; once the drop has halved at least once, the phase has stalled (the problem's FP32
// round-off floor) when no halving came for max(stall_min, stall_mult x the last interval
// between halvings) iterations. it = 0 starts the record.
__device__ __forceinline__ bool fp32_stalled(double rel, int it, StallRec *r, const LoopParams &L)
{
  if (it == 0)
  {
    r->best    = rel;
    r->best_it = 0;
    r->gap     = 0;
    return false;
  }
  if (rel <= 0.5 * r->best)
  {
    r->gap     = it - r->best_it;
    r->best    = rel;
    r->best_it = it;
    return false;
  }
  if (r->gap == 0)
    return false; // initial transient: no rate known yet
  const double window = fmax(double(L.stall_min), L.stall_mult * double(r->gap));
  return double(it - r->best_it) > window;
}

// DC (defect-correction loop, one equation): 1 = exact sweep that also keeps its update
// dt res, dt / V and the state the sweep starts from; 2 = correction sweep: every slot holds
// the FP32 change of its contribution since the exact sweep, u -= dt res + (dt / V) sum
// (nothing else is written).
template <int NEQ, bool DT, bool UPDATE, bool NORM, bool RK = false, int DC = 0>
__device__ __forceinline__ void gather_node(const GatherArgs &a, const int v, const double cfl,
                                            double *sq)
{
  static_assert(DC == 0 || NEQ == 1, "the defect-correction gather is scalar");
  if (DC == 2)
  {
    dc_correction_node<false>(a, v);
    return;
  }
  double acc[NEQ];
#pragma unroll
  for (int e = 0; e < NEQ; ++e)
    acc[e] = 0.0;
  double ws       = 0.0;
  // 1 / V formed here (correctly rounded, the same value as the stored inverse) instead of
  // loaded: one 8-byte read less per node; V itself is read once for both uses
  const double vv = a.vol[v];
  const double iv = __drcp_rn(vv);
  const int i0 = a.row[v], i1 = a.row[v + 1];
  int i        = i0;
  // four entries at a time: all their loads are issued before the ordered sums consume them
  // (same summation order as the one-by-one loop below)
  constexpr int B = 4;
  for (; i + B <= i1; i += B)
  {
    long long s[B];
    int w[B];
#pragma unroll
    for (int k = 0; k < B; ++k)
    {
      s[k] = __ldg(a.ent_slot + i + k);
      w[k] = __ldg(a.ent_ws + i + k);
    }
    double cv[B][NEQ], wv[B];
#pragma unroll
    for (int k = 0; k < B; ++k)
    {
#pragma unroll
      for (int e = 0; e < NEQ; ++e)
        cv[k][e] = __ldcs(a.contrib + e * a.S + s[k]);
      wv[k] = __ldcs(a.wsc + w[k]);
    }
#pragma unroll
    for (int k = 0; k < B; ++k)
    {
#pragma unroll
      for (int e = 0; e < NEQ; ++e)
        acc[e] = __dadd_rn(acc[e], __dmul_rn(iv, cv[k][e]));
      ws = __dadd_rn(ws, wv[k]);
    }
  }
  for (; i < i1; ++i)
  {
    const long long s = __ldg(a.ent_slot + i);
    const int w       = __ldg(a.ent_ws + i);
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
      acc[e] = __dadd_rn(acc[e], __dmul_rn(iv, __ldcs(a.contrib + e * a.S + s)));
    ws = __dadd_rn(ws, __ldcs(a.wsc + w));
  }
  if (DC == 1)
    a.ur[v] = a.u[v];
#pragma unroll
  for (int e = 0; e < NEQ; ++e)
    a.res[(size_t)e * a.nnodes + v] = acc[e];
  a.ws[v] = ws;
  if (RK)
  {
    // Runge-Kutta stage combination of solver/time/ExplicitTimeStepper.cpp:66-100, evaluated
    // left to right without contraction like the reference's expression templates:
    //   first stage   u_1 = u_n - dt * r
    //   later stages  u_k = (ca * u_n + cb * u_s) - cc * (dt * r)
    // dt is this stage's (first) or the first stage's (later stages; assemble_rhs keeps it)
    const double d = DT ? __ddiv_rn(__dmul_rn(cfl, vv), ws) : a.dt[v];
    if (DT)
      a.dt[v] = d;
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
    {
      const size_t k   = (size_t)e * a.nnodes + v;
      const double r   = __dmul_rn(d, acc[e]);
      const double un  = a.rk_un[k];
      a.rk_out[k]      = a.rk_first ? __dsub_rn(un, r)
                                    : __dsub_rn(__dadd_rn(__dmul_rn(a.rk_ca, un),
                                                          __dmul_rn(a.rk_cb, a.rk_us[k])),
                                                __dmul_rn(a.rk_cc, r));
    }
    return;
  }
  if (DT)
  {
    const double dtv = __ddiv_rn(__dmul_rn(cfl, vv), ws);
    a.dt[v]          = dtv;
    if (DC == 1)
    {
      a.dres[v] = __dmul_rn(dtv, acc[0]); // this sweep's update, u_new = u - dres
      a.dtv[v]  = float(dtv * iv);
    }
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

template <int NEQ, bool DT, bool UPDATE, bool NORM, bool FINAL, bool RK = false, int DC = 0>
__global__ void __launch_bounds__(kGBlock) gather_nodes(const __grid_constant__ GatherArgs a)
{
  __shared__ double smem[kGBlock / 32];
  pdl_wait_and_release();
  if (*a.stop)
    return;
  const int v = a.vbeg + blockIdx.x * blockDim.x + threadIdx.x;
  double sq[NEQ];
#pragma unroll
  for (int e = 0; e < NEQ; ++e)
    sq[e] = 0.0;
  if (v < (a.vend > 0 ? a.vend : a.nnodes))
    gather_node<NEQ, DT, UPDATE, NORM, RK, DC>(a, v, a.loop ? a.loop->cfl : a.cfl, sq);
  if (NORM)
  {
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
    {
      const double s = block_sum<kGBlock>(sq[e], smem);
      if (threadIdx.x == 0)
        a.part[(size_t)(a.part_off + blockIdx.x) * NEQ + e] = s;
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
        if (a.sq_out)
        {
          // partitioned form: the plain sum of the block sums (fixed order) for the caller
#pragma unroll
          for (int e = 0; e < NEQ; ++e)
          {
            double t = 0.0;
            for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
              t += a.part[(size_t)(a.part_off + b) * NEQ + e];
            t = block_sum<kGBlock>(t, smem);
            if (threadIdx.x == 0)
              a.sq_out[e] = t;
          }
        }
        else
        {
          const int max_iter = a.loop ? a.loop->max_iter : a.max_iter;
          const double drop  = a.loop ? a.loop->drop : a.drop;
          reduce_final(a.part, gridDim.x, NEQ, a.nnodes, a.norm, a.norm0, a.hist, a.iter,
                       max_iter, drop, a.stop_w, a.status, smem, nv, a.stall, a.loop);
        }
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
                             int *stop, unsigned *status, double *smem, double *nv,
                             StallRec *stall, const LoopParams *loop)
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
  // defect-correction loop: this exact sweep is followed by m - 1 correction sweeps, which
  // count as iterations and repeat this norm in the history; the loop stops only here, so it
  // also stops when the next exact sweep would fall past max_iter
  const int m = (loop && loop->dc_m > 1) ? loop->dc_m : 1;
  *iter       = it + 1;
  if (!finite)
  {
    atomicOr(status, kFlagNonFinite);
    *stop = 1;
  }
  else if ((drop > 0.0 && rel <= drop) || it + m >= max_iter)
  {
    *stop = 1;
  }
  else if (loop && loop->stall && fp32_stalled(rel, it, stall, *loop))
  {
    *stop = 1;
  }
  else if (m > 1)
  {
    for (int j = 1; j < m; ++j)
      for (int e = 0; e < neq; ++e)
        hist[(size_t)(it + j) * neq + e] = nv[e];
    *iter = it + m;
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

// The host's node-major state [n][neq] and the device's equation-major one [neq][n]: one thread
// per element, the node-major side read or written contiguously (to_soa: aos -> soa).
__global__ void transpose_state(long long total, int n, int neq, const double *__restrict__ src,
                                double *__restrict__ dst, int to_soa)
{
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total)
    return;
  const long long v = i / neq;
  const int e       = (int)(i - v * neq);
  if (to_soa)
    dst[(size_t)e * n + v] = src[i];
  else
    dst[i] = src[(size_t)e * n + v];
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

// ---- batched independent problems ---------------------------------------------------------

// Largest p with prefix[p] <= t, for prefix[0] = 0 <= t < prefix[np] (non-decreasing prefix).
__device__ __forceinline__ int find_segment(const int32_t *prefix, int np, int t)
{
  int lo = 0, hi = np;
  while (hi - lo > 1)
  {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= t)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// Norm and stop test of problem p (whole block; the result is written by thread 0): the same
// fixed-order reduction of the problem's node-block partials as the single-problem loop, then
// the phase change FP32 -> FP64 at max(drop, sw), done at drop, or at the iteration cap.
template <int NEQ>
__device__ void problem_final(const GatherArgs &a, const BatchArgs &b, const int p,
                              const int nblk, double *smem, double *nv)
{
  const int base = b.nb_base[p];
  const int nn   = b.node_off[p + 1] - b.node_off[p];
  for (int e = 0; e < NEQ; ++e)
  {
    double s = 0.0;
    for (int k = threadIdx.x; k < nblk; k += blockDim.x)
      s += __ldcg(a.part + (size_t)(base + k) * NEQ + e);
    s = block_sum<kGBlock>(s, smem);
    if (threadIdx.x == 0)
      nv[e] = sqrt(s / nn);
  }
  if (threadIdx.x != 0)
    return;
  const int it = b.iter[p];
  const int ph = b.phase[p];
  double rel   = 0.0;
  bool finite  = true;
  for (int e = 0; e < NEQ; ++e)
  {
    const double n = nv[e];
    b.norm[(size_t)p * NEQ + e] = n;
    if (it == 0)
      b.norm0[(size_t)p * NEQ + e] = n;
    if (!isfinite(n))
      finite = false;
    const double n0 = (it == 0) ? n : b.norm0[(size_t)p * NEQ + e];
    const double r  = n0 > 0.0 ? n / n0 : 0.0;
    rel             = r > rel ? r : rel;
  }
  const LoopParams &L    = *b.loop;
  // defect-correction loop: m - 1 correction sweeps follow this exact sweep and count as
  // iterations; the problem stops here when the next exact sweep would fall past max_iter
  const int m            = L.dc_m > 1 ? L.dc_m : 1;
  int nph                = ph;
  const double drop1     = L.drop > L.sw ? L.drop : L.sw;
  if (!finite)
  {
    atomicOr(b.pstatus + p, kFlagNonFinite);
    atomicOr(a.status, kFlagNonFinite);
    nph = 2;
  }
  else if (ph == 0 && (rel <= drop1 || fp32_stalled(rel, it, b.stall + p, L)))
    nph = 1;
  else if (ph == 1 && L.drop > 0.0 && rel <= L.drop)
    nph = 2;
  if (nph != 2 && it + m >= L.max_iter)
    nph = 2;
  b.iter[p] = (nph == 2) ? it + 1 : it + m;
  if (nph != ph)
  {
    b.phase[p] = nph;
    *b.changed = 1;
  }
  b.pcount[p] = 0u;
}

// Persistent gather over the node blocks of the problems still iterating: each problem's nodes
// are split into blocks of kGBlock from its first node, exactly as a single-problem context
// splits them, and the block that completes a problem's iteration reduces its norm.
// DC: 0 plain; 1 exact sweep of the defect-correction loop (also keeps dres / dtv / ur);
// 2 correction sweep (FP32 changes of every slot, no norm or stop test).
// RKS: a Runge-Kutta stage instead (1 the first: residual, dt and u_1; 2 a later one), with each
// problem's CFL, no norm or stop test.
template <int NEQ, int DC = 0, int RKS = 0>
__global__ void __launch_bounds__(kGBlock)
    gather_batch(const __grid_constant__ GatherArgs a, const __grid_constant__ BatchArgs b)
{
  __shared__ double smem[kGBlock / 32];
  __shared__ double nv[kMaxNeq];
  __shared__ bool last;
  if (*a.stop)
    return;
  const int np    = b.nprob;
  const int total = b.nb_prefix[np];
  for (int t = blockIdx.x; t < total; t += gridDim.x)
  {
    const int p  = find_segment(b.nb_prefix, np, t);
    const int j  = t - b.nb_prefix[p];
    const int n0 = b.node_off[p], n1 = b.node_off[p + 1];
    const int v  = n0 + j * kGBlock + threadIdx.x;
    double sq[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
      sq[e] = 0.0;
    if (v < n1)
    {
      if constexpr (RKS != 0)
        gather_node<NEQ, RKS == 1, false, false, true, 0>(a, v, b.cfl[p], sq);
      else
        gather_node<NEQ, DC != 2, DC != 2, DC != 2, false, DC>(a, v, b.cfl[p], sq);
    }
    if (DC == 2 || RKS != 0)
      continue; // uniform over the block: no barrier is skipped by part of it
    const int slot = b.nb_base[p] + j;
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
    {
      const double s = block_sum<kGBlock>(sq[e], smem);
      if (threadIdx.x == 0)
        a.part[(size_t)slot * NEQ + e] = s;
    }
    const int nblk = (n1 - n0 + kGBlock - 1) / kGBlock;
    if (threadIdx.x == 0)
    {
      __threadfence();
      const unsigned done = atomicAdd(b.pcount + p, 1u);
      last                = (done == (unsigned)nblk - 1u);
    }
    __syncthreads();
    if (last)
    {
      __threadfence();
      problem_final<NEQ>(a, b, p, nblk, smem, nv);
    }
    __syncthreads();
  }
}

// Block-wide exclusive scan of one int per thread (blockDim.x a multiple of 32, <= 1024).
__device__ __forceinline__ int block_exclusive_scan(int x, int *sh, int *total)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int v = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1)
  {
    const int y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o)
      v += y;
  }
  __syncthreads();
  if (lane == 31)
    sh[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0)
  {
    int acc = 0;
    for (int w = 0; w < nw; ++w)
    {
      const int t = sh[w];
      sh[w]       = acc;
      acc += t;
    }
    sh[32] = acc;
  }
  __syncthreads();
  *total = sh[32];
  return sh[warp] + v - x;
}

// Exclusive prefix over p of cnt(p) into out[0..np], one block, chunked per thread.
template <typename F>
__device__ void prefix_over_problems(int np, F cnt, int32_t *out, int *sh)
{
  const int per = (np + blockDim.x - 1) / blockDim.x;
  const int p0  = min(np, (int)threadIdx.x * per), p1 = min(np, p0 + per);
  int local     = 0;
  for (int p = p0; p < p1; ++p)
    local += cnt(p);
  int total;
  int off = block_exclusive_scan(local, sh, &total);
  for (int p = p0; p < p1; ++p)
  {
    out[p] = off;
    off += cnt(p);
  }
  if (threadIdx.x == 0)
    out[np] = total;
}

// Active lists after a phase change: per cell group and phase the tiles of the problems in
// that phase, and the node blocks of the problems not done; raises the stop flag when every
// problem is done. Does nothing when no problem changed phase in the last iteration.
__global__ void __launch_bounds__(1024) batch_rebuild(const __grid_constant__ RebuildArgs r)
{
  __shared__ int sh[33];
  if (*r.stop || *r.changed == 0)
    return;
  const int np = r.nprob;
  for (int g = 0; g < r.ngroups; ++g)
    for (int ph = 0; ph < 2; ++ph)
    {
      const int tile    = r.tile[g * 2 + ph];
      const int32_t *cb = r.cbeg + (size_t)g * np, *ce = r.cend + (size_t)g * np;
      prefix_over_problems(
          np,
          [&](int p) { return r.phase[p] == ph ? (ce[p] - cb[p] + tile - 1) / tile : 0; },
          r.tile_prefix + ((size_t)g * 2 + ph) * (np + 1), sh);
    }
  prefix_over_problems(
      np,
      [&](int p) {
        return r.phase[p] < 2 ? (r.node_off[p + 1] - r.node_off[p] + kGBlock - 1) / kGBlock : 0;
      },
      r.nb_prefix, sh);
  __syncthreads();
  if (threadIdx.x == 0)
  {
    *r.changed = 0;
    if (r.nb_prefix[np] == 0)
      *r.stop = 1;
  }
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
    return launch_kernel(gather_nodes<NEQ, true, true, true, true>, dim3(nblocks), dim3(kGBlock),
                         0, s, a.pdl != 0, a);
  case 16:
    gather_nodes<NEQ, false, false, false, false, true><<<nblocks, kGBlock, 0, s>>>(a);
    break;
  case 17:
    gather_nodes<NEQ, true, false, false, false, true><<<nblocks, kGBlock, 0, s>>>(a);
    break;
  default:
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// defect-correction loop (one equation): 18 exact fused sweep keeping dres / dtv / ur, 19
// correction sweep
cudaError_t launch_gather_dc(const GatherArgs &a, int mode, int nblocks, cudaStream_t s)
{
  if (mode == 18)
    return launch_kernel(gather_nodes<1, true, true, true, true, false, 1>, dim3(nblocks),
                         dim3(kGBlock), 0, s, a.pdl != 0, a);
  if (mode == 19)
    return launch_kernel(gather_nodes<1, false, false, false, false, false, 2>, dim3(nblocks),
                         dim3(kGBlock), 0, s, a.pdl != 0, a);
  return cudaErrorInvalidValue;
}

} // namespace

cudaError_t launch_gather(const GatherArgs &a, int mode, int nblocks, cudaStream_t s,
                          const char **name)
{
  *name = (mode == 15)  ? "gather_update_norm_final"
          : (mode == 7) ? "gather_update_norm"
          : (mode == 18) ? "gather_dc_exact"
          : (mode == 19) ? "gather_dc_correction"
          : (mode >= 16) ? "gather_rk_stage"
                        : "gather_nodes";
  if (mode == 18 || mode == 19)
    return a.neq == 1 ? launch_gather_dc(a, mode, nblocks, s) : cudaErrorInvalidValue;
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

cudaError_t launch_transpose_state(int nnodes, int neq, const double *src, double *dst,
                                   bool to_soa, cudaStream_t s, const char **name)
{
  *name                 = to_soa ? "state_to_soa" : "state_to_aos";
  const long long total = (long long)nnodes * neq;
  transpose_state<<<(unsigned)((total + kGBlock - 1) / kGBlock), kGBlock, 0, s>>>(
      total, nnodes, neq, src, dst, to_soa ? 1 : 0);
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

cudaError_t launch_gather_batch(const GatherArgs &a, const BatchArgs &b, int grid, cudaStream_t s,
                                const char **name, int dc, int rk)
{
  if (rk == 1 || rk == 2)
  {
    *name = "gather_batch_rk_stage";
    switch (a.neq)
    {
    case 1:
      rk == 1 ? gather_batch<1, 0, 1><<<grid, kGBlock, 0, s>>>(a, b)
              : gather_batch<1, 0, 2><<<grid, kGBlock, 0, s>>>(a, b);
      break;
    case 4:
      rk == 1 ? gather_batch<4, 0, 1><<<grid, kGBlock, 0, s>>>(a, b)
              : gather_batch<4, 0, 2><<<grid, kGBlock, 0, s>>>(a, b);
      break;
    case 5:
      rk == 1 ? gather_batch<5, 0, 1><<<grid, kGBlock, 0, s>>>(a, b)
              : gather_batch<5, 0, 2><<<grid, kGBlock, 0, s>>>(a, b);
      break;
    default:
      return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
  }
  if (dc == 1 || dc == 2)
  {
    if (a.neq != 1)
      return cudaErrorInvalidValue;
    *name = dc == 1 ? "gather_batch_dc_exact" : "gather_batch_dc_correction";
    if (dc == 1)
      gather_batch<1, 1><<<grid, kGBlock, 0, s>>>(a, b);
    else
      gather_batch<1, 2><<<grid, kGBlock, 0, s>>>(a, b);
    return cudaGetLastError();
  }
  *name = "gather_batch";
  switch (a.neq)
  {
  case 1:
    gather_batch<1><<<grid, kGBlock, 0, s>>>(a, b);
    break;
  case 4:
    gather_batch<4><<<grid, kGBlock, 0, s>>>(a, b);
    break;
  case 5:
    gather_batch<5><<<grid, kGBlock, 0, s>>>(a, b);
    break;
  default:
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_batch_rebuild(const RebuildArgs &r, cudaStream_t s, const char **name)
{
  *name = "batch_rebuild";
  batch_rebuild<<<1, 1024, 0, s>>>(r);
  return cudaGetLastError();
}

} // namespace rds
