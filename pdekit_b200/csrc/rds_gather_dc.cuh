// The node update of a correction sweep of the defect-correction loop (mixed form, one
// equation), shared by the gather kernel (rds_gather.cu, mode 19) and the fused correction
// sweeps (rds_cells_scalar_dc.cu): u_v -= dt R64(u_r)_v + (dt / V)_v sum of the FP32 changes of
// the node's contributions, summed in FP64 in the node's entry order. COHERENT: the changes are
// read through L2 (ld.global.cg), as a kernel must that reads values other blocks of the same
// launch have written.
#pragma once

#include "rds_internal.h"

namespace rds
{

namespace
{

template <bool COHERENT>
__device__ __forceinline__ float dc_load_change(const float *p)
{
  if constexpr (COHERENT)
    return __ldcg(p);
  else
    return __ldcs(p);
}

template <bool COHERENT>
__device__ __forceinline__ void dc_correction_node(const GatherArgs &a, const int v)
{
  const int i0 = a.row[v], i1 = a.row[v + 1];
  double sum   = 0.0;
  int i        = i0;
  constexpr int B = 4;
  for (; i + B <= i1; i += B)
  {
    float c[B];
#pragma unroll
    for (int k = 0; k < B; ++k)
      c[k] = dc_load_change<COHERENT>(a.c32 + __ldg(a.ent_slot + i + k));
#pragma unroll
    for (int k = 0; k < B; ++k)
      sum += double(c[k]);
  }
  for (; i < i1; ++i)
    sum += double(dc_load_change<COHERENT>(a.c32 + __ldg(a.ent_slot + i)));
  double *pu = a.u + v;
  *pu        = *pu - (a.dres[v] + double(a.dtv[v]) * sum);
}

// A node's correction-sweep data that stay the same within a cycle (its first kNodeCache entry
// slots, dt R64(u_r), dt / V) and its own state, for a thread that updates the same node every
// sweep of a launch (the fused sweeps): the node's value stays in a register between sweeps,
// since no other thread writes it. dc_node_sweep is dc_correction_node<true> on these.
constexpr int kNodeCache = 8;
struct DcNodeState
{
  int i0, i1;
  int slot[kNodeCache];
  double dres, u;
  float dtv;
};

__device__ __forceinline__ void dc_node_state(const GatherArgs &a, const int v, DcNodeState &ns)
{
  ns.i0 = a.row[v];
  ns.i1 = a.row[v + 1];
#pragma unroll
  for (int k = 0; k < kNodeCache; ++k)
    ns.slot[k] = ns.i0 + k < ns.i1 ? __ldg(a.ent_slot + ns.i0 + k) : 0;
  ns.dres = a.dres[v];
  ns.dtv  = a.dtv[v];
  ns.u    = __ldcg(a.u + v);
}

__device__ __forceinline__ void dc_node_sweep(const GatherArgs &a, const int v, DcNodeState &ns)
{
  float c[kNodeCache];
#pragma unroll
  for (int k = 0; k < kNodeCache; ++k)
    c[k] = ns.i0 + k < ns.i1 ? __ldcg(a.c32 + ns.slot[k]) : 0.f;
  double sum = 0.0;
#pragma unroll
  for (int k = 0; k < kNodeCache; ++k)
    if (ns.i0 + k < ns.i1)
      sum += double(c[k]);
  for (int i = ns.i0 + kNodeCache; i < ns.i1; ++i)
    sum += double(__ldcg(a.c32 + __ldg(a.ent_slot + i)));
  ns.u   = ns.u - (ns.dres + double(ns.dtv) * sum);
  a.u[v] = ns.u;
}

} // namespace

} // namespace rds
