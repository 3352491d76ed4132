// Internal declarations shared by the host runtime (rds_api.cu) and the kernel files.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "rds_b200.h"

namespace rds
{

constexpr int kMaxNeq  = 5;
constexpr int kMaxDim  = 3;
constexpr int kBlock   = 128; // threads per block of the cell/facet kernels
constexpr int kGBlock  = 256; // threads per block of the node gather kernel

// Programmatic dependent launch (sm_90+): a kernel launched with launch_kernel(pdl = true) may
// start while the kernel before it on the stream finishes; it waits here, before touching
// anything that kernel wrote, and lets the kernel after it start early in turn. Both are no-ops
// for a kernel launched without the attribute.
#ifdef __CUDACC__
__device__ __forceinline__ void pdl_wait_and_release()
{
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}

// Launches kernel k, with the programmatic-dependent-launch attribute when pdl is set.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_kernel(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                 cudaStream_t s, bool pdl, Args &&...args)
{
  if (!pdl)
  {
    k<<<grid, block, smem, s>>>(std::forward<Args>(args)...);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg{};
  cfg.gridDim          = grid;
  cfg.blockDim         = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream           = s;
  cudaLaunchAttribute attr[1];
  attr[0].id                                         = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs                                          = attr;
  cfg.numAttrs                                       = 1;
  return cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}
#endif

// Device-side status word bits (ORed by kernels, read by the host).
enum : unsigned
{
  kFlagNonFinite   = 1u,
  kFlagNegPressure = 2u,
  kFlagTimeout     = 4u // a bounded device wait gave up
};

// Host copy of one element type's tables; passed to kernels by value through the parameter
// space (constant bank), see rds_tables.cuh.
struct HostCellGroup
{
  rds_cell_group desc{};
  std::vector<double> w, V, dV, dVgeo, dVf, Vsf;
  std::vector<double> wv, dVgeo_v; // dual-volume rule (empty: use w, dVgeo)
  int32_t *d_sol_conn = nullptr; // SoA [ndof][ncells]
  int32_t *d_geo_conn = nullptr; // SoA [ngeo][ncells]
  long long slot_base = 0;       // first contribution slot of this group
  long long ws_base   = 0;       // first wave-speed slot of this group
  bool affine         = false;   // simplex with straight edges: Jacobian constant per cell
  bool const_jac      = false;   // every cell's Jacobian constant (simplices, parallelograms)
  int physics         = 0;       // physics / scheme of this group's cells
  int scheme          = 0;
  // batched problems: cells of problem p are [cbeg[p], cend[p]) of this group
  std::vector<int32_t> pcells;   // [P+1] offsets (empty outside a batch)
  int32_t *d_cbeg = nullptr, *d_cend = nullptr;
  int tune_tile[2] = {128, 128}; // cells per CTA tile (phase 0 FP32, phase 1 FP64)
  int tune_grid[2] = {0, 0};     // persistent grid (CTAs), 0: 4 per SM
  float *d_tc      = nullptr;    // tensor-core tables of the FP32 kernel (rds_cells_scalar_tc.cu)
  double *d_lt64   = nullptr;    // lane-indexed tables of the Euler kernels (FP64, FP32)
  float *d_lt32    = nullptr;
};

struct HostBC
{
  rds_bc_group desc{};
  std::vector<double> fw, fV, fdVgeo;
  int32_t *d_sol_conn = nullptr; // SoA [nfdof][nfacets]
  int32_t *d_geo_conn = nullptr; // SoA [nfgeo][nfacets]
  double *d_gq        = nullptr; // [neq][nfq][nfacets]; farfield [neq]; strong [neq][nstrong]
  int nstrong         = 0;       // strong Dirichlet: distinct dofs (d_sol_conn holds them)
  long long slot_base = 0;
  long long ws_base   = 0;
  int physics         = 0;
};

// Loop parameters read by the device from memory, so a captured loop graph stays valid when
// they change between calls.
struct LoopParams
{
  double cfl;
  double drop;     // stop at max_eq norm/norm0 <= drop (0: never)
  double sw;       // batched mixed form: switch from FP32 to FP64 cells at this drop
  double stall_mult; // FP32 phase stalled: no halving of the drop for
  int stall_min;     //   max(stall_min, stall_mult x the last interval between halvings)
  int max_iter;
  int stall;       // nonzero: FP32 phase, also stop when progress stalls
  int dc_m;        // defect-correction loop: an exact FP64 sweep every dc_m sweeps (0, 1: off)
};

// Progress record of the FP32 phase of the mixed loop.
struct StallRec
{
  double best; // best drop (a halving of the previous best)
  int best_it; // iteration it was reached
  int gap;     // iterations between the last two halvings (0: no halving yet)
};

// Active-tile map of one cell group in a batch (persistent cell kernels): tile t of the
// active list belongs to the problem p with prefix[p] <= t < prefix[p+1], and covers cells
// cbeg[p] + (t - prefix[p]) * blockDim.x + [0, blockDim.x) clipped to cend[p].
struct BatchTileMap
{
  const int32_t *prefix; // [P+1], rebuilt on the device when a problem changes phase
  const int32_t *cbeg;   // [P]
  const int32_t *cend;   // [P]
  int nprob;
};

// Per-problem state of a batch (one context holding the disjoint union of the problems).
struct BatchArgs
{
  int nprob;
  const int32_t *node_off;  // [P+1] node range of each problem
  const int32_t *nb_base;   // [P] first norm-partial slot (node block) of each problem
  const int32_t *nb_prefix; // [P+1] active node blocks, exclusive prefix
  const double *cfl;        // [P]
  unsigned *pcount;         // [P] node blocks of the problem done in this iteration
  int32_t *phase;           // [P] 0: FP32 cells, 1: FP64 cells, 2: done
  int32_t *iter;            // [P] iterations done
  double *norm, *norm0;     // [P][neq]
  unsigned *pstatus;        // [P] status bits of each problem
  int32_t *changed;         // a problem changed phase in this iteration
  const LoopParams *loop;
  StallRec *stall;          // [P] FP32-phase progress records
};

// Rebuild of the active lists after a phase change (one block).
struct RebuildArgs
{
  int nprob;
  int ngroups;
  const int32_t *phase;     // [P]
  const int32_t *cbeg;      // [ngroups][P]
  const int32_t *cend;      // [ngroups][P]
  const int32_t *tile;      // [ngroups][2] cells per tile of each phase
  int32_t *tile_prefix;     // [ngroups][2][P+1]
  const int32_t *node_off;  // [P+1]
  int32_t *nb_prefix;       // [P+1]
  int32_t *changed;
  int *stop;
};

// Arguments common to every cell kernel.
struct CellArgs
{
  int ncells;
  int nnodes;
  const int32_t *__restrict__ sol_conn; // SoA [ndof][ncells]
  const int32_t *__restrict__ geo_conn; // SoA [ngeo][ncells]
  const double *__restrict__ X;         // geometry coords SoA [dim][ngeo_nodes]
  int ngeo_nodes;
  const double *__restrict__ u; // state SoA [neq][nnodes]
  double *__restrict__ contrib; // [neq][S], this group's slots start at slot_base
  long long S;                  // total contribution slots
  long long slot_base;
  double *__restrict__ wsc; // wave-speed contributions, this group at ws_base
  long long ws_base;
  double adv0, adv1, adv2, gamma;
  unsigned *status;
  const int *stop; // nonzero: skip the work (converged loop)
  BatchTileMap bt; // batch mode only
  double *theta;   // PGB: the cell's blending coefficient [ncells] when not null (Jacobians)
  const double *blend; // PGB: external nodal blending coefficient [nnodes] when not null
  int pdl;         // launch with programmatic dependent launch (loop graphs)
  const void *lt;  // Euler cells: lane-indexed tables in the kernel's precision (set at launch)
  int tc_test_wait; // tensor-core cells: tries of a wait nothing completes (timeout test; 0 none)
};

// FP32 correction sweep of the defect-correction loop (rds_cells_scalar_dc.cu): the change of
// the cell residual from u_r to u, written as FP32 values to the cell slots of c32.
struct DcCellArgs
{
  int ncells;
  const int32_t *__restrict__ sol_conn; // SoA [ndof][ncells]
  const int32_t *__restrict__ geo_conn; // SoA [ngeo][ncells]
  const double *__restrict__ X;
  int ngeo_nodes;
  const double *__restrict__ u;  // current state [nnodes]
  const double *__restrict__ ur; // reference state of the cycle [nnodes]
  float *__restrict__ c32;       // [slots]
  long long slot_base;
  const double *__restrict__ theta; // PGB: the cell's blending coefficient at u_r [ncells]
  double adv0, adv1;
  const int *stop;
  BatchTileMap bt; // batch form only
  int pdl;         // launch with programmatic dependent launch (loop graphs)
  const void *lt;  // Euler cells: lane-indexed tables in the kernel's precision (set at launch)
  int tc_test_wait; // tensor-core cells: tries of a wait nothing completes (timeout test; 0 none)
};

struct BCArgs
{
  int nfacets;
  const int32_t *__restrict__ sol_conn;
  const int32_t *__restrict__ geo_conn;
  const double *__restrict__ X;
  int ngeo_nodes;
  const double *__restrict__ u;
  int nnodes;
  const double *__restrict__ gq; // [neq][nfq][nfacets]
  const double *__restrict__ vol;
  double *__restrict__ contrib;
  long long S;
  long long slot_base;
  double *__restrict__ wsc;
  long long ws_base;
  double adv0, adv1, gamma;
  double relax;      // WeakWall: 1 for P1 facets, 1/(3p) otherwise
  double params[4];  // WeakSubInlet: T_tot, p_tot; WeakSubOutlet: p_out
  unsigned *status;
  const int *stop;
  double *u_strong; // strong Dirichlet: the state it overwrites (the same buffer as u)
  // correction sweep of the defect-correction loop (one equation): when set, the facet writes
  // the change of its contribution since the exact sweep (still in contrib) to c32[slot]
  // instead of contrib, and no wave speed
  float *c32;
};

struct GatherArgs
{
  int nnodes;
  int neq;
  int vbeg, vend; // node range of the launch (vend 0: all nodes)
  int part_off;    // first block partial written (norm modes)
  double *sq_out;  // fused final (mode bit 3) when set: the plain sum of the block sums here
  const int32_t *__restrict__ row;     // [nnodes+1]
  const int32_t *__restrict__ ent_slot; // [E]
  const int32_t *__restrict__ ent_ws;   // [E]
  const double *__restrict__ contrib;   // [neq][S]
  long long S;
  const double *__restrict__ wsc;
  const double *__restrict__ vol;
  const double *__restrict__ inv_vol;
  double *__restrict__ res; // SoA [neq][nnodes]
  double *__restrict__ ws;  // [nnodes]
  double *__restrict__ dt;  // [nnodes]
  double *__restrict__ u;   // SoA [neq][nnodes]
  double *__restrict__ part; // [nblocks][neq] norm partial sums
  double cfl;
  const int *stop;
  // fused final reduction (mode bit 3): the last block to finish reduces the partials
  unsigned *counter; // blocks done; reset to 0 by the last block
  double *norm, *norm0, *hist;
  int *iter;
  int max_iter;
  double drop;
  int *stop_w;
  unsigned *status;
  const LoopParams *loop; // non-null: cfl, drop, max_iter are read from here
  StallRec *stall;        // FP32-phase progress record (mixed loop)
  // Runge-Kutta stage combination (modes 16 / 17): rk_out = ca * rk_un + cb * rk_us
  // - cc * (dt * res), or rk_out = rk_un - dt * res when rk_first
  int rk_first;
  double rk_ca, rk_cb, rk_cc;
  const double *rk_un; // SoA [neq][nnodes]
  const double *rk_us;
  double *rk_out;
  // defect-correction loop (modes 18 / 19, one equation):
  // 18: the fused FP64 sweep that also keeps dres = dt res (its update), dtv = dt / V and the
  //     state it started from (ur);
  // 19: a correction sweep, u -= dres + dtv sum(c32 entries): c32 holds, per slot, the FP32
  //     change of the cell or facet contribution since the exact sweep
  const float *c32;
  double *dres;
  float *dtv;
  double *ur;
  int pdl; // launch with programmatic dependent launch (loop graphs)
};

// ---- launchers (return cudaError_t of the launch) --------------------------------------
// Cell residual kernels: dispatch over (physics, scheme, element type, order, precision).
cudaError_t launch_cells(const HostCellGroup &g, const CellArgs &a, int physics, int scheme,
                         int precision, int dim, int neq, cudaStream_t s, const char **name);
cudaError_t launch_bc(const HostBC &b, const BCArgs &a, int physics, int dim, int neq,
                      cudaStream_t s, const char **name);
// Node gather: mode bit 0 = compute dt, bit 1 = update u, bit 2 = norm partials, bit 3 = final
// reduction; 16 / 17 = residual (17: and dt) followed by a Runge-Kutta stage combination.
cudaError_t launch_gather(const GatherArgs &a, int mode, int nblocks, cudaStream_t s,
                          const char **name);
cudaError_t launch_norm_final(const double *part, int nblocks, int neq, int nnodes,
                              double *norm, double *norm0, double *hist, int *iter,
                              int max_hist, double drop, int *stop, unsigned *status,
                              cudaStream_t s, const char **name);
cudaError_t launch_norm_partials(int nnodes, int neq, const double *res, const double *dt,
                                 double *part, int nblocks, cudaStream_t s);
cudaError_t launch_cell_volume_raw(int ncells, int dim, int nq, int ngeo, const int32_t *geo_conn,
                                   const double *X, int ngeo_nodes, const double *w,
                                   const double *dVgeo, double *cvol, cudaStream_t s);
cudaError_t launch_cells_scalar(const HostCellGroup &g, const CellArgs &a, int physics,
                                int scheme, int precision, cudaStream_t s, const char **name,
                                bool *ok);
// lane-indexed tables of an Euler cell group (rds_cells_euler.cu); empty for other shapes
void euler_lane_tables(const HostCellGroup &g, int dim, std::vector<double> &out);

cudaError_t launch_cells_euler(const HostCellGroup &g, const CellArgs &a, int physics,
                               int scheme, int precision, cudaStream_t s, const char **name,
                               bool *ok);
cudaError_t launch_dual_volume(int nnodes, const int32_t *row, const int32_t *ent_ws,
                               const double *cvol, double *vol, double *inv_vol, cudaStream_t s);
// Batch mode: persistent cell kernel of a scalar group over its active tiles (block = tile).
cudaError_t launch_cells_scalar_batch(const HostCellGroup &g, const CellArgs &a, int precision,
                                      int grid, int tile, cudaStream_t s, const char **name,
                                      bool *ok);
// Batch mode: persistent gather over the active problems' node blocks with per-problem dt,
// update, norm and stop test; then the rebuild of the active lists after phase changes.
// dc: 0 plain, 1 exact sweep of the defect-correction loop (keeps rcell / ur), 2 correction
// sweep (no norm, no stop test).
cudaError_t launch_gather_batch(const GatherArgs &a, const BatchArgs &b, int grid, cudaStream_t s,
                                const char **name, int dc = 0,
                                int rk = 0);
cudaError_t launch_batch_rebuild(const RebuildArgs &r, cudaStream_t s, const char **name);
// Mixed form, scalar physics on straight-sided triangles: the cell kernel with the basis
// contractions on the tensor cores (persistent over 128-cell tiles; batch: active tiles).
bool tc_supported(const HostCellGroup &g);
void tc_tables(const HostCellGroup &g, std::vector<float> &out);
cudaError_t launch_cells_scalar_tc(const HostCellGroup &g, const CellArgs &a, bool batch, int grid,
                                   int ntiles, cudaStream_t s, const char **name, bool *ok);
// node-major [n][neq] <-> equation-major [neq][n] state (to_soa: the former to the latter)
cudaError_t launch_transpose_state(int nnodes, int neq, const double *src, double *dst,
                                   bool to_soa, cudaStream_t s, const char **name);
cudaError_t launch_update(int nnodes, int neq, const double *dt, const double *res, double *u,
                          cudaStream_t s, const char **name);
// Mixed form, scalar physics: FP32 correction-sweep cell kernels of the defect-correction loop;
// grid > 0 launches the batch form (persistent over a.bt's active tiles of `tile` cells).
bool dc_supported(const HostCellGroup &g);
cudaError_t launch_cells_scalar_dc(const HostCellGroup &g, const DcCellArgs &a, int grid,
                                   int tile, cudaStream_t s, const char **name, bool *ok);
// The correction sweeps between two exact sweeps in one launch (rds_cells_scalar_dc.cu,
// dc_sweeps_fused): one triangle group, up to kFuseMaxBC weak Dirichlet conditions. bar: two
// device words the launcher clears before the launch (grid barrier).
constexpr int kFuseMaxBC = 4;
struct DcFusedArgs
{
  DcCellArgs cell;
  BCArgs bc[kFuseMaxBC]; // with c32 set: the facets' changes
  int nbc;
  GatherArgs ga; // mode 19 fields: row, ent_slot, c32, dres, dtv, u, nnodes
  int nsweeps;
  unsigned *bar;
  unsigned *status;  // kFlagTimeout when a barrier wait gives up
  int wait_limit;    // polls of a barrier wait
  int test_extra;    // test option: arrivals a barrier waits for beyond the grid (0; 1 never
                     // completes, so every wait runs out)
};
bool dc_fused_supported(const HostCellGroup &g, const HostBC *const *bcs, int nbc);
cudaError_t launch_dc_fused(const HostCellGroup &g, const HostBC *const *bcs,
                            const DcFusedArgs &a, cudaStream_t s, const char **name, bool *ok);
// PGLDA / PGN element Jacobians (rds_jacobian.cu): jac [ncells][ndof*neq][ndof*neq]
cudaError_t launch_jacobians(const HostCellGroup &g, const CellArgs &a, int physics, int scheme,
                             int dim, int neq, double *jac, cudaStream_t s);

cudaError_t launch_assemble_bsr(long long nnzb, int neq, const int32_t *brow, const int64_t *cptr,
                                const int64_t *coff, const int32_t *cnr, const double *jac,
                                const double *vol, double *values, cudaStream_t s);

// partitioned single mesh (rds_partition.cu)
cudaError_t launch_pack_interface(int n, int neq, int nnodes, const int32_t *nodes,
                                  const int32_t *slots, const double *res, const double *ws,
                                  double *buf, size_t buf_len, cudaStream_t s);
cudaError_t launch_unpack_interface(int n, int neq, int nnodes, const int32_t *nodes,
                                    const int32_t *slots, const double *buf, double *res,
                                    double *ws, cudaStream_t s);
cudaError_t launch_rk_combine(int v0, int v1, int nnodes, int neq, int first, double cfl, double ca,
                              double cb, double cc, const double *vol, const double *ws,
                              const double *res, double *dt, const double *un, const double *us,
                              double *out, cudaStream_t s);
cudaError_t launch_finish(int v0, int v1, int nnodes, int neq, double cfl, int update,
                          const double *vol, const double *ws, const double *res, double *dt,
                          double *u, const uint8_t *owned, double *part, int part_off,
                          unsigned *counter, double *sq, cudaStream_t s);

// stabilisation operators (rds_stab.cu)
constexpr int kStabMaxGroups = 8;
constexpr int kStabMaxGeo    = 4; // geometry nodes of a cell the sensor maps (bilinear quads)
// cell groups as the node-parallel kernels decode them from the gather lists
struct StabGroups
{
  int n;
  long long slot_base[kStabMaxGroups];
  long long ws_base[kStabMaxGroups];
  int ncells[kStabMaxGroups], ndof[kStabMaxGroups], nvert[kStabMaxGroups];
  const int32_t *sol_conn[kStabMaxGroups];
  const double *P1[kStabMaxGroups]; // [ndof][nvert] vertex interpolant at the nodes
};
struct ViscArgs
{
  int ncells, ndof, nq, ngeo, nnodes, ngeo_nodes, affine;
  const int32_t *sol_conn, *geo_conn;
  const double *X, *u, *eps;
  const double *w, *V, *dV, *dVgeo; // [nq], [nq][ndof], [D][nq][ndof], [D][nq][ngeo]
  double *contrib;
  long long S, slot_base;
  const int *stop;
};
struct SensorArgs
{
  int ncells, ndof, nq, order, ngeo_nodes, blend;
  const int32_t *sol_conn, *geo_conn;
  const double *X, *u;           // u: the first state component [nnodes]
  const double *w, *Vn, *R;      // [nq], [nq][ndof], [nq][ndof]
  const double *dVgeo;           // [D][nq][ngeo] at the points: detJ per point (bilinear
  int ngeo;                      // quadrilaterals); NULL: affine simplices, detJ constant
  double kappa, factor;
  double *out;                   // [ncells]
};
cudaError_t launch_viscous(const ViscArgs &a, int dim, int neq, cudaStream_t s, const char **name);
cudaError_t launch_sensor(const SensorArgs &a, int dim, cudaStream_t s);
cudaError_t launch_normalise_max(int n, double *v, cudaStream_t s);
// kind 0: LF_Blend cell values ksi (pass 1), 1: Wong-Jansen (u_inf)
// Bonanni's pressure-based blending coefficient (rds_stab.cu)
struct BonanniArgs
{
  int ncells, ndof, nq, ngeo, nnodes, ngeo_nodes;
  const int32_t *sol_conn, *geo_conn; // SoA [ndof][ncells], [ngeo][ncells]
  const double *X, *u;                // SoA coordinates, state
  const double *w, *V, *dV, *dVgeo;   // the coefficient's rule: [nq], [nq][ndof], [D][nq][..]
  double gamma;
  double *f, *lc;                     // per cell: (v . grad p) |v| (cell means), |K|^(1/D)
  double *part;                       // per block: |K|, int V [D], p_min, p_max
};
cudaError_t launch_bonanni_cells(const BonanniArgs &a, int dim, cudaStream_t s);
// the block sums of all groups' launches ([nblocks][dim + 3]) -> delta = (p_max - p_min)|v_dom|^2,
// then theta = min(1, max(f / delta, 0)^2 lc) for the n cells of f / lc (in place in f)
cudaError_t launch_bonanni_finish(int dim, int nblocks, const double *part, double *delta, int n,
                                  double *f, const double *lc, cudaStream_t s);
int bonanni_blocks(int ncells);

cudaError_t launch_blend_cells(int kind, int ncells, int ndof, const int32_t *sol_conn,
                               const double *u, double param, double *out, cudaStream_t s);
// LF_Blend pass 2 / 3: nodal max of the cells' values; 1 - max over each cell's nodes
cudaError_t launch_node_max(int nnodes, const int32_t *row, const int32_t *ent_ws, long long wcells,
                            const double *cellf, double *nodef, cudaStream_t s);
cudaError_t launch_lf_finish(int ncells, int ndof, const int32_t *sol_conn, const double *nodef,
                             double *out, cudaStream_t s);
// cell values -> nodal field: vertex max, then the vertex interpolant at the other nodes
cudaError_t launch_cells_to_nodes(int nnodes, const int32_t *row, const int32_t *ent_slot,
                                  long long scells, const StabGroups &g, const double *cellf,
                                  double *nodef, cudaStream_t s);

} // namespace rds
