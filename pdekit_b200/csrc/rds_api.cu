// Host runtime behind the C ABI (include/rds_b200.h): device buffers, the node-centred gather
// lists, launch sequencing, the CUDA-graph pseudo-time loop, error reporting and per-kernel
// event timing.

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "rds_internal.h"

using namespace rds;

namespace
{

struct TimingRec
{
  const char *name;
  cudaEvent_t a, b;
};

} // namespace

struct rds_ctx
{
  rds_desc desc{};
  int device             = 0;
  cudaStream_t stream    = nullptr;
  cudaStream_t side      = nullptr; // boundary kernels, concurrent with the cell kernels
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // one more side stream per further weak condition (they write disjoint slots, so they run
  // concurrently with each other as well), with its join event
  static constexpr int kMaxSides = 8;
  cudaStream_t sides[kMaxSides] = {};
  cudaEvent_t ev_joins[kMaxSides] = {};
  bool own_stream        = false;
  bool finalized         = false;
  std::string err;
  long long launches = 0;

  std::vector<HostCellGroup> groups;
  std::vector<double> hX; // geometry coordinates [dim][node] (constant-Jacobian checks)
  std::vector<HostBC> bcs;

  double *d_X       = nullptr; // SoA coords [dim][ngeo_nodes]
  double *d_u       = nullptr; // SoA [neq][nnodes]
  double *d_res     = nullptr;
  double *d_ws      = nullptr;
  double *d_dt      = nullptr;
  double *d_vol     = nullptr;
  double *d_inv_vol = nullptr;
  double *d_contrib = nullptr; // [neq][S]
  double *d_wsc     = nullptr; // [W]
  double *d_stage   = nullptr; // AoS staging [nnodes*neq]
  int32_t *d_row = nullptr, *d_ent_slot = nullptr, *d_ent_ws = nullptr;
  double *d_part = nullptr, *d_norm = nullptr, *d_norm0 = nullptr, *d_hist = nullptr;
  int *d_iter = nullptr, *d_stop = nullptr, *d_zero = nullptr;
  unsigned *d_status = nullptr;
  unsigned *d_counter = nullptr; // blocks done in the fused gather (last-block reduction)
  long long S = 0, W = 0, E = 0;
  int gblocks   = 0;
  int hist_cap  = 0;

  // sparse (block CSR) Jacobian: pattern over node pairs, per-block contribution lists into
  // the element-Jacobian buffer (built on first use)
  bool jp_built = false;
  long long jp_nnzb = 0, jp_njac = 0;
  std::vector<int32_t> jp_row_ptr, jp_col_idx;
  std::vector<long long> jp_gbase;
  int32_t *d_jp_brow = nullptr, *d_jp_cnr = nullptr;
  int64_t *d_jp_cptr = nullptr, *d_jp_coff = nullptr;
  double *d_jp_jac = nullptr;
  double *d_theta   = nullptr; // PGB Jacobians: per-cell blending coefficients of one group
  long long theta_cap = 0;

  // stabilisation (rds_stab.cu): external nodal blending coefficient read by PGB cells, nodal
  // artificial viscosity added by PGLDA cells, scratch cell / node values; per group the
  // sensor tables (w, Vn, R), the vertex interpolant P1 and device copies of the tables of the
  // viscous term. All in 'extra'.
  double *d_blend = nullptr, *d_av = nullptr, *d_cellf = nullptr, *d_nodef = nullptr;
  bool blend_on = false, av_on = false;
  struct StabTab
  {
    int nq = 0, nvert = 0;
    double *w = nullptr, *Vn = nullptr, *R = nullptr, *P1 = nullptr;
    double *vw = nullptr, *vV = nullptr, *vdV = nullptr, *vdVgeo = nullptr;
    int sngeo  = 0; // the sensor's geometry derivatives at its points (non-affine cells)
    double *sdVgeo = nullptr;
    int bnq    = 0; // Bonanni's coefficient: its rule, basis and geometry derivatives
    double *bw = nullptr, *bV = nullptr, *bdV = nullptr, *bdVgeo = nullptr;
  };
  std::vector<StabTab> stab;
  double *d_bon = nullptr; // Bonanni's coefficient: lc per cell, block sums, delta
  size_t bon_len = 0;

  // pipelined host-buffer steps (rds_step_host): copy streams, double-buffered staging
  cudaStream_t h_in = nullptr, h_out = nullptr;
  cudaEvent_t ev_in_ready[2] = {nullptr, nullptr}, ev_in_free[2] = {nullptr, nullptr};
  cudaEvent_t ev_out_ready[2] = {nullptr, nullptr}, ev_out_free[2] = {nullptr, nullptr};
  double *d_hin[2] = {nullptr, nullptr}, *d_hout[2] = {nullptr, nullptr};
  double *d_hnorm[2] = {nullptr, nullptr};
  long long hstep = 0;

  // partitioned single mesh: the nodes this rank shares with others, their slots in the
  // exchange buffer, and the nodes whose (res dt)^2 this rank counts in the norm
  int32_t *d_if_nodes = nullptr, *d_if_slots = nullptr;
  uint8_t *d_owned    = nullptr;
  int n_if = 0, n_slots = 0;

  // pinned host scalars for the loop's stop test
  int *h_stop = nullptr;

  // CUDA graphs: a chunk of fused iterations with FP64 cells (0), FP32 cells (1), batched
  // problems (2); one iteration without stop test for rds_run, FP64 (3) / FP32 (4) cells;
  // one third-order TVD Runge-Kutta step (5); cycles of the defect-correction loop (6).
  // The loop parameters are read from d_loop, so a graph stays valid across calls.
  static constexpr int kChunk    = 16;
  static constexpr int kGraphs   = 7;
  cudaGraphExec_t graph_exec[kGraphs] = {nullptr, nullptr, nullptr, nullptr,
                                         nullptr, nullptr, nullptr};
  LoopParams *d_loop            = nullptr;
  double rk_cfl                 = 0.0; // CFL the Runge-Kutta graph was captured with

  // Runge-Kutta stage states u_1, u_2 and the later stages' residual (SoA [neq][nnodes])
  double *d_rk_u1 = nullptr, *d_rk_u2 = nullptr, *d_rk_res = nullptr;
  int rk_stage = 0; // partitioned RK3TVD: the stage rds_rk_stage_state selected (0: none)
  double *rk_base_u = nullptr, *rk_base_res = nullptr; // the context's own state / residual

  // precision of the cell kernels being launched (the mixed loop finishes in FP64)
  int active_precision = RDS_FP64;
  // mixed form: relative residual at which the loop switches from FP32 to FP64 cell kernels
  // (earlier when the FP32 phase stops making progress)
  double mixed_switch = 1.e-6;
  // mixed form: basis contractions on the tensor cores where built (option "tensor_cores";
  // off by default: slower than the CUDA-core FP32 kernel at these contraction sizes)
  bool use_tc         = false;
  int stall_min       = 200; // FP32 phase stalled: no halving of the drop for
  double stall_mult   = 3.0; //   max(stall_min, stall_mult x the last interval between halvings)
  StallRec *d_stall   = nullptr; // FP32-phase progress record of the single-problem loop

  // mixed form, scalar physics on triangles: defect-correction loop (run_loop_dc). An exact
  // FP64 sweep every dc_m sweeps keeps its update dt res (d_dres), dt / V (d_dtv) and the state
  // it started from (d_ur); the sweeps in between add the FP32 changes of every cell and facet
  // contribution since then (d_c32, one value per slot), the cells' with the blending
  // coefficients of PGB frozen at d_ur (d_dc_theta, one per cell)
  bool dc_ok         = false;
  int dc_m           = 24; // 32 let 3 of configuration 5's Burgers P1 problems diverge
  int dc_phase       = 0; // launch_residual_kernels: 0 plain, 1 exact DC sweep, 2 correction
  int part_used      = 0;     // norm partials written by rds_gather_finish (partitioned)
  LoopParams *h_loop = nullptr;   // pinned host copy of the loop parameters (set_loop_params)
  cudaEvent_t ev_loop = nullptr;  // the last copy from it
  LoopParams loop_last{};         // the parameters on the device
  bool loop_set = false;
  int tc_test_wait   = 0;     // option "tc_test_wait" (the bounded-wait test)
  int grp_beg        = 0;     // launch_residual_kernels: cell groups [grp_beg, grp_end)
  int grp_end        = -1;    //   (-1: all) and the weak conditions unless no_bcs
  bool no_bcs        = false;
  // loop graphs: the main-stream kernels of an iteration (first cell group, gather) with
  // programmatic dependent launch (option "loop_pdl", default off: measured no gain on the
  // configurations, whose critical path runs through the side-stream boundary kernels)
  int loop_pdl       = 0;
  double *d_ur = nullptr, *d_dres = nullptr, *d_dc_theta = nullptr;
  float *d_c32 = nullptr, *d_dtv = nullptr;
  // the correction sweeps of a cycle in one launch (dc_sweeps_fused) for meshes of at most
  // dc_fuse_cells cells (option "mixed_fuse_cells"; 0: separate launches); d_fbar its barrier
  long long dc_fuse_cells = 1LL << 16;
  unsigned *d_fbar        = nullptr;
  int fuse_test_wait      = 0; // option "fuse_test_wait" (the barrier's bounded-wait test)
  std::vector<long long> dc_cell_base; // first cell of each group in d_dc_theta
  StallRec *d_pstall  = nullptr; // the same per batched problem

  // batched independent problems (rds_set_problems): one context holds their disjoint union
  int nprob = 0;
  std::vector<int32_t> prob_nodes; // [P+1] node offsets
  std::vector<double> prob_cfl;    // [P]
  int32_t *d_node_off = nullptr, *d_nb_base = nullptr, *d_nb_prefix = nullptr;
  int32_t *d_phase = nullptr, *d_piter = nullptr, *d_changed = nullptr;
  int32_t *d_tile = nullptr, *d_tile_prefix = nullptr, *d_cbeg = nullptr, *d_cend = nullptr;
  double *d_pcfl = nullptr, *d_pnorm = nullptr, *d_pnorm0 = nullptr;
  unsigned *d_pcount = nullptr, *d_pstatus = nullptr;
  int nsm         = 0;
  int batch_grid  = 0; // persistent grid of the batched gather
  bool tuned      = false;
  std::string tune_report;
  std::vector<void *> extra; // further device buffers, freed with the context

  bool timing = false;
  std::vector<TimingRec> trecs;
  std::vector<cudaEvent_t> ev_pool;
};

namespace
{

rds_status fail(rds_ctx *c, rds_status st, const std::string &msg)
{
  if (c)
    c->err = msg;
  return st;
}

#define RDS_CUDA(call)                                                                             \
  do                                                                                               \
  {                                                                                                \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return fail(ctx, RDS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));          \
  } while (0)

cudaEvent_t get_event(rds_ctx *ctx)
{
  if (!ctx->ev_pool.empty())
  {
    cudaEvent_t e = ctx->ev_pool.back();
    ctx->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

// Launch wrapper: optional event timing around the launch (on the stream it is issued to),
// launch counting, error text.
template <typename F>
rds_status launch_on(rds_ctx *ctx, cudaStream_t s, F &&f)
{
  cudaEvent_t a = nullptr, b = nullptr;
  if (ctx->timing)
  {
    a = get_event(ctx);
    b = get_event(ctx);
    cudaEventRecord(a, s);
  }
  const char *name = "?";
  cudaError_t e    = f(&name);
  if (e == cudaErrorNotSupported)
    return fail(ctx, RDS_ERR_UNSUPPORTED,
                std::string("no kernel compiled for this configuration (") + name + ")");
  if (e != cudaSuccess)
    return fail(ctx, RDS_ERR_CUDA, std::string(name) + ": " + cudaGetErrorString(e));
  ctx->launches++;
  if (ctx->timing)
  {
    cudaEventRecord(b, s);
    ctx->trecs.push_back({name, a, b});
  }
  return RDS_OK;
}

template <typename F>
rds_status launch(rds_ctx *ctx, F &&f)
{
  return launch_on(ctx, ctx->stream, f);
}

template <typename T>
rds_status dalloc(rds_ctx *ctx, T **p, size_t n)
{
  if (n == 0)
    n = 1;
  cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
  if (e != cudaSuccess)
    return fail(ctx, RDS_ERR_CUDA,
                std::string("cudaMalloc(") + std::to_string(n * sizeof(T)) +
                    " bytes): " + cudaGetErrorString(e));
  return RDS_OK;
}

template <typename T>
rds_status upload(rds_ctx *ctx, T *d, const T *h, size_t n)
{
  RDS_CUDA(cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  return RDS_OK;
}

// SoA transposition of a [rows][cols] int32 table to [cols][rows] on the host.
std::vector<int32_t> transpose_i32(const int32_t *a, int rows, int cols)
{
  std::vector<int32_t> t((size_t)rows * cols);
  for (int r = 0; r < rows; ++r)
    for (int c = 0; c < cols; ++c)
      t[(size_t)c * rows + r] = a[(size_t)r * cols + c];
  return t;
}

bool supported_physics(const rds_desc &d)
{
  switch (d.physics)
  {
  case RDS_ADVECTION_CONST:
  case RDS_BURGERS2D:
    return d.dim == 2 && d.neq == 1;
  case RDS_EULER2D:
    return d.dim == 2 && d.neq == 4;
  case RDS_EULER3D:
    return d.dim == 3 && d.neq == 5;
  default:
    return false;
  }
}

CellArgs cell_args(rds_ctx *ctx, const HostCellGroup &g, const int *stop)
{
  CellArgs a{};
  a.ncells     = g.desc.ncells;
  a.nnodes     = ctx->desc.nnodes;
  a.sol_conn   = g.d_sol_conn;
  a.geo_conn   = g.d_geo_conn;
  a.X          = ctx->d_X;
  a.ngeo_nodes = ctx->desc.ngeo_nodes;
  a.u          = ctx->d_u;
  a.contrib    = ctx->d_contrib;
  a.S          = ctx->S;
  a.slot_base  = g.slot_base;
  a.wsc        = ctx->d_wsc;
  a.ws_base    = g.ws_base;
  a.adv0       = ctx->desc.adv[0];
  a.adv1       = ctx->desc.adv[1];
  a.adv2       = ctx->desc.adv[2];
  a.gamma      = ctx->desc.gamma;
  a.status     = ctx->d_status;
  a.stop       = stop;
  a.blend      = ctx->blend_on ? ctx->d_blend : nullptr;
  a.tc_test_wait = ctx->tc_test_wait;
  return a;
}

ViscArgs visc_args(rds_ctx *ctx, size_t ig, const int *stop)
{
  const HostCellGroup &g   = ctx->groups[ig];
  const rds_ctx::StabTab &t = ctx->stab[ig];
  ViscArgs a{};
  a.ncells     = g.desc.ncells;
  a.ndof       = g.desc.ndof;
  a.nq         = (int)g.w.size();
  a.ngeo       = g.desc.ngeo;
  a.nnodes     = ctx->desc.nnodes;
  a.ngeo_nodes = ctx->desc.ngeo_nodes;
  a.affine     = g.affine ? 1 : 0;
  a.sol_conn   = g.d_sol_conn;
  a.geo_conn   = g.d_geo_conn;
  a.X          = ctx->d_X;
  a.u          = ctx->d_u;
  a.eps        = ctx->d_av;
  a.w          = t.vw;
  a.V          = t.vV;
  a.dV         = t.vdV;
  a.dVgeo      = t.vdVgeo;
  a.contrib    = ctx->d_contrib;
  a.S          = ctx->S;
  a.slot_base  = g.slot_base;
  a.stop       = stop;
  return a;
}

BCArgs bc_args(rds_ctx *ctx, const HostBC &b, const int *stop)
{
  BCArgs a{};
  a.nfacets    = b.desc.nfacets;
  a.sol_conn   = b.d_sol_conn;
  a.geo_conn   = b.d_geo_conn;
  a.X          = ctx->d_X;
  a.ngeo_nodes = ctx->desc.ngeo_nodes;
  a.u          = ctx->d_u;
  a.nnodes     = ctx->desc.nnodes;
  a.gq         = b.d_gq;
  a.vol        = ctx->d_vol;
  a.contrib    = ctx->d_contrib;
  a.S          = ctx->S;
  a.slot_base  = b.slot_base;
  a.wsc        = ctx->d_wsc;
  a.ws_base    = b.ws_base;
  a.adv0       = ctx->desc.adv[0];
  a.adv1       = ctx->desc.adv[1];
  a.gamma      = ctx->desc.gamma;
  // WeakWall relaxation of the dof residuals (bc/WeakWall.hpp:112-116)
  a.relax = (b.desc.order <= 1) ? 1.0 : 1. / (3. * b.desc.order);
  for (int k = 0; k < 4; ++k)
    a.params[k] = b.desc.params[k];
  a.status     = ctx->d_status;
  a.stop       = stop;
  if (b.desc.kind == RDS_BC_STRONG_DIRICHLET)
  {
    a.nfacets  = b.nstrong;
    a.u_strong = ctx->d_u;
  }
  return a;
}

GatherArgs gather_args(rds_ctx *ctx, double cfl, const int *stop)
{
  GatherArgs a{};
  a.nnodes   = ctx->desc.nnodes;
  a.neq      = ctx->desc.neq;
  a.row      = ctx->d_row;
  a.ent_slot = ctx->d_ent_slot;
  a.ent_ws   = ctx->d_ent_ws;
  a.contrib  = ctx->d_contrib;
  a.S        = ctx->S;
  a.wsc      = ctx->d_wsc;
  a.vol      = ctx->d_vol;
  a.inv_vol  = ctx->d_inv_vol;
  a.res      = ctx->d_res;
  a.ws       = ctx->d_ws;
  a.dt       = ctx->d_dt;
  a.u        = ctx->d_u;
  a.part     = ctx->d_part;
  a.cfl      = cfl;
  a.stop     = stop;
  return a;
}

// Side stream of the k-th weak condition (the first one is ctx->side).
cudaStream_t side_stream(rds_ctx *ctx, int k)
{
  const int n = std::min((int)ctx->bcs.size(), rds_ctx::kMaxSides);
  k           = k % std::max(1, n);
  return k == 0 ? ctx->side : ctx->sides[k];
}

// Forks the side streams of the conditions from the main stream (a parallel graph branch each
// when captured).
rds_status fork_sides(rds_ctx *ctx)
{
  const int n = std::min((int)ctx->bcs.size(), rds_ctx::kMaxSides);
  RDS_CUDA(cudaEventRecord(ctx->ev_fork, ctx->stream));
  for (int k = 0; k < n; ++k)
    RDS_CUDA(cudaStreamWaitEvent(side_stream(ctx, k), ctx->ev_fork, 0));
  return RDS_OK;
}

// Joins the side streams into the main stream.
rds_status join_sides(rds_ctx *ctx)
{
  const int n = std::min((int)ctx->bcs.size(), rds_ctx::kMaxSides);
  for (int k = 0; k < n; ++k)
  {
    cudaEvent_t e = k == 0 ? ctx->ev_join : ctx->ev_joins[k];
    RDS_CUDA(cudaEventRecord(e, side_stream(ctx, k)));
    RDS_CUDA(cudaStreamWaitEvent(ctx->stream, e, 0));
  }
  return RDS_OK;
}

// Arguments of a correction sweep's cell kernel (defect-correction loop) for group ig.
static DcCellArgs dc_cell_args(rds_ctx *ctx, size_t ig, const int *stop)
{
  const HostCellGroup &g = ctx->groups[ig];
  DcCellArgs da{};
  da.ncells     = g.desc.ncells;
  da.sol_conn   = g.d_sol_conn;
  da.geo_conn   = g.d_geo_conn;
  da.X          = ctx->d_X;
  da.ngeo_nodes = ctx->desc.ngeo_nodes;
  da.u          = ctx->d_u;
  da.ur         = ctx->d_ur;
  da.c32        = ctx->d_c32;
  da.slot_base  = g.slot_base;
  da.theta      = ctx->d_dc_theta + ctx->dc_cell_base[ig];
  da.adv0       = ctx->desc.adv[0];
  da.adv1       = ctx->desc.adv[1];
  da.stop       = stop;
  return da;
}

// Residual contributions of all cells and boundary facets (assemble_rhs without the gather).
// The boundary-facet kernels only touch their own contribution slots, so they run on a side
// stream concurrently with the cell kernels (a parallel branch when captured in a graph) and
// join the main stream before the gather.
rds_status launch_residual_kernels(rds_ctx *ctx, const int *stop)
{
  const rds_desc &d = ctx->desc;
  // A strong Dirichlet condition writes the state that the cells read and that the conditions
  // after it read: then the conditions run after the cells, in order, on the main stream.
  bool strong = false;
  for (const HostBC &b : ctx->bcs)
    strong |= b.desc.kind == RDS_BC_STRONG_DIRICHLET;
  const bool with_bcs = !ctx->bcs.empty() && !ctx->no_bcs;
  // per-kernel event timing: every kernel alone on the main stream, so that each event pair
  // brackets one kernel and not its overlap with the others (the results do not change: the
  // conditions write their own slots)
  const bool fork     = with_bcs && !strong && !ctx->timing;
  // stream of the k-th condition: all on s (in order), or one side stream each when forked
  auto launch_bcs = [&](cudaStream_t s, bool spread) -> rds_status {
    for (size_t k = 0; k < ctx->bcs.size(); ++k)
    {
      const HostBC &b    = ctx->bcs[k];
      const cudaStream_t sk = spread ? side_stream(ctx, (int)k) : s;
      BCArgs a = bc_args(ctx, b, stop);
      if (ctx->dc_phase == 2)
        a.c32 = ctx->d_c32; // the change since the exact sweep, in FP32
      rds_status st  = launch_on(ctx, sk, [&](const char **name) {
        return launch_bc(b, a, b.physics, d.dim, d.neq, sk, name);
      });
      if (st != RDS_OK)
        return st;
    }
    return RDS_OK;
  };
  if (fork)
  {
    rds_status st = fork_sides(ctx);
    if (st == RDS_OK)
      st = launch_bcs(ctx->side, true);
    if (st != RDS_OK)
      return st;
  }
  const size_t gend = ctx->grp_end < 0 ? ctx->groups.size() : (size_t)ctx->grp_end;
  for (size_t ig = (size_t)ctx->grp_beg; ig < gend; ++ig)
  {
    const HostCellGroup &g = ctx->groups[ig];
    CellArgs a             = cell_args(ctx, g, stop);
    // programmatic dependent launch for the first cell group of a loop iteration (the kernel
    // before it on the stream is the previous iteration's gather)
    a.pdl = (ctx->loop_pdl && !ctx->timing && ig == 0) ? 1 : 0;
    if (ctx->dc_phase == 1 && g.scheme == RDS_PGB)
      a.theta = ctx->d_dc_theta + ctx->dc_cell_base[ig]; // blending coefficients at u_r
    rds_status st          = launch(ctx, [&](const char **name) {
      if (ctx->dc_phase == 2)
      {
        // correction sweep: the FP32 change of the cell residual since the exact sweep
        DcCellArgs da = dc_cell_args(ctx, ig, stop);
        da.pdl        = (ctx->loop_pdl && !ctx->timing && ig == 0) ? 1 : 0;
        bool ok       = false;
        const cudaError_t e = launch_cells_scalar_dc(g, da, 0, 0, ctx->stream, name, &ok);
        return ok ? e : cudaErrorNotSupported;
      }
      if (ctx->active_precision == RDS_MIXED && ctx->use_tc && g.d_tc && !ctx->blend_on)
      {
        // FP32 cells with the basis contractions on the tensor cores, persistent CTAs
        const int ntiles = (g.desc.ncells + 127) / 128;
        const int grid   = std::max(1, std::min(ntiles, 4 * ctx->nsm));
        bool ok          = false;
        const cudaError_t e =
            launch_cells_scalar_tc(g, a, false, grid, ntiles, ctx->stream, name, &ok);
        return ok ? e : cudaErrorNotSupported;
      }
      return launch_cells(g, a, g.physics, g.scheme, ctx->active_precision, d.dim, d.neq,
                          ctx->stream, name);
    });
    if (st != RDS_OK)
      return st;
    // PGLDA with a nodal artificial viscosity: the viscous term added to the group's slots
    if (ctx->av_on && g.scheme == RDS_PGLDA)
    {
      const ViscArgs va = visc_args(ctx, ig, stop);
      st                = launch(ctx, [&](const char **name) {
        return launch_viscous(va, d.dim, d.neq, ctx->stream, name);
      });
      if (st != RDS_OK)
        return st;
    }
  }
  if (fork)
    return join_sides(ctx);
  if (with_bcs)
    return launch_bcs(ctx->stream, false);
  return RDS_OK;
}

rds_status check_status(rds_ctx *ctx)
{
  unsigned st = 0;
  RDS_CUDA(cudaMemcpyAsync(&st, ctx->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost,
                           ctx->stream));
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  if (st & kFlagNonFinite)
    return fail(ctx, RDS_ERR_NONFINITE, "non-finite residual norm");
  if (st & kFlagNegPressure)
    return fail(ctx, RDS_ERR_NEG_PRESSURE, "non-positive pressure met");
  if (st & kFlagTimeout)
    return fail(ctx, RDS_ERR_CUDA, "a bounded device wait (tensor-core commit or fused-sweep barrier) gave up");
  return RDS_OK;
}

void release_graph(rds_ctx *ctx)
{
  for (int k = 0; k < rds_ctx::kGraphs; ++k)
    if (ctx->graph_exec[k])
    {
      cudaGraphExecDestroy(ctx->graph_exec[k]);
      ctx->graph_exec[k] = nullptr;
    }
}

} // namespace

namespace rds
{

cudaError_t launch_cells(const HostCellGroup &g, const CellArgs &a, int physics, int scheme,
                         int precision, int dim, int neq, cudaStream_t s, const char **name)
{
  bool ok         = false;
  cudaError_t err = cudaSuccess;
  if (physics == RDS_ADVECTION_CONST || physics == RDS_BURGERS2D)
    err = launch_cells_scalar(g, a, physics, scheme, precision, s, name, &ok);
  else
    err = launch_cells_euler(g, a, physics, scheme, precision, s, name, &ok);
  (void)dim;
  (void)neq;
  if (!ok)
    return cudaErrorNotSupported;
  return err;
}

} // namespace rds

// ============================================================================================
// C ABI
// ============================================================================================

extern "C" {

const char *rds_version(void)
{
  return "rds_b200 0.1 (sm_100a)";
}

const char *rds_last_error(rds_ctx *ctx)
{
  return ctx ? ctx->err.c_str() : "null context";
}

void *rds_stream(rds_ctx *ctx)
{
  return ctx ? (void *)ctx->stream : nullptr;
}

long long rds_launch_count(rds_ctx *ctx)
{
  return ctx ? ctx->launches : 0;
}

rds_status rds_create(rds_ctx **out, const rds_desc *desc, void *stream)
{
  if (!out || !desc)
    return RDS_ERR_INVALID;
  *out         = nullptr;
  rds_ctx *ctx = new rds_ctx();
  ctx->desc    = *desc;
  ctx->active_precision = desc->precision;
  const rds_desc &d = ctx->desc;
  if (!supported_physics(d) || d.scheme < RDS_PGLDA || d.scheme > RDS_PGPSI ||
      (d.precision != RDS_FP64 && d.precision != RDS_MIXED) || d.nnodes <= 0 ||
      d.ngeo_nodes <= 0 || !desc->geo_coords)
  {
    rds_status st = RDS_ERR_INVALID;
    *out          = ctx;
    return fail(ctx, st, "invalid descriptor (physics/dim/neq/scheme/precision/sizes)");
  }
  if (d.scheme == RDS_PGPSI && (d.neq != 1 || d.precision != RDS_FP64))
  {
    *out = ctx;
    return fail(ctx, RDS_ERR_UNSUPPORTED, "the PSI scheme: scalar physics in FP64 contexts only");
  }
  *out = ctx;
  if (cudaGetDevice(&ctx->device) != cudaSuccess)
    return fail(ctx, RDS_ERR_CUDA, "no CUDA device");
  if (stream)
    ctx->stream = (cudaStream_t)stream;
  else
  {
    RDS_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    ctx->own_stream = true;
  }
  RDS_CUDA(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
  RDS_CUDA(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
  RDS_CUDA(cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
  rds_status st;
  const size_t ng = (size_t)d.ngeo_nodes;
  std::vector<double> X(ng * d.dim);
  for (size_t i = 0; i < ng; ++i)
    for (int k = 0; k < d.dim; ++k)
      X[k * ng + i] = desc->geo_coords[i * d.dim + k];
  if ((st = dalloc(ctx, &ctx->d_X, X.size())) != RDS_OK)
    return st;
  if ((st = upload(ctx, ctx->d_X, X.data(), X.size())) != RDS_OK)
    return st;
  ctx->hX = X;
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->desc.geo_coords = nullptr;
  return RDS_OK;
}

// True when the bilinear map of every cell of a 4-node quadrilateral group has a constant
// Jacobian (all cells parallelograms, to 1e-14 of the cell's extent). The per-point Jacobian
// derivatives of the geometry basis then differ from those at point 0 by multiples of one
// nodal "twist" vector t (the bilinear mode); a cell is a parallelogram when sum_g t_g X_g = 0.
static bool parallelogram_cells(const rds_ctx *ctx, const rds_cell_group &g)
{
  const int D = ctx->desc.dim, NG = g.ngeo;
  if (ctx->hX.empty() || D != 2)
    return false;
  double t[4] = {0, 0, 0, 0}, best = 0.0;
  for (int xi = 0; xi < D; ++xi)
    for (int q = 1; q < g.nq; ++q)
    {
      double dv[4], nrm = 0.0;
      for (int k = 0; k < NG; ++k)
      {
        dv[k] = g.dVgeo[((size_t)xi * g.nq + q) * NG + k] - g.dVgeo[((size_t)xi * g.nq) * NG + k];
        nrm += dv[k] * dv[k];
      }
      if (nrm > best)
      {
        best = nrm;
        for (int k = 0; k < NG; ++k)
          t[k] = dv[k];
      }
    }
  if (best == 0.0)
    return true;
  const size_t ng = (size_t)ctx->desc.ngeo_nodes;
  for (int c = 0; c < g.ncells; ++c)
  {
    const int32_t *cn = g.geo_conn + (size_t)c * NG;
    for (int x = 0; x < D; ++x)
    {
      const double *Xx = ctx->hX.data() + (size_t)x * ng;
      double tw = 0.0, ext = 0.0;
      for (int k = 0; k < NG; ++k)
      {
        tw += t[k] * Xx[cn[k]];
        ext = std::max(ext, std::fabs(Xx[cn[k]] - Xx[cn[0]]));
      }
      if (std::fabs(tw) > 1.e-14 * ext * std::sqrt(best))
        return false;
    }
  }
  return true;
}

rds_status rds_add_cell_group(rds_ctx *ctx, const rds_cell_group *g)
{
  if (!ctx || !g)
    return RDS_ERR_INVALID;
  if (ctx->finalized)
    return fail(ctx, RDS_ERR_INVALID, "rds_add_cell_group after rds_finalize");
  const int D = ctx->desc.dim;
  if (g->ncells <= 0 || g->ndof <= 0 || g->ndof > 32 || g->ngeo <= 0 || g->ngeo > 27 ||
      g->nq <= 0 || g->nq > 64 || g->nfl <= 0 || g->nfl > 64 || !g->sol_conn || !g->geo_conn ||
      !g->w || !g->V || !g->dV || !g->dVgeo || !g->dVf || !g->Vsf)
    return fail(ctx, RDS_ERR_INVALID, "invalid cell group");
  for (size_t i = 0; i < (size_t)g->ncells * g->ndof; ++i)
    if (g->sol_conn[i] < 0 || g->sol_conn[i] >= ctx->desc.nnodes)
      return fail(ctx, RDS_ERR_INVALID, "solution connectivity out of range");
  for (size_t i = 0; i < (size_t)g->ncells * g->ngeo; ++i)
    if (g->geo_conn[i] < 0 || g->geo_conn[i] >= ctx->desc.ngeo_nodes)
      return fail(ctx, RDS_ERR_INVALID, "geometry connectivity out of range");
  HostCellGroup h;
  h.desc = *g;
  h.w.assign(g->w, g->w + g->nq);
  h.V.assign(g->V, g->V + (size_t)g->nq * g->ndof);
  h.dV.assign(g->dV, g->dV + (size_t)D * g->nq * g->ndof);
  h.dVgeo.assign(g->dVgeo, g->dVgeo + (size_t)D * g->nq * g->ngeo);
  h.dVf.assign(g->dVf, g->dVf + (size_t)D * g->nq * g->nfl);
  h.Vsf.assign(g->Vsf, g->Vsf + (size_t)g->nfl * g->ndof);
  if (g->nqv > 0)
  {
    if (!g->wv || !g->dVgeo_v || g->nqv > 64)
      return fail(ctx, RDS_ERR_INVALID, "invalid dual-volume rule");
    h.wv.assign(g->wv, g->wv + g->nqv);
    h.dVgeo_v.assign(g->dVgeo_v, g->dVgeo_v + (size_t)D * g->nqv * g->ngeo);
  }
  h.affine = (g->shape == RDS_TRIAG && g->ngeo == 3) || (g->shape == RDS_TETRA && g->ngeo == 4);
  h.const_jac = h.affine || (g->shape == RDS_QUAD && g->ngeo == 4 &&
                                parallelogram_cells(ctx, *g));
  h.physics = ctx->desc.physics;
  h.scheme  = ctx->desc.scheme;
  rds_status st;
  const std::vector<int32_t> sc = transpose_i32(g->sol_conn, g->ncells, g->ndof);
  const std::vector<int32_t> gc = transpose_i32(g->geo_conn, g->ncells, g->ngeo);
  if ((st = dalloc(ctx, &h.d_sol_conn, sc.size())) != RDS_OK)
    return st;
  if ((st = dalloc(ctx, &h.d_geo_conn, gc.size())) != RDS_OK)
    return st;
  if ((st = upload(ctx, h.d_sol_conn, sc.data(), sc.size())) != RDS_OK)
    return st;
  if ((st = upload(ctx, h.d_geo_conn, gc.data(), gc.size())) != RDS_OK)
    return st;
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  h.desc.sol_conn = h.desc.geo_conn = nullptr;
  h.desc.w = h.desc.V = h.desc.dV = h.desc.dVgeo = h.desc.dVf = h.desc.Vsf = nullptr;
  h.desc.wv = h.desc.dVgeo_v = nullptr;
  ctx->groups.push_back(h);
  return RDS_OK;
}

rds_status rds_add_bc(rds_ctx *ctx, const rds_bc_group *b)
{
  if (!ctx || !b)
    return RDS_ERR_INVALID;
  if (ctx->finalized)
    return fail(ctx, RDS_ERR_INVALID, "rds_add_bc after rds_finalize");
  const int D = ctx->desc.dim, NEQ = ctx->desc.neq;
  const bool dirichlet = b->kind == RDS_BC_WEAK_DIRICHLET;
  const bool farfield  = b->kind == RDS_BC_WEAK_FARFIELD;
  const bool strong    = b->kind == RDS_BC_STRONG_DIRICHLET;
  if (b->kind < RDS_BC_WEAK_DIRICHLET || b->kind > RDS_BC_WEAK_SYMMETRY || b->nfacets <= 0 ||
      b->nfdof <= 0 || b->nfdof > 16 || !b->sol_conn || ((dirichlet || farfield || strong) && !b->gq))
    return fail(ctx, RDS_ERR_INVALID, "invalid boundary group");
  if (!strong && (b->nfgeo <= 0 || b->nfgeo > 16 || b->nfq <= 0 || b->nfq > 32 || !b->geo_conn ||
                  !b->fw || !b->fV || !b->fdVgeo))
    return fail(ctx, RDS_ERR_INVALID, "invalid boundary group");
  if (NEQ == 1 && !(dirichlet || strong))
    return fail(ctx, RDS_ERR_UNSUPPORTED, "this boundary condition needs Euler physics");
  for (size_t i = 0; i < (size_t)b->nfacets * b->nfdof; ++i)
    if (b->sol_conn[i] < 0 || b->sol_conn[i] >= ctx->desc.nnodes)
      return fail(ctx, RDS_ERR_INVALID, "boundary solution connectivity out of range");
  if (!strong)
    for (size_t i = 0; i < (size_t)b->nfacets * b->nfgeo; ++i)
      if (b->geo_conn[i] < 0 || b->geo_conn[i] >= ctx->desc.ngeo_nodes)
        return fail(ctx, RDS_ERR_INVALID, "boundary geometry connectivity out of range");
  HostBC h;
  h.desc    = *b;
  h.physics = ctx->desc.physics;
  std::vector<int32_t> sc, gc(1, 0);
  std::vector<double> gq(1, 0.0);
  if (strong)
  {
    // the value each dof ends with (the last facet that names it) for the distinct dofs in
    // ascending order, so that the kernel writes every dof once
    std::vector<long long> last(ctx->desc.nnodes, -1);
    for (size_t i = 0; i < (size_t)b->nfacets * b->nfdof; ++i)
      last[b->sol_conn[i]] = (long long)i;
    for (int v = 0; v < ctx->desc.nnodes; ++v)
      if (last[v] >= 0)
        sc.push_back(v);
    h.nstrong = (int)sc.size();
    gq.assign((size_t)NEQ * sc.size(), 0.0);
    for (size_t k = 0; k < sc.size(); ++k)
      for (int e = 0; e < NEQ; ++e)
        gq[(size_t)e * sc.size() + k] = b->gq[(size_t)last[sc[k]] * NEQ + e];
  }
  else
  {
    h.fw.assign(b->fw, b->fw + b->nfq);
    h.fV.assign(b->fV, b->fV + (size_t)b->nfq * b->nfdof);
    h.fdVgeo.assign(b->fdVgeo, b->fdVgeo + (size_t)(D - 1) * b->nfq * b->nfgeo);
    sc = transpose_i32(b->sol_conn, b->nfacets, b->nfdof);
    gc = transpose_i32(b->geo_conn, b->nfacets, b->nfgeo);
    if (dirichlet)
    {
      gq.assign((size_t)NEQ * b->nfq * b->nfacets, 0.0);
      for (int f = 0; f < b->nfacets; ++f)
        for (int q = 0; q < b->nfq; ++q)
          for (int e = 0; e < NEQ; ++e)
            gq[((size_t)e * b->nfq + q) * b->nfacets + f] =
                b->gq[((size_t)f * b->nfq + q) * NEQ + e];
    }
    else if (farfield)
      gq.assign(b->gq, b->gq + NEQ);
  }
  rds_status st;
  if ((st = dalloc(ctx, &h.d_sol_conn, sc.size())) != RDS_OK ||
      (st = dalloc(ctx, &h.d_geo_conn, gc.size())) != RDS_OK ||
      (st = dalloc(ctx, &h.d_gq, gq.size())) != RDS_OK)
    return st;
  if ((st = upload(ctx, h.d_sol_conn, sc.data(), sc.size())) != RDS_OK ||
      (st = upload(ctx, h.d_geo_conn, gc.data(), gc.size())) != RDS_OK ||
      (st = upload(ctx, h.d_gq, gq.data(), gq.size())) != RDS_OK)
    return st;
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  h.desc.sol_conn = h.desc.geo_conn = nullptr;
  h.desc.fw = h.desc.fV = h.desc.fdVgeo = h.desc.gq = nullptr;
  ctx->bcs.push_back(h);
  return RDS_OK;
}

// Batch set-up: per-problem node ranges and norm-partial slots, per-group problem cell ranges
// and tile sizes, and the device-side phase / iteration / norm arrays of the problems.
static rds_status finalize_batch(rds_ctx *ctx)
{
  const int P = ctx->nprob, NEQ = ctx->desc.neq, G = (int)ctx->groups.size();
  for (const HostCellGroup &g : ctx->groups)
    if (g.pcells.empty())
      return fail(ctx, RDS_ERR_INVALID,
                  "batched context: every cell group needs its problem ranges "
                  "(rds_add_batch_cell_group)");
  std::vector<int32_t> nb_base(P), cbeg((size_t)G * P), cend((size_t)G * P), tile((size_t)G * 2);
  long long nb = 0;
  for (int p = 0; p < P; ++p)
  {
    nb_base[p] = (int32_t)nb;
    nb += (ctx->prob_nodes[p + 1] - ctx->prob_nodes[p] + kGBlock - 1) / kGBlock;
  }
  for (int g = 0; g < G; ++g)
  {
    const HostCellGroup &h = ctx->groups[g];
    for (int p = 0; p < P; ++p)
    {
      cbeg[(size_t)g * P + p] = h.pcells[p];
      cend[(size_t)g * P + p] = h.pcells[p + 1];
    }
    tile[g * 2]     = h.tune_tile[0];
    tile[g * 2 + 1] = h.tune_tile[1];
  }
  rds_status st = RDS_OK;
  auto track    = [&](auto **ptr, size_t n) {
    if (st == RDS_OK && (st = dalloc(ctx, ptr, n)) == RDS_OK)
      ctx->extra.push_back((void *)*ptr);
  };
  track(&ctx->d_node_off, P + 1);
  track(&ctx->d_nb_base, P);
  track(&ctx->d_nb_prefix, P + 1);
  track(&ctx->d_pcfl, P);
  track(&ctx->d_pcount, P);
  track(&ctx->d_phase, P);
  track(&ctx->d_piter, P);
  track(&ctx->d_pnorm, (size_t)P * NEQ);
  track(&ctx->d_pnorm0, (size_t)P * NEQ);
  track(&ctx->d_pstatus, P);
  track(&ctx->d_changed, 1);
  track(&ctx->d_tile, (size_t)G * 2);
  track(&ctx->d_tile_prefix, (size_t)G * 2 * (P + 1));
  track(&ctx->d_cbeg, (size_t)G * P);
  track(&ctx->d_cend, (size_t)G * P);
  track(&ctx->d_pstall, P);
  if (st != RDS_OK)
    return st;
  if (nb > ctx->gblocks)
  {
    cudaFree(ctx->d_part);
    ctx->d_part = nullptr;
    if ((st = dalloc(ctx, &ctx->d_part, (size_t)nb * NEQ)) != RDS_OK)
      return st;
  }
  if ((st = upload(ctx, ctx->d_node_off, ctx->prob_nodes.data(), P + 1)) ||
      (st = upload(ctx, ctx->d_nb_base, nb_base.data(), P)) ||
      (st = upload(ctx, ctx->d_pcfl, ctx->prob_cfl.data(), P)) ||
      (st = upload(ctx, ctx->d_tile, tile.data(), tile.size())) ||
      (st = upload(ctx, ctx->d_cbeg, cbeg.data(), cbeg.size())) ||
      (st = upload(ctx, ctx->d_cend, cend.data(), cend.size())))
    return st;
  RDS_CUDA(cudaMemsetAsync(ctx->d_pcount, 0, P * sizeof(unsigned), ctx->stream));
  for (int g = 0; g < G; ++g)
  {
    ctx->groups[g].d_cbeg = ctx->d_cbeg + (size_t)g * P;
    ctx->groups[g].d_cend = ctx->d_cend + (size_t)g * P;
  }
  ctx->batch_grid = ctx->nsm * 8; // 8 resident blocks of kGBlock threads per SM
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  return RDS_OK;
}

rds_status rds_finalize(rds_ctx *ctx)
{
  if (!ctx)
    return RDS_ERR_INVALID;
  if (ctx->finalized)
    return RDS_OK;
  if (ctx->groups.empty())
    return fail(ctx, RDS_ERR_INVALID, "no cell group");
  const rds_desc &d = ctx->desc;
  const int N       = d.nnodes;

  // Slot layout: per group n-major [ndof][ncells], then per BC [nfdof][nfacets].
  long long S = 0, W = 0;
  for (HostCellGroup &g : ctx->groups)
  {
    g.slot_base = S;
    g.ws_base   = W;
    S += (long long)g.desc.ndof * g.desc.ncells;
    W += g.desc.ncells;
  }
  for (HostBC &b : ctx->bcs)
  {
    if (b.desc.kind == RDS_BC_STRONG_DIRICHLET)
      continue; // writes the state, no residual contributions
    b.slot_base = S;
    b.ws_base   = W;
    S += (long long)b.desc.nfdof * b.desc.nfacets;
    W += (long long)b.desc.nfdof * b.desc.nfacets;
  }
  if (S >= (1LL << 31) || W >= (1LL << 31))
    return fail(ctx, RDS_ERR_TOO_LARGE, "more than 2^31 contribution slots");
  ctx->S = S;
  ctx->W = W;

  // Gather lists (CSR over nodes): cells of each group in ascending order, then BC facets in
  // the order the conditions were added. Host copies of the connectivity are rebuilt from the
  // device (they were transposed on upload).
  std::vector<int32_t> count(N + 1, 0);
  std::vector<std::vector<int32_t>> gconn(ctx->groups.size()), bconn(ctx->bcs.size());
  for (size_t ig = 0; ig < ctx->groups.size(); ++ig)
  {
    const HostCellGroup &g = ctx->groups[ig];
    gconn[ig].resize((size_t)g.desc.ncells * g.desc.ndof);
    RDS_CUDA(cudaMemcpy(gconn[ig].data(), g.d_sol_conn, gconn[ig].size() * 4,
                        cudaMemcpyDeviceToHost));
    for (int32_t v : gconn[ig])
      count[v + 1]++;
  }
  for (size_t ib = 0; ib < ctx->bcs.size(); ++ib)
  {
    const HostBC &b = ctx->bcs[ib];
    if (b.desc.kind == RDS_BC_STRONG_DIRICHLET)
      continue;
    bconn[ib].resize((size_t)b.desc.nfacets * b.desc.nfdof);
    RDS_CUDA(cudaMemcpy(bconn[ib].data(), b.d_sol_conn, bconn[ib].size() * 4,
                        cudaMemcpyDeviceToHost));
    for (int32_t v : bconn[ib])
      count[v + 1]++;
  }
  for (int i = 0; i < N; ++i)
    count[i + 1] += count[i];
  const long long E = count[N];
  ctx->E            = E;
  std::vector<int32_t> pos(count.begin(), count.end() - 1);
  std::vector<int32_t> ent_slot(E), ent_ws(E);
  for (size_t ig = 0; ig < ctx->groups.size(); ++ig)
  {
    const HostCellGroup &g = ctx->groups[ig];
    const int nc = g.desc.ncells, nd = g.desc.ndof;
    for (int c = 0; c < nc; ++c)
      for (int n = 0; n < nd; ++n)
      {
        const int v      = gconn[ig][(size_t)n * nc + c];
        const int p      = pos[v]++;
        ent_slot[p]      = (int32_t)(g.slot_base + (long long)n * nc + c);
        ent_ws[p]        = (int32_t)(g.ws_base + c);
      }
  }
  for (size_t ib = 0; ib < ctx->bcs.size(); ++ib)
  {
    const HostBC &b = ctx->bcs[ib];
    if (b.desc.kind == RDS_BC_STRONG_DIRICHLET)
      continue;
    const int nf = b.desc.nfacets, nd = b.desc.nfdof;
    for (int f = 0; f < nf; ++f)
      for (int n = 0; n < nd; ++n)
      {
        const int v = bconn[ib][(size_t)n * nf + f];
        const int p = pos[v]++;
        ent_slot[p] = (int32_t)(b.slot_base + (long long)n * nf + f);
        ent_ws[p]   = (int32_t)(b.ws_base + (long long)n * nf + f);
      }
  }
  for (int v = 0; v < N; ++v)
    if (count[v + 1] == count[v])
      return fail(ctx, RDS_ERR_INVALID, "solution node " + std::to_string(v) +
                                            " belongs to no cell");

  rds_status st;
  const int NEQ = d.neq;
  ctx->gblocks  = (N + kGBlock - 1) / kGBlock;
  if ((st = dalloc(ctx, &ctx->d_u, (size_t)N * NEQ)) || (st = dalloc(ctx, &ctx->d_res, (size_t)N * NEQ)) ||
      (st = dalloc(ctx, &ctx->d_ws, N)) || (st = dalloc(ctx, &ctx->d_dt, N)) ||
      (st = dalloc(ctx, &ctx->d_vol, N)) || (st = dalloc(ctx, &ctx->d_inv_vol, N)) ||
      (st = dalloc(ctx, &ctx->d_contrib, (size_t)S * NEQ)) || (st = dalloc(ctx, &ctx->d_wsc, W)) ||
      (st = dalloc(ctx, &ctx->d_stage, (size_t)N * NEQ)) || (st = dalloc(ctx, &ctx->d_row, N + 1)) ||
      (st = dalloc(ctx, &ctx->d_ent_slot, E)) || (st = dalloc(ctx, &ctx->d_ent_ws, E)) ||
      (st = dalloc(ctx, &ctx->d_part, (size_t)(ctx->gblocks + 1) * NEQ)) || // +1: two node ranges
      (st = dalloc(ctx, &ctx->d_norm, NEQ)) || (st = dalloc(ctx, &ctx->d_norm0, NEQ)) ||
      (st = dalloc(ctx, &ctx->d_iter, 1)) || (st = dalloc(ctx, &ctx->d_stop, 1)) ||
      (st = dalloc(ctx, &ctx->d_zero, 1)) || (st = dalloc(ctx, &ctx->d_status, 1)) ||
      (st = dalloc(ctx, &ctx->d_counter, 1)))
    return st;
  RDS_CUDA(cudaMallocHost(&ctx->h_stop, sizeof(int)));
  RDS_CUDA(cudaMemsetAsync(ctx->d_u, 0, (size_t)N * NEQ * sizeof(double), ctx->stream));
  RDS_CUDA(cudaMemsetAsync(ctx->d_res, 0, (size_t)N * NEQ * sizeof(double), ctx->stream));
  RDS_CUDA(cudaMemsetAsync(ctx->d_dt, 0, (size_t)N * sizeof(double), ctx->stream));
  RDS_CUDA(cudaMemsetAsync(ctx->d_ws, 0, (size_t)N * sizeof(double), ctx->stream));
  RDS_CUDA(cudaMemsetAsync(ctx->d_zero, 0, sizeof(int), ctx->stream));
  RDS_CUDA(cudaMemsetAsync(ctx->d_stop, 0, sizeof(int), ctx->stream));
  RDS_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(unsigned), ctx->stream));
  RDS_CUDA(cudaMemsetAsync(ctx->d_counter, 0, sizeof(unsigned), ctx->stream));
  RDS_CUDA(cudaMemsetAsync(ctx->d_wsc, 0, (size_t)W * sizeof(double), ctx->stream));
  if ((st = upload(ctx, ctx->d_row, count.data(), N + 1)) ||
      (st = upload(ctx, ctx->d_ent_slot, ent_slot.data(), E)) ||
      (st = upload(ctx, ctx->d_ent_ws, ent_ws.data(), E)))
    return st;

  // Dual volumes: per-cell volume into the wave-speed slot space, then a gather (boundary
  // slots hold zero).
  for (const HostCellGroup &g : ctx->groups)
  {
    // the cell's own-order rule when given (as the reference), else the residual rule
    const bool own                  = !g.wv.empty();
    const std::vector<double> &w    = own ? g.wv : g.w;
    const std::vector<double> &dvg  = own ? g.dVgeo_v : g.dVgeo;
    const int nqv                   = (int)w.size();
    double *dw = nullptr, *ddv = nullptr;
    if ((st = dalloc(ctx, &dw, w.size())) || (st = dalloc(ctx, &ddv, dvg.size())))
      return st;
    if ((st = upload(ctx, dw, w.data(), w.size())) ||
        (st = upload(ctx, ddv, dvg.data(), dvg.size())))
      return st;
    RDS_CUDA(launch_cell_volume_raw(g.desc.ncells, d.dim, nqv, g.desc.ngeo, g.d_geo_conn,
                                    ctx->d_X, d.ngeo_nodes, dw, ddv, ctx->d_wsc + g.ws_base,
                                    ctx->stream));
    RDS_CUDA(cudaStreamSynchronize(ctx->stream));
    cudaFree(dw);
    cudaFree(ddv);
  }
  RDS_CUDA(launch_dual_volume(N, ctx->d_row, ctx->d_ent_ws, ctx->d_wsc, ctx->d_vol,
                              ctx->d_inv_vol, ctx->stream));
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  if ((st = dalloc(ctx, &ctx->d_loop, 1)) != RDS_OK ||
      (st = dalloc(ctx, &ctx->d_stall, 1)) != RDS_OK)
    return st;
  ctx->extra.push_back(ctx->d_stall);
  // mixed form: operand tables of the tensor-core cell kernel (scalar physics, triangles)
  if (d.precision == RDS_MIXED)
    for (HostCellGroup &g : ctx->groups)
    {
      std::vector<float> tct;
      tc_tables(g, tct);
      if (tct.empty())
        continue;
      if ((st = dalloc(ctx, &g.d_tc, tct.size())) != RDS_OK ||
          (st = upload(ctx, g.d_tc, tct.data(), tct.size())) != RDS_OK)
        return st;
      ctx->extra.push_back(g.d_tc);
      g.tune_tile[0] = 128; // one cell per TMEM lane
    }
  // Euler 2D: lane-indexed tables of the cell kernels (FP64, and FP32 for the mixed form)
  if (NEQ > 1 && d.dim == 2)
    for (HostCellGroup &g : ctx->groups)
    {
      std::vector<double> lt;
      euler_lane_tables(g, d.dim, lt);
      if ((st = dalloc(ctx, &g.d_lt64, lt.size())) != RDS_OK ||
          (st = upload(ctx, g.d_lt64, lt.data(), lt.size())) != RDS_OK)
        return st;
      ctx->extra.push_back(g.d_lt64);
      if (d.precision == RDS_MIXED)
      {
        std::vector<float> lt32(lt.begin(), lt.end());
        if ((st = dalloc(ctx, &g.d_lt32, lt32.size())) != RDS_OK ||
            (st = upload(ctx, g.d_lt32, lt32.data(), lt32.size())) != RDS_OK)
          return st;
        ctx->extra.push_back(g.d_lt32);
      }
    }
  // side streams of the weak conditions after the first (rds_ctx::sides)
  for (int k = 1; k < std::min((int)ctx->bcs.size(), rds_ctx::kMaxSides); ++k)
  {
    RDS_CUDA(cudaStreamCreateWithFlags(&ctx->sides[k], cudaStreamNonBlocking));
    RDS_CUDA(cudaEventCreateWithFlags(&ctx->ev_joins[k], cudaEventDisableTiming));
  }
  // mixed form, scalar physics: buffers of the defect-correction loop
  if (d.precision == RDS_MIXED && NEQ == 1)
  {
    bool ok = true;
    for (const HostCellGroup &g : ctx->groups)
      ok = ok && dc_supported(g);
    if (ok)
    {
      long long nc = 0;
      ctx->dc_cell_base.clear();
      for (const HostCellGroup &g : ctx->groups)
      {
        ctx->dc_cell_base.push_back(nc);
        nc += g.desc.ncells;
      }
      if ((st = dalloc(ctx, &ctx->d_ur, N)) != RDS_OK ||
          (st = dalloc(ctx, &ctx->d_dres, N)) != RDS_OK ||
          (st = dalloc(ctx, &ctx->d_dtv, N)) != RDS_OK ||
          (st = dalloc(ctx, &ctx->d_c32, (size_t)S)) != RDS_OK ||
          (st = dalloc(ctx, &ctx->d_dc_theta, (size_t)nc)) != RDS_OK ||
          (st = dalloc(ctx, &ctx->d_fbar, 2)) != RDS_OK)
        return st;
      ctx->extra.push_back(ctx->d_fbar);
      ctx->extra.push_back(ctx->d_ur);
      ctx->extra.push_back(ctx->d_dres);
      ctx->extra.push_back(ctx->d_dtv);
      ctx->extra.push_back(ctx->d_c32);
      ctx->extra.push_back(ctx->d_dc_theta);
      RDS_CUDA(cudaMemsetAsync(ctx->d_dc_theta, 0, (size_t)nc * sizeof(double), ctx->stream));
      ctx->dc_ok = true;
    }
  }
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  RDS_CUDA(cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, ctx->device));
  if (ctx->nprob > 0 && (st = finalize_batch(ctx)) != RDS_OK)
    return st;
  ctx->finalized = true;
  return RDS_OK;
}

rds_status rds_set_state(rds_ctx *ctx, const double *u)
{
  if (!ctx || !u || !ctx->finalized)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_set_state: not finalized or null") : RDS_ERR_INVALID;
  const int N = ctx->desc.nnodes, NEQ = ctx->desc.neq;
  if (NEQ == 1)
  {
    RDS_CUDA(cudaMemcpyAsync(ctx->d_u, u, (size_t)N * sizeof(double), cudaMemcpyHostToDevice,
                             ctx->stream));
  }
  else
  {
    RDS_CUDA(cudaMemcpyAsync(ctx->d_stage, u, (size_t)N * NEQ * sizeof(double),
                             cudaMemcpyHostToDevice, ctx->stream));
    // node-major staging -> equation-major state
    return launch(ctx, [&](const char **name) {
      return launch_transpose_state(N, NEQ, ctx->d_stage, ctx->d_u, true, ctx->stream, name);
    });
  }
  return RDS_OK;
}

static rds_status get_soa(rds_ctx *ctx, const double *d_soa, double *h_aos, int neq)
{
  const int N = ctx->desc.nnodes;
  if (neq == 1)
  {
    RDS_CUDA(cudaMemcpyAsync(h_aos, d_soa, (size_t)N * sizeof(double), cudaMemcpyDeviceToHost,
                             ctx->stream));
  }
  else
  {
    const rds_status st = launch(ctx, [&](const char **name) {
      return launch_transpose_state(N, neq, d_soa, ctx->d_stage, false, ctx->stream, name);
    });
    if (st != RDS_OK)
      return st;
    RDS_CUDA(cudaMemcpyAsync(h_aos, ctx->d_stage, (size_t)N * neq * sizeof(double),
                             cudaMemcpyDeviceToHost, ctx->stream));
  }
  return RDS_OK;
}

rds_status rds_get_state(rds_ctx *ctx, double *u)
{
  if (!ctx || !u || !ctx->finalized)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_get_state: not finalized or null") : RDS_ERR_INVALID;
  rds_status st = get_soa(ctx, ctx->d_u, u, ctx->desc.neq);
  if (st != RDS_OK)
    return st;
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  return RDS_OK;
}

static rds_status assemble_impl(rds_ctx *ctx, double cfl, int mode)
{
  if (!ctx || !ctx->finalized)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "not finalized") : RDS_ERR_INVALID;
  rds_status st = launch_residual_kernels(ctx, ctx->d_zero);
  if (st != RDS_OK)
    return st;
  const GatherArgs ga = gather_args(ctx, cfl, ctx->d_zero);
  return launch(ctx, [&](const char **name) {
    return launch_gather(ga, mode, ctx->gblocks, ctx->stream, name);
  });
}

rds_status rds_assemble(rds_ctx *ctx, double cfl)
{
  return assemble_impl(ctx, cfl, 1);
}

rds_status rds_assemble_rhs(rds_ctx *ctx)
{
  return assemble_impl(ctx, 0.0, 0);
}

rds_status rds_assemble_rhs_cells(rds_ctx *ctx, int g0, int g1, int with_bcs)
{
  if (!ctx || !ctx->finalized)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "not finalized") : RDS_ERR_INVALID;
  if (g0 < 0 || g1 < g0 || g1 > (int)ctx->groups.size())
    return fail(ctx, RDS_ERR_INVALID, "rds_assemble_rhs_cells: group range out of bounds");
  ctx->grp_beg         = g0;
  ctx->grp_end         = g1;
  ctx->no_bcs          = with_bcs == 0;
  const rds_status st  = launch_residual_kernels(ctx, ctx->d_zero);
  ctx->grp_beg         = 0;
  ctx->grp_end         = -1;
  ctx->no_bcs          = false;
  return st;
}

rds_status rds_gather_rhs(rds_ctx *ctx, int v0, int v1)
{
  if (!ctx || !ctx->finalized)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "not finalized") : RDS_ERR_INVALID;
  if (v0 < 0 || v1 < v0 || v1 > ctx->desc.nnodes)
    return fail(ctx, RDS_ERR_INVALID, "rds_gather_rhs: node range out of bounds");
  if (v1 == v0)
    return RDS_OK;
  GatherArgs ga = gather_args(ctx, 0.0, ctx->d_zero);
  ga.vbeg       = v0;
  ga.vend       = v1;
  const int nb  = (v1 - v0 + kGBlock - 1) / kGBlock;
  return launch(ctx, [&](const char **name) {
    return launch_gather(ga, 0, nb, ctx->stream, name);
  });
}

rds_status rds_update(rds_ctx *ctx)
{
  if (!ctx || !ctx->finalized)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "not finalized") : RDS_ERR_INVALID;
  return launch(ctx, [&](const char **name) {
    return launch_update(ctx->desc.nnodes, ctx->desc.neq, ctx->d_dt, ctx->d_res, ctx->d_u,
                         ctx->stream, name);
  });
}

rds_status rds_residual_norm(rds_ctx *ctx, double *norm)
{
  if (!ctx || !norm || !ctx->finalized)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "not finalized or null") : RDS_ERR_INVALID;
  const int N = ctx->desc.nnodes, NEQ = ctx->desc.neq;
  rds_status st = launch(ctx, [&](const char **name) {
    *name = "norm_partials";
    return launch_norm_partials(N, NEQ, ctx->d_res, ctx->d_dt, ctx->d_part, ctx->gblocks,
                                ctx->stream);
  });
  if (st != RDS_OK)
    return st;
  st = launch(ctx, [&](const char **name) {
    return launch_norm_final(ctx->d_part, ctx->gblocks, NEQ, N, ctx->d_norm, nullptr, nullptr,
                             nullptr, 0, 0.0, nullptr, nullptr, ctx->stream, name);
  });
  if (st != RDS_OK)
    return st;
  RDS_CUDA(cudaMemcpyAsync(norm, ctx->d_norm, NEQ * sizeof(double), cudaMemcpyDeviceToHost,
                           ctx->stream));
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  return RDS_OK;
}

// ---- element Jacobians ------------------------------------------------------------------

// Cell arguments of a Jacobian launch; for PGB the cells' blending coefficients are computed
// first by the FP64 residual kernel at the current state (its contributions are scratch).
static rds_status jacobian_args(rds_ctx *ctx, size_t ig, CellArgs *out)
{
  const HostCellGroup &g = ctx->groups[ig];
  CellArgs a             = cell_args(ctx, g, ctx->d_zero);
  if (ctx->desc.scheme == RDS_PGB)
  {
    if (ctx->theta_cap < g.desc.ncells)
    {
      cudaFree(ctx->d_theta);
      ctx->d_theta   = nullptr;
      ctx->theta_cap = 0;
      rds_status st  = dalloc(ctx, &ctx->d_theta, (size_t)g.desc.ncells);
      if (st != RDS_OK)
        return st;
      ctx->theta_cap = g.desc.ncells;
    }
    a.theta       = ctx->d_theta;
    rds_status st = launch(ctx, [&](const char **name) {
      return launch_cells(g, a, g.physics, g.scheme, RDS_FP64, ctx->desc.dim, ctx->desc.neq,
                          ctx->stream, name);
    });
    if (st != RDS_OK)
      return st;
  }
  *out = a;
  return RDS_OK;
}

rds_status rds_element_jacobians(rds_ctx *ctx, int group, double *jac)
{
  if (!ctx || !jac || !ctx->finalized || group < 0 || group >= (int)ctx->groups.size())
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_element_jacobians: invalid group or not finalized")
               : RDS_ERR_INVALID;
  if (ctx->nprob > 0)
    return fail(ctx, RDS_ERR_UNSUPPORTED, "rds_element_jacobians: not in batched contexts");
  if (ctx->desc.scheme == RDS_PGPSI)
    return fail(ctx, RDS_ERR_UNSUPPORTED, "rds_element_jacobians: not for the PSI scheme");
  const HostCellGroup &g = ctx->groups[group];
  if (ctx->blend_on && ctx->desc.scheme == RDS_PGB)
    return fail(ctx, RDS_ERR_UNSUPPORTED,
                "rds_element_jacobians: PGB with an external blending coefficient");
  CellArgs a;
  rds_status st = jacobian_args(ctx, (size_t)group, &a);
  if (st != RDS_OK)
    return st;
  return launch(ctx, [&](const char **name) {
    *name = "cells_jacobian";
    return launch_jacobians(g, a, g.physics, ctx->desc.scheme, ctx->desc.dim, ctx->desc.neq, jac,
                            ctx->stream);
  });
}

// ---- sparse Jacobian ---------------------------------------------------------------------

// Block pattern of the assembled Jacobian: block (v, w) exists when a cell holds both nodes;
// its contributions are the (m(v), n(w)) blocks of those cells' element matrices, in ascending
// group and cell order.
static rds_status build_jac_pattern(rds_ctx *ctx)
{
  if (ctx->jp_built)
    return RDS_OK;
  const long long N = ctx->desc.nnodes;
  const int NEQ     = ctx->desc.neq;
  struct Contrib
  {
    long long key, off;
    int32_t nr;
  };
  std::vector<Contrib> t;
  long long total = 0, base = 0;
  for (const HostCellGroup &g : ctx->groups)
    total += (long long)g.desc.ncells * g.desc.ndof * g.desc.ndof;
  t.reserve((size_t)total);
  ctx->jp_gbase.clear();
  for (const HostCellGroup &g : ctx->groups)
  {
    const int nc = g.desc.ncells, nd = g.desc.ndof, NR = nd * NEQ;
    std::vector<int32_t> conn((size_t)nc * nd);
    RDS_CUDA(cudaMemcpy(conn.data(), g.d_sol_conn, conn.size() * 4, cudaMemcpyDeviceToHost));
    ctx->jp_gbase.push_back(base);
    for (int c = 0; c < nc; ++c)
      for (int m = 0; m < nd; ++m)
        for (int n = 0; n < nd; ++n)
        {
          const long long v = conn[(size_t)m * nc + c], w = conn[(size_t)n * nc + c];
          t.push_back({v * N + w,
                       base + (long long)c * NR * NR + (long long)m * NEQ * NR + (long long)n * NEQ,
                       NR});
        }
    base += (long long)nc * NR * NR;
  }
  ctx->jp_njac = base;
  std::stable_sort(t.begin(), t.end(),
                   [](const Contrib &a, const Contrib &b) { return a.key < b.key; });
  std::vector<int32_t> brow, cnr(t.size());
  std::vector<int64_t> cptr, coff(t.size());
  ctx->jp_row_ptr.assign((size_t)N + 1, 0);
  ctx->jp_col_idx.clear();
  for (size_t k = 0; k < t.size(); ++k)
  {
    if (k == 0 || t[k].key != t[k - 1].key)
    {
      const long long v = t[k].key / N, w = t[k].key % N;
      brow.push_back((int32_t)v);
      ctx->jp_col_idx.push_back((int32_t)w);
      ctx->jp_row_ptr[(size_t)v + 1]++;
      cptr.push_back((int64_t)k);
    }
    coff[k] = t[k].off;
    cnr[k]  = t[k].nr;
  }
  cptr.push_back((int64_t)t.size());
  for (long long v = 0; v < N; ++v)
    ctx->jp_row_ptr[(size_t)v + 1] += ctx->jp_row_ptr[(size_t)v];
  ctx->jp_nnzb = (long long)brow.size();
  rds_status st;
  if ((st = dalloc(ctx, &ctx->d_jp_brow, brow.size())) != RDS_OK ||
      (st = dalloc(ctx, &ctx->d_jp_cptr, cptr.size())) != RDS_OK ||
      (st = dalloc(ctx, &ctx->d_jp_coff, coff.size())) != RDS_OK ||
      (st = dalloc(ctx, &ctx->d_jp_cnr, cnr.size())) != RDS_OK ||
      (st = dalloc(ctx, &ctx->d_jp_jac, (size_t)ctx->jp_njac)) != RDS_OK)
    return st;
  if ((st = upload(ctx, ctx->d_jp_brow, brow.data(), brow.size())) != RDS_OK ||
      (st = upload(ctx, ctx->d_jp_cptr, cptr.data(), cptr.size())) != RDS_OK ||
      (st = upload(ctx, ctx->d_jp_coff, coff.data(), coff.size())) != RDS_OK ||
      (st = upload(ctx, ctx->d_jp_cnr, cnr.data(), cnr.size())) != RDS_OK)
    return st;
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->jp_built = true;
  return RDS_OK;
}

rds_status rds_jacobian_pattern(rds_ctx *ctx, int64_t *nnzb, int32_t *row_ptr, int32_t *col_idx)
{
  if (!ctx || !nnzb || !ctx->finalized || ctx->nprob > 0)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_jacobian_pattern: not a finalized single context")
               : RDS_ERR_INVALID;
  rds_status st = build_jac_pattern(ctx);
  if (st != RDS_OK)
    return st;
  *nnzb = ctx->jp_nnzb;
  if (row_ptr)
    std::copy(ctx->jp_row_ptr.begin(), ctx->jp_row_ptr.end(), row_ptr);
  if (col_idx)
    std::copy(ctx->jp_col_idx.begin(), ctx->jp_col_idx.end(), col_idx);
  return RDS_OK;
}

rds_status rds_assemble_jacobian(rds_ctx *ctx, double *values)
{
  if (!ctx || !values || !ctx->finalized || ctx->nprob > 0)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_assemble_jacobian: not a finalized single context")
               : RDS_ERR_INVALID;
  if (ctx->desc.scheme == RDS_PGPSI)
    return fail(ctx, RDS_ERR_UNSUPPORTED, "rds_assemble_jacobian: not for the PSI scheme");
  rds_status st = build_jac_pattern(ctx);
  if (st != RDS_OK)
    return st;
  for (size_t ig = 0; ig < ctx->groups.size(); ++ig)
  {
    const HostCellGroup &g = ctx->groups[ig];
    CellArgs a;
    if ((st = jacobian_args(ctx, ig, &a)) != RDS_OK)
      return st;
    st = launch(ctx, [&](const char **name) {
      *name = "cells_jacobian";
      return launch_jacobians(g, a, g.physics, ctx->desc.scheme, ctx->desc.dim, ctx->desc.neq,
                              ctx->d_jp_jac + ctx->jp_gbase[ig], ctx->stream);
    });
    if (st != RDS_OK)
      return st;
  }
  return launch(ctx, [&](const char **name) {
    *name = "assemble_bsr";
    return launch_assemble_bsr(ctx->jp_nnzb, ctx->desc.neq, ctx->d_jp_brow, ctx->d_jp_cptr,
                               ctx->d_jp_coff, ctx->d_jp_cnr, ctx->d_jp_jac, ctx->d_vol, values,
                               ctx->stream);
  });
}

// ---- pipelined host-buffer steps --------------------------------------------------------

// Per call: upload (stream h_in) into staging buffer k, compute stream: layout conversion into
// the state, one fused iteration, the norm, the state into output buffer k; download (stream
// h_out). Buffers alternate between calls, so the upload of the next call and the download of
// the previous one overlap this call's compute; events keep a buffer from being overwritten
// while a copy still reads it.
// ---- stabilisation fields and operators --------------------------------------------------

static rds_status stab_alloc(rds_ctx *ctx, double **p, size_t n)
{
  const rds_status st = dalloc(ctx, p, n);
  if (st == RDS_OK)
    ctx->extra.push_back(*p);
  return st;
}

static rds_status stab_upload(rds_ctx *ctx, double **p, const double *h, size_t n)
{
  rds_status st;
  if ((st = stab_alloc(ctx, p, n)) != RDS_OK || (st = upload(ctx, *p, h, n)) != RDS_OK)
    return st;
  return RDS_OK;
}

static rds_status stab_check(rds_ctx *ctx, const char *fn)
{
  if (!ctx)
    return RDS_ERR_INVALID;
  if (!ctx->finalized)
    return fail(ctx, RDS_ERR_INVALID, std::string(fn) + ": not finalized");
  if (ctx->nprob > 0)
    return fail(ctx, RDS_ERR_UNSUPPORTED, std::string(fn) + ": not in batched contexts");
  ctx->stab.resize(ctx->groups.size());
  return RDS_OK;
}

// device copies of the residual tables each group's viscous term reads
static rds_status ensure_visc_tables(rds_ctx *ctx)
{
  for (size_t ig = 0; ig < ctx->groups.size(); ++ig)
  {
    const HostCellGroup &g = ctx->groups[ig];
    rds_ctx::StabTab &t    = ctx->stab[ig];
    if (t.vw)
      continue;
    rds_status st;
    if ((st = stab_upload(ctx, &t.vw, g.w.data(), g.w.size())) ||
        (st = stab_upload(ctx, &t.vV, g.V.data(), g.V.size())) ||
        (st = stab_upload(ctx, &t.vdV, g.dV.data(), g.dV.size())) ||
        (st = stab_upload(ctx, &t.vdVgeo, g.dVgeo.data(), g.dVgeo.size())))
      return st;
  }
  return RDS_OK;
}

static rds_status set_field(rds_ctx *ctx, const double *h, double **d, bool *on)
{
  release_graph(ctx); // captured iterations change with the field's presence
  if (!h)
  {
    *on = false;
    return RDS_OK;
  }
  rds_status st;
  if (!*d && (st = stab_alloc(ctx, d, ctx->desc.nnodes)) != RDS_OK)
    return st;
  if ((st = upload(ctx, *d, h, ctx->desc.nnodes)) != RDS_OK)
    return st;
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  *on = true;
  return RDS_OK;
}

rds_status rds_set_blending_coeff(rds_ctx *ctx, const double *theta)
{
  const rds_status st = stab_check(ctx, "rds_set_blending_coeff");
  if (st != RDS_OK)
    return st;
  return set_field(ctx, theta, &ctx->d_blend, &ctx->blend_on);
}

rds_status rds_set_artificial_viscosity(rds_ctx *ctx, const double *eps)
{
  rds_status st = stab_check(ctx, "rds_set_artificial_viscosity");
  if (st != RDS_OK || (eps && (st = ensure_visc_tables(ctx)) != RDS_OK))
    return st;
  return set_field(ctx, eps, &ctx->d_av, &ctx->av_on);
}

rds_status rds_set_stab_tables(rds_ctx *ctx, int group, int nq, const double *w, const double *Vn,
                               const double *R, int nvert, const double *P1)
{
  rds_status st = stab_check(ctx, "rds_set_stab_tables");
  if (st != RDS_OK)
    return st;
  if (group < 0 || group >= (int)ctx->groups.size())
    return fail(ctx, RDS_ERR_INVALID, "rds_set_stab_tables: invalid group");
  const int ndof      = ctx->groups[group].desc.ndof;
  rds_ctx::StabTab &t = ctx->stab[group];
  if (nq < 0 || nvert < 1 || nvert > ndof || !P1 || (nq > 0 && (!w || !Vn || !R)))
    return fail(ctx, RDS_ERR_INVALID, "rds_set_stab_tables: invalid sizes or missing tables");
  if ((t.P1 && t.nvert != nvert) || (t.w && t.nq != nq))
    return fail(ctx, RDS_ERR_INVALID, "rds_set_stab_tables: table sizes differ from the first call");
  if ((!t.P1 && (st = stab_alloc(ctx, &t.P1, (size_t)ndof * nvert))) ||
      (st = upload(ctx, t.P1, P1, (size_t)ndof * nvert)))
    return st;
  t.nvert = nvert;
  if (nq > 0)
  {
    if ((!t.w && ((st = stab_alloc(ctx, &t.w, nq)) || (st = stab_alloc(ctx, &t.Vn, (size_t)nq * ndof)) ||
                  (st = stab_alloc(ctx, &t.R, (size_t)nq * ndof)))) ||
        (st = upload(ctx, t.w, w, nq)) || (st = upload(ctx, t.Vn, Vn, (size_t)nq * ndof)) ||
        (st = upload(ctx, t.R, R, (size_t)nq * ndof)))
      return st;
    t.nq = nq;
  }
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  return RDS_OK;
}

rds_status rds_set_stab_geo_tables(rds_ctx *ctx, int group, int ngeo, const double *dVgeo)
{
  rds_status st = stab_check(ctx, "rds_set_stab_geo_tables");
  if (st != RDS_OK)
    return st;
  if (group < 0 || group >= (int)ctx->groups.size())
    return fail(ctx, RDS_ERR_INVALID, "rds_set_stab_geo_tables: invalid group");
  rds_ctx::StabTab &t = ctx->stab[group];
  const int D = ctx->desc.dim;
  if (t.nq == 0 || !dVgeo || ngeo != ctx->groups[group].desc.ngeo || ngeo > kStabMaxGeo)
    return fail(ctx, RDS_ERR_INVALID, "rds_set_stab_geo_tables: no sensor rule for the group "
                                      "(rds_set_stab_tables first), or ngeo is not the group's "
                                      "(at most 4)");
  if ((!t.sdVgeo && (st = stab_alloc(ctx, &t.sdVgeo, (size_t)D * t.nq * ngeo))) ||
      (st = upload(ctx, t.sdVgeo, dVgeo, (size_t)D * t.nq * ngeo)))
    return st;
  t.sngeo = ngeo;
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  return RDS_OK;
}

rds_status rds_set_bonanni_tables(rds_ctx *ctx, int group, int nq, const double *w,
                                  const double *V, const double *dV, const double *dVgeo)
{
  rds_status st = stab_check(ctx, "rds_set_bonanni_tables");
  if (st != RDS_OK)
    return st;
  if (group < 0 || group >= (int)ctx->groups.size())
    return fail(ctx, RDS_ERR_INVALID, "rds_set_bonanni_tables: invalid group");
  const HostCellGroup &g = ctx->groups[group];
  const int D = ctx->desc.dim, ndof = g.desc.ndof, ngeo = g.desc.ngeo;
  rds_ctx::StabTab &t = ctx->stab[group];
  if (nq <= 0 || nq > 64 || !w || !V || !dV || !dVgeo || ngeo > 4)
    return fail(ctx, RDS_ERR_INVALID, "rds_set_bonanni_tables: invalid sizes or missing tables "
                                      "(straight-sided cells, at most 64 points)");
  if (t.bw && t.bnq != nq)
    return fail(ctx, RDS_ERR_INVALID, "rds_set_bonanni_tables: table sizes differ from the first call");
  if ((!t.bw && ((st = stab_alloc(ctx, &t.bw, nq)) || (st = stab_alloc(ctx, &t.bV, (size_t)nq * ndof)) ||
                 (st = stab_alloc(ctx, &t.bdV, (size_t)D * nq * ndof)) ||
                 (st = stab_alloc(ctx, &t.bdVgeo, (size_t)D * nq * ngeo)))) ||
      (st = upload(ctx, t.bw, w, nq)) || (st = upload(ctx, t.bV, V, (size_t)nq * ndof)) ||
      (st = upload(ctx, t.bdV, dV, (size_t)D * nq * ndof)) ||
      (st = upload(ctx, t.bdVgeo, dVgeo, (size_t)D * nq * ngeo)))
    return st;
  t.bnq = nq;
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  return RDS_OK;
}

rds_status rds_compute_stabilisation(rds_ctx *ctx, int op, double p0, double p1, int install,
                                     double *cells_out, double *nodes_out)
{
  rds_status st = stab_check(ctx, "rds_compute_stabilisation");
  if (st != RDS_OK)
    return st;
  const int G = (int)ctx->groups.size(), N = ctx->desc.nnodes;
  const bool sensor = op == RDS_STAB_ART_VISC || op == RDS_STAB_INDICATOR || op == RDS_STAB_BLEND_VISC;
  const bool nodal  = install || nodes_out;
  const bool bonanni = op == RDS_STAB_BLEND_BONANNI;
  if (op < RDS_STAB_ART_VISC || op > RDS_STAB_BLEND_BONANNI ||
      (op == RDS_STAB_INDICATOR && nodal))
    return fail(ctx, RDS_ERR_INVALID, "rds_compute_stabilisation: unknown operator, or a nodal "
                                      "field of the normalised indicator");
  if (G > kStabMaxGroups)
    return fail(ctx, RDS_ERR_UNSUPPORTED, "rds_compute_stabilisation: more than 8 cell groups");
  if (sensor && !(p0 > 0.0))
    return fail(ctx, RDS_ERR_INVALID, "rds_compute_stabilisation: kappa must be positive");
  if (bonanni && ctx->desc.neq != ctx->desc.dim + 2)
    return fail(ctx, RDS_ERR_UNSUPPORTED, "rds_compute_stabilisation: Bonanni's coefficient needs "
                                          "Euler physics");
  long long wc = 0, sc = 0;
  for (int k = 0; k < G; ++k)
  {
    const rds_ctx::StabTab &t = ctx->stab[k];
    if (sensor && (t.nq == 0 || (!ctx->groups[k].affine && !t.sdVgeo)))
      return fail(ctx, RDS_ERR_UNSUPPORTED, "rds_compute_stabilisation: the smoothness sensor "
                                            "needs sensor tables, and geometry tables "
                                            "(rds_set_stab_geo_tables) where cells are not "
                                            "affine simplices");
    if (nodal && t.nvert == 0)
      return fail(ctx, RDS_ERR_INVALID, "rds_compute_stabilisation: no vertex interpolant "
                                        "(rds_set_stab_tables) for a group");
    if (bonanni && t.bnq == 0)
      return fail(ctx, RDS_ERR_UNSUPPORTED, "rds_compute_stabilisation: no Bonanni tables "
                                            "(rds_set_bonanni_tables) for a group");
    wc += ctx->groups[k].desc.ncells;
    sc += (long long)ctx->groups[k].desc.ncells * ctx->groups[k].desc.ndof;
  }
  if ((!ctx->d_cellf && (st = stab_alloc(ctx, &ctx->d_cellf, wc))) ||
      (!ctx->d_nodef && (st = stab_alloc(ctx, &ctx->d_nodef, N))))
    return st;
  cudaStream_t s = ctx->stream;
  int bon_blocks = 0; // Bonanni: block sums of all groups, after the cells' lc values
  if (bonanni)
  {
    for (int k = 0; k < G; ++k)
      bon_blocks += bonanni_blocks(ctx->groups[k].desc.ncells);
    const size_t need = (size_t)wc + (size_t)bon_blocks * (ctx->desc.dim + 3) + 1;
    if (need > ctx->bon_len)
    {
      cudaFree(ctx->d_bon);
      ctx->d_bon   = nullptr;
      ctx->bon_len = 0;
      if ((st = dalloc(ctx, &ctx->d_bon, need)) != RDS_OK)
        return st;
      ctx->bon_len = need;
    }
  }
  int bon_done = 0;
  for (int k = 0; k < G; ++k)
  {
    const HostCellGroup &g    = ctx->groups[k];
    const rds_ctx::StabTab &t = ctx->stab[k];
    double *out               = ctx->d_cellf + g.ws_base;
    if (sensor)
    {
      SensorArgs a{};
      a.ncells     = g.desc.ncells;
      a.ndof       = g.desc.ndof;
      a.nq         = t.nq;
      a.order      = g.desc.order;
      a.ngeo_nodes = ctx->desc.ngeo_nodes;
      a.blend      = op == RDS_STAB_BLEND_VISC;
      a.sol_conn   = g.d_sol_conn;
      a.geo_conn   = g.d_geo_conn;
      a.X          = ctx->d_X;
      a.u          = ctx->d_u;
      a.w          = t.w;
      a.Vn         = t.Vn;
      a.R          = t.R;
      a.dVgeo      = g.affine ? nullptr : t.sdVgeo;
      a.ngeo       = t.sngeo;
      a.kappa      = p0;
      a.factor     = op == RDS_STAB_ART_VISC ? p1 : 1.0;
      a.out        = out;
      RDS_CUDA(launch_sensor(a, ctx->desc.dim, s));
    }
    else if (bonanni)
    {
      BonanniArgs a{};
      a.ncells     = g.desc.ncells;
      a.ndof       = g.desc.ndof;
      a.nq         = t.bnq;
      a.ngeo       = g.desc.ngeo;
      a.nnodes     = N;
      a.ngeo_nodes = ctx->desc.ngeo_nodes;
      a.sol_conn   = g.d_sol_conn;
      a.geo_conn   = g.d_geo_conn;
      a.X          = ctx->d_X;
      a.u          = ctx->d_u;
      a.w          = t.bw;
      a.V          = t.bV;
      a.dV         = t.bdV;
      a.dVgeo      = t.bdVgeo;
      a.gamma      = ctx->desc.gamma;
      a.f          = out;
      a.lc         = ctx->d_bon + g.ws_base;
      a.part       = ctx->d_bon + wc + (size_t)bon_done * (ctx->desc.dim + 3);
      RDS_CUDA(launch_bonanni_cells(a, ctx->desc.dim, s));
      bon_done += bonanni_blocks(g.desc.ncells);
    }
    else
      RDS_CUDA(launch_blend_cells(op == RDS_STAB_BLEND_LF ? 0 : 1, g.desc.ncells, g.desc.ndof,
                                  g.d_sol_conn, ctx->d_u, p0, out, s));
  }
  if (bonanni)
    RDS_CUDA(launch_bonanni_finish(ctx->desc.dim, bon_blocks, ctx->d_bon + wc,
                                   ctx->d_bon + wc + (size_t)bon_blocks * (ctx->desc.dim + 3),
                                   (int)wc, ctx->d_cellf, ctx->d_bon, s));
  if (op == RDS_STAB_INDICATOR)
    RDS_CUDA(launch_normalise_max((int)wc, ctx->d_cellf, s));
  if (op == RDS_STAB_BLEND_LF)
  {
    RDS_CUDA(launch_node_max(N, ctx->d_row, ctx->d_ent_ws, wc, ctx->d_cellf, ctx->d_nodef, s));
    for (int k = 0; k < G; ++k)
    {
      const HostCellGroup &g = ctx->groups[k];
      RDS_CUDA(launch_lf_finish(g.desc.ncells, g.desc.ndof, g.d_sol_conn, ctx->d_nodef,
                                ctx->d_cellf + g.ws_base, s));
    }
  }
  if (cells_out)
    RDS_CUDA(cudaMemcpyAsync(cells_out, ctx->d_cellf, wc * sizeof(double),
                             cudaMemcpyDeviceToHost, s));
  if (nodal)
  {
    double *target = ctx->d_nodef;
    if (install)
    {
      double **d = op == RDS_STAB_ART_VISC ? &ctx->d_av : &ctx->d_blend;
      if ((!*d && (st = stab_alloc(ctx, d, N))) ||
          (op == RDS_STAB_ART_VISC && (st = ensure_visc_tables(ctx))))
        return st;
      target = *d;
    }
    StabGroups sg{};
    sg.n = G;
    for (int k = 0; k < G; ++k)
    {
      const HostCellGroup &g = ctx->groups[k];
      sg.slot_base[k]        = g.slot_base;
      sg.ws_base[k]          = g.ws_base;
      sg.ncells[k]           = g.desc.ncells;
      sg.ndof[k]             = g.desc.ndof;
      sg.nvert[k]            = ctx->stab[k].nvert;
      sg.sol_conn[k]         = g.d_sol_conn;
      sg.P1[k]               = ctx->stab[k].P1;
    }
    RDS_CUDA(launch_cells_to_nodes(N, ctx->d_row, ctx->d_ent_slot, sc, sg, ctx->d_cellf, target,
                                   s));
    if (nodes_out)
      RDS_CUDA(cudaMemcpyAsync(nodes_out, target, (size_t)N * sizeof(double),
                               cudaMemcpyDeviceToHost, s));
    if (install)
    {
      release_graph(ctx);
      (op == RDS_STAB_ART_VISC ? ctx->av_on : ctx->blend_on) = true;
    }
  }
  RDS_CUDA(cudaStreamSynchronize(s));
  return RDS_OK;
}

static rds_status step_host_init(rds_ctx *ctx)
{
  if (ctx->h_in)
    return RDS_OK;
  const size_t n = (size_t)ctx->desc.nnodes * ctx->desc.neq;
  RDS_CUDA(cudaStreamCreateWithFlags(&ctx->h_in, cudaStreamNonBlocking));
  RDS_CUDA(cudaStreamCreateWithFlags(&ctx->h_out, cudaStreamNonBlocking));
  for (int k = 0; k < 2; ++k)
  {
    RDS_CUDA(cudaEventCreateWithFlags(&ctx->ev_in_ready[k], cudaEventDisableTiming));
    RDS_CUDA(cudaEventCreateWithFlags(&ctx->ev_in_free[k], cudaEventDisableTiming));
    RDS_CUDA(cudaEventCreateWithFlags(&ctx->ev_out_ready[k], cudaEventDisableTiming));
    RDS_CUDA(cudaEventCreateWithFlags(&ctx->ev_out_free[k], cudaEventDisableTiming));
    rds_status st;
    if ((st = dalloc(ctx, &ctx->d_hin[k], n)) != RDS_OK ||
        (st = dalloc(ctx, &ctx->d_hout[k], n)) != RDS_OK ||
        (st = dalloc(ctx, &ctx->d_hnorm[k], (size_t)ctx->desc.neq)) != RDS_OK)
      return st;
  }
  return RDS_OK;
}

rds_status rds_step_host(rds_ctx *ctx, const double *u_in, double *u_out, double cfl, double *norm)
{
  if (!ctx || !u_in || !u_out || !ctx->finalized || ctx->nprob > 0)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_step_host: not a finalized single context")
               : RDS_ERR_INVALID;
  rds_status st = step_host_init(ctx);
  if (st != RDS_OK)
    return st;
  const int N = ctx->desc.nnodes, NEQ = ctx->desc.neq;
  const size_t bytes = (size_t)N * NEQ * sizeof(double);
  const int k        = (int)(ctx->hstep++ & 1);
  cudaStream_t s     = ctx->stream;

  // upload
  RDS_CUDA(cudaStreamWaitEvent(ctx->h_in, ctx->ev_in_free[k], 0));
  RDS_CUDA(cudaMemcpyAsync(ctx->d_hin[k], u_in, bytes, cudaMemcpyHostToDevice, ctx->h_in));
  RDS_CUDA(cudaEventRecord(ctx->ev_in_ready[k], ctx->h_in));

  // compute: AoS staging -> SoA state, one iteration (assemble + update + norm partials)
  RDS_CUDA(cudaStreamWaitEvent(s, ctx->ev_in_ready[k], 0));
  if (NEQ == 1)
    RDS_CUDA(cudaMemcpyAsync(ctx->d_u, ctx->d_hin[k], bytes, cudaMemcpyDeviceToDevice, s));
  else if ((st = launch(ctx, [&](const char **name) {
             return launch_transpose_state(N, NEQ, ctx->d_hin[k], ctx->d_u, true, s, name);
           })) != RDS_OK)
    return st;
  RDS_CUDA(cudaEventRecord(ctx->ev_in_free[k], s));
  if ((st = rds_run(ctx, cfl, 1)) != RDS_OK)
    return st;
  st = launch(ctx, [&](const char **name) {
    return launch_norm_final(ctx->d_part, ctx->gblocks, NEQ, N, ctx->d_hnorm[k], nullptr,
                             nullptr, nullptr, 0, 0.0, nullptr, nullptr, s, name);
  });
  if (st != RDS_OK)
    return st;
  RDS_CUDA(cudaStreamWaitEvent(s, ctx->ev_out_free[k], 0));
  if (NEQ == 1)
    RDS_CUDA(cudaMemcpyAsync(ctx->d_hout[k], ctx->d_u, bytes, cudaMemcpyDeviceToDevice, s));
  else if ((st = launch(ctx, [&](const char **name) {
             return launch_transpose_state(N, NEQ, ctx->d_u, ctx->d_hout[k], false, s, name);
           })) != RDS_OK)
    return st;
  RDS_CUDA(cudaEventRecord(ctx->ev_out_ready[k], s));

  // download
  RDS_CUDA(cudaStreamWaitEvent(ctx->h_out, ctx->ev_out_ready[k], 0));
  RDS_CUDA(cudaMemcpyAsync(u_out, ctx->d_hout[k], bytes, cudaMemcpyDeviceToHost, ctx->h_out));
  if (norm)
    RDS_CUDA(cudaMemcpyAsync(norm, ctx->d_hnorm[k], NEQ * sizeof(double), cudaMemcpyDeviceToHost,
                             ctx->h_out));
  RDS_CUDA(cudaEventRecord(ctx->ev_out_free[k], ctx->h_out));
  return RDS_OK;
}

rds_status rds_step_sync(rds_ctx *ctx)
{
  if (!ctx)
    return RDS_ERR_INVALID;
  if (ctx->h_out)
    RDS_CUDA(cudaStreamSynchronize(ctx->h_out));
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  return check_status(ctx);
}

// ---- partitioned single mesh ------------------------------------------------------------

rds_status rds_set_dual_volume(rds_ctx *ctx, const double *vol)
{
  if (!ctx || !vol || !ctx->finalized)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_set_dual_volume: not finalized or null")
               : RDS_ERR_INVALID;
  const int N = ctx->desc.nnodes;
  std::vector<double> v(vol, vol + N), iv(N);
  for (int i = 0; i < N; ++i)
  {
    if (!(v[i] > 0.0))
      return fail(ctx, RDS_ERR_INVALID, "rds_set_dual_volume: non-positive volume");
    iv[i] = 1. / v[i];
  }
  rds_status st;
  if ((st = upload(ctx, ctx->d_vol, v.data(), N)) != RDS_OK ||
      (st = upload(ctx, ctx->d_inv_vol, iv.data(), N)) != RDS_OK)
    return st;
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  return RDS_OK;
}

rds_status rds_set_interface(rds_ctx *ctx, int n, const int32_t *nodes, const int32_t *slots,
                             int nslots, const uint8_t *owned)
{
  if (!ctx || !ctx->finalized || n < 0 || nslots < 0 || (n > 0 && (!nodes || !slots)) || !owned)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_set_interface: invalid arguments")
               : RDS_ERR_INVALID;
  const int N = ctx->desc.nnodes;
  for (int i = 0; i < n; ++i)
    if (nodes[i] < 0 || nodes[i] >= N || slots[i] < 0 || slots[i] >= nslots)
      return fail(ctx, RDS_ERR_INVALID, "rds_set_interface: node or slot out of range");
  cudaFree(ctx->d_if_nodes);
  cudaFree(ctx->d_if_slots);
  cudaFree(ctx->d_owned);
  ctx->d_if_nodes = ctx->d_if_slots = nullptr;
  ctx->d_owned                      = nullptr;
  rds_status st;
  if ((st = dalloc(ctx, &ctx->d_if_nodes, n)) != RDS_OK ||
      (st = dalloc(ctx, &ctx->d_if_slots, n)) != RDS_OK ||
      (st = dalloc(ctx, &ctx->d_owned, N)) != RDS_OK)
    return st;
  if ((n > 0 && ((st = upload(ctx, ctx->d_if_nodes, nodes, n)) != RDS_OK ||
                 (st = upload(ctx, ctx->d_if_slots, slots, n)) != RDS_OK)) ||
      (st = upload(ctx, ctx->d_owned, owned, N)) != RDS_OK)
    return st;
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->n_if    = n;
  ctx->n_slots = nslots;
  return RDS_OK;
}

rds_status rds_pack_interface(rds_ctx *ctx, double *buf)
{
  if (!ctx || !buf || !ctx->d_owned)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_pack_interface: rds_set_interface first")
               : RDS_ERR_INVALID;
  const int NEQ = ctx->desc.neq;
  if (ctx->n_slots == 0)
    return RDS_OK; // nothing is exchanged (one rank)
  return launch(ctx, [&](const char **name) {
    *name = "pack_interface";
    return launch_pack_interface(ctx->n_if, NEQ, ctx->desc.nnodes, ctx->d_if_nodes,
                                 ctx->d_if_slots, ctx->d_res, ctx->d_ws, buf,
                                 (size_t)ctx->n_slots * (NEQ + 1), ctx->stream);
  });
}

rds_status rds_unpack_interface(rds_ctx *ctx, const double *buf)
{
  if (!ctx || !buf || !ctx->d_owned)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_unpack_interface: rds_set_interface first")
               : RDS_ERR_INVALID;
  return launch(ctx, [&](const char **name) {
    *name = "unpack_interface";
    return launch_unpack_interface(ctx->n_if, ctx->desc.neq, ctx->desc.nnodes, ctx->d_if_nodes,
                                   ctx->d_if_slots, buf, ctx->d_res, ctx->d_ws, ctx->stream);
  });
}

rds_status rds_finish(rds_ctx *ctx, double cfl, int update, double *sq)
{
  if (ctx && !sq)
    return fail(ctx, RDS_ERR_INVALID, "rds_finish: sq is null");
  if (ctx)
    ctx->part_used = 0;
  return rds_finish_nodes(ctx, cfl, update, 0, ctx ? ctx->desc.nnodes : 0, sq);
}

rds_status rds_gather_finish(rds_ctx *ctx, int v0, int v1, double cfl, double *sq)
{
  if (!ctx || !ctx->finalized)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "not finalized") : RDS_ERR_INVALID;
  if (v0 < 0 || v1 < v0 || v1 > ctx->desc.nnodes)
    return fail(ctx, RDS_ERR_INVALID, "rds_gather_finish: node range out of bounds");
  ctx->part_used = 0;
  if (v1 == v0)
    return RDS_OK;
  GatherArgs ga = gather_args(ctx, cfl, ctx->d_zero);
  ga.vbeg       = v0;
  ga.vend       = v1;
  ga.sq_out     = sq;
  ga.counter    = ctx->d_counter; // last-block-done (with sq)
  const int nb  = (v1 - v0 + kGBlock - 1) / kGBlock;
  // sums, dt, update, block sums of (res dt)^2; with sq, also their sum (last block)
  const rds_status st = launch(ctx, [&](const char **name) {
    return launch_gather(ga, sq ? 15 : 7, nb, ctx->stream, name);
  });
  if (st == RDS_OK && !sq)
    ctx->part_used = nb;
  return st;
}

rds_status rds_finish_nodes(rds_ctx *ctx, double cfl, int update, int v0, int v1, double *sq)
{
  if (!ctx || !ctx->d_owned)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_finish: rds_set_interface first")
               : RDS_ERR_INVALID;
  if (v0 < 0 || v1 < v0 || v1 > ctx->desc.nnodes)
    return fail(ctx, RDS_ERR_INVALID, "rds_finish_nodes: node range out of bounds");
  const int off  = ctx->part_used;
  ctx->part_used = 0;
  return launch(ctx, [&](const char **name) {
    *name = "finish_nodes";
    return launch_finish(v0, v1, ctx->desc.nnodes, ctx->desc.neq, cfl, update, ctx->d_vol,
                         ctx->d_ws, ctx->d_res, ctx->d_dt, ctx->d_u, ctx->d_owned, ctx->d_part,
                         off, ctx->d_counter, sq, ctx->stream);
  });
}

static rds_status rk_buffers(rds_ctx *ctx)
{
  rds_status st;
  const size_t n = (size_t)ctx->desc.nnodes * ctx->desc.neq;
  for (double **p : {&ctx->d_rk_u1, &ctx->d_rk_u2, &ctx->d_rk_res})
    if (!*p && (st = dalloc(ctx, p, n)) != RDS_OK)
      return st;
  return RDS_OK;
}

// RK3TVD stage coefficients (solver/time/ExplicitTimeStepper.cpp:66-100)
static void rk_coeffs(int k, double &ca, double &cb, double &cc)
{
  ca = k == 2 ? 3. / 4. : 1. / 3.;
  cb = k == 2 ? 1. / 4. : 2. / 3;
  cc = k == 2 ? 1. / 4. : 2. / 3.;
}

rds_status rds_rk_stage_state(rds_ctx *ctx, int stage)
{
  if (!ctx || !ctx->finalized || stage < 0 || stage > 3)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_rk_stage_state: stage 0-3 of a finalized context")
               : RDS_ERR_INVALID;
  rds_status st = rk_buffers(ctx);
  if (st != RDS_OK)
    return st;
  if (ctx->rk_stage == 0)
  {
    ctx->rk_base_u   = ctx->d_u;
    ctx->rk_base_res = ctx->d_res;
  }
  ctx->d_u      = stage <= 1 ? ctx->rk_base_u : stage == 2 ? ctx->d_rk_u1 : ctx->d_rk_u2;
  ctx->d_res    = stage <= 1 ? ctx->rk_base_res : ctx->d_rk_res;
  ctx->rk_stage = stage;
  return RDS_OK;
}

rds_status rds_gather_rk(rds_ctx *ctx, int v0, int v1, double cfl)
{
  if (!ctx || !ctx->finalized || ctx->rk_stage == 0)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_gather_rk: select a stage (rds_rk_stage_state)")
               : RDS_ERR_INVALID;
  if (v0 < 0 || v1 < v0 || v1 > ctx->desc.nnodes)
    return fail(ctx, RDS_ERR_INVALID, "rds_gather_rk: node range out of bounds");
  if (v1 == v0)
    return RDS_OK;
  const int k   = ctx->rk_stage;
  GatherArgs ga = gather_args(ctx, k == 1 ? cfl : 0.0, ctx->d_zero);
  ga.vbeg       = v0;
  ga.vend       = v1;
  ga.rk_first   = k == 1;
  ga.rk_un      = ctx->rk_base_u;
  ga.rk_us      = ctx->d_u;
  ga.rk_out     = k == 1 ? ctx->d_rk_u1 : k == 2 ? ctx->d_rk_u2 : ctx->rk_base_u;
  rk_coeffs(k, ga.rk_ca, ga.rk_cb, ga.rk_cc);
  const int nb = (v1 - v0 + kGBlock - 1) / kGBlock;
  return launch(ctx, [&](const char **name) {
    return launch_gather(ga, k == 1 ? 17 : 16, nb, ctx->stream, name);
  });
}

rds_status rds_combine_rk(rds_ctx *ctx, int v0, int v1, double cfl)
{
  if (!ctx || !ctx->finalized || ctx->rk_stage == 0)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_combine_rk: select a stage (rds_rk_stage_state)")
               : RDS_ERR_INVALID;
  if (v0 < 0 || v1 < v0 || v1 > ctx->desc.nnodes)
    return fail(ctx, RDS_ERR_INVALID, "rds_combine_rk: node range out of bounds");
  const int k = ctx->rk_stage;
  double ca, cb, cc;
  rk_coeffs(k, ca, cb, cc);
  double *out = k == 1 ? ctx->d_rk_u1 : k == 2 ? ctx->d_rk_u2 : ctx->rk_base_u;
  return launch(ctx, [&](const char **name) {
    *name = "rk_combine";
    return launch_rk_combine(v0, v1, ctx->desc.nnodes, ctx->desc.neq, k == 1, cfl, ca, cb, cc,
                             ctx->d_vol, ctx->d_ws, ctx->d_res, ctx->d_dt, ctx->rk_base_u,
                             ctx->d_u, out, ctx->stream);
  });
}

rds_status rds_check(rds_ctx *ctx)
{
  if (!ctx)
    return RDS_ERR_INVALID;
  return check_status(ctx);
}

rds_status rds_get_fields(rds_ctx *ctx, double *res, double *dt, double *ws, double *vol)
{
  if (!ctx || !ctx->finalized)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "not finalized") : RDS_ERR_INVALID;
  const int N = ctx->desc.nnodes;
  rds_status st;
  if (res && (st = get_soa(ctx, ctx->d_res, res, ctx->desc.neq)) != RDS_OK)
    return st;
  if (dt)
    RDS_CUDA(cudaMemcpyAsync(dt, ctx->d_dt, N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (ws)
    RDS_CUDA(cudaMemcpyAsync(ws, ctx->d_ws, N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (vol)
    RDS_CUDA(cudaMemcpyAsync(vol, ctx->d_vol, N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  return check_status(ctx);
}

// One fused iteration: cell + facet kernels, gather with time step, update and norm partials,
// final norm with the stop test. All launches honour the device stop flag.
static rds_status enqueue_iteration(rds_ctx *ctx, double cfl, int max_iter, double drop)
{
  rds_status st = launch_residual_kernels(ctx, ctx->d_stop);
  if (st != RDS_OK)
    return st;
  // gather + dt + update + norm, with the final reduction and stop test done by the last block
  GatherArgs ga = gather_args(ctx, cfl, ctx->d_stop);
  ga.pdl        = (ctx->loop_pdl && !ctx->timing) ? 1 : 0;
  ga.counter    = ctx->d_counter;
  ga.norm       = ctx->d_norm;
  ga.norm0      = ctx->d_norm0;
  ga.hist       = ctx->d_hist;
  ga.iter       = ctx->d_iter;
  ga.max_iter   = max_iter;
  ga.drop       = drop;
  ga.stop_w     = ctx->d_stop;
  ga.status     = ctx->d_status;
  ga.loop       = ctx->d_loop;
  ga.stall      = ctx->d_stall;
  return launch(ctx, [&](const char **name) {
    return launch_gather(ga, 15, ctx->gblocks, ctx->stream, name);
  });
}

// The loop parameters to the device: from a pinned host copy, and only when they changed, so the
// per-step paths (rds_run, rds_step_host) issue no copy (a copy from pageable memory, like a
// stack variable, lets the driver synchronise with the stream). Not inside a stream capture.
extern "C++" static rds_status set_loop_params(rds_ctx *ctx, const LoopParams &lp)
{
  if (ctx->loop_set && std::memcmp(&ctx->loop_last, &lp, sizeof(LoopParams)) == 0)
    return RDS_OK;
  if (!ctx->h_loop)
  {
    RDS_CUDA(cudaMallocHost((void **)&ctx->h_loop, sizeof(LoopParams)));
    RDS_CUDA(cudaEventCreateWithFlags(&ctx->ev_loop, cudaEventDisableTiming));
  }
  else
    RDS_CUDA(cudaEventSynchronize(ctx->ev_loop)); // the previous copy has read the buffer
  *ctx->h_loop = lp;
  RDS_CUDA(cudaMemcpyAsync(ctx->d_loop, ctx->h_loop, sizeof(LoopParams), cudaMemcpyHostToDevice,
                           ctx->stream));
  RDS_CUDA(cudaEventRecord(ctx->ev_loop, ctx->stream));
  ctx->loop_last = lp;
  ctx->loop_set  = true;
  return RDS_OK;
}

// Captures `count` iterations (enqueued by `one`) into graph slot gi once; later calls reuse
// it.
extern "C++" template <typename F>
rds_status capture_graph(rds_ctx *ctx, int gi, int count, F &&one)
{
  if (ctx->graph_exec[gi])
    return RDS_OK;
  rds_status st;
  cudaGraph_t graph = nullptr;
  RDS_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  const long long l0 = ctx->launches;
  for (int k = 0; k < count; ++k)
  {
    st = one();
    if (st != RDS_OK)
    {
      cudaStreamEndCapture(ctx->stream, &graph);
      if (graph)
        cudaGraphDestroy(graph);
      return st;
    }
  }
  ctx->launches = l0; // launches are counted when the graph runs
  RDS_CUDA(cudaStreamEndCapture(ctx->stream, &graph));
  cudaError_t e = cudaGraphInstantiate(&ctx->graph_exec[gi], graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess)
  {
    ctx->graph_exec[gi] = nullptr;
    return fail(ctx, RDS_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  }
  return RDS_OK;
}

extern "C++" template <typename F>
rds_status capture_chunk(rds_ctx *ctx, int gi, F &&one)
{
  return capture_graph(ctx, gi, rds_ctx::kChunk, one);
}

// Replays graph slot gi up to nchunks times, polling the device stop flag every 4 chunks
// (chunks enqueued after the stop exit at once).
static rds_status replay_chunks(rds_ctx *ctx, int gi, int nchunks, long long launches_per_chunk)
{
  for (int k = 0; k < nchunks; ++k)
  {
    RDS_CUDA(cudaGraphLaunch(ctx->graph_exec[gi], ctx->stream));
    ctx->launches += launches_per_chunk;
    if (k + 1 < nchunks && (k % 4) == 3)
    {
      RDS_CUDA(cudaMemcpyAsync(ctx->h_stop, ctx->d_stop, sizeof(int), cudaMemcpyDeviceToHost,
                               ctx->stream));
      RDS_CUDA(cudaStreamSynchronize(ctx->stream));
      if (*ctx->h_stop)
        break;
    }
  }
  return RDS_OK;
}

// Device loop at the active precision: chunks of `chunk` fused iterations captured once in a
// CUDA graph and replayed until the device stop flag is raised (drop reached, iteration cap,
// non-finite norm); the host polls the flag every 4 chunks.
static rds_status run_loop(rds_ctx *ctx, double cfl, int max_iter, double drop)
{
  rds_status st;
  LoopParams lp{};
  lp.cfl      = cfl;
  lp.drop     = drop;
  lp.sw       = ctx->mixed_switch;
  lp.max_iter   = max_iter;
  lp.stall      = ctx->active_precision == RDS_MIXED ? 1 : 0;
  lp.stall_min  = ctx->stall_min;
  lp.stall_mult = ctx->stall_mult;
  if ((st = set_loop_params(ctx, lp)) != RDS_OK)
    return st;
  if (ctx->timing)
  {
    // event timing wants plain launches: run the loop without a graph
    for (int it = 0; it < max_iter; ++it)
      if ((st = enqueue_iteration(ctx, cfl, max_iter, drop)) != RDS_OK)
        return st;
    return RDS_OK;
  }
  const int gi    = ctx->active_precision == RDS_MIXED ? 1 : 0;
  const int chunk = rds_ctx::kChunk;
  if ((st = capture_chunk(ctx, gi, [&] { return enqueue_iteration(ctx, cfl, max_iter, drop); })) !=
      RDS_OK)
    return st;
  const long long per_iter = (long long)ctx->groups.size() + (long long)ctx->bcs.size() + 1;
  return replay_chunks(ctx, gi, (max_iter + chunk - 1) / chunk, per_iter * chunk);
}

// One sweep of the defect-correction loop (mixed form, scalar physics): exact = the fused FP64
// iteration whose gather also keeps its update dt res, dt / V and the state it started from,
// with its norm and stop test; otherwise a correction sweep: the FP32 change of each cell's
// contribution since then (rds_cells_scalar_dc.cu), each facet's FP64 contribution at the
// current state minus its exact-sweep value, written as FP32, and u -= dt res + (dt / V) sum.
static rds_status enqueue_dc_sweep(rds_ctx *ctx, bool exact, double cfl, int max_iter,
                                   double drop)
{
  ctx->dc_phase = exact ? 1 : 2;
  rds_status st = launch_residual_kernels(ctx, ctx->d_stop);
  ctx->dc_phase = 0;
  if (st != RDS_OK)
    return st;
  GatherArgs ga = gather_args(ctx, cfl, ctx->d_stop);
  ga.c32        = ctx->d_c32;
  ga.dres       = ctx->d_dres;
  ga.dtv        = ctx->d_dtv;
  ga.ur         = ctx->d_ur;
  ga.loop       = ctx->d_loop;
  ga.pdl        = (ctx->loop_pdl && !ctx->timing) ? 1 : 0;
  if (exact)
  {
    ga.counter  = ctx->d_counter;
    ga.norm     = ctx->d_norm;
    ga.norm0    = ctx->d_norm0;
    ga.hist     = ctx->d_hist;
    ga.iter     = ctx->d_iter;
    ga.max_iter = max_iter;
    ga.drop     = drop;
    ga.stop_w   = ctx->d_stop;
    ga.status   = ctx->d_status;
    ga.stall    = ctx->d_stall;
  }
  return launch(ctx, [&](const char **name) {
    return launch_gather(ga, exact ? 18 : 19, ctx->gblocks, ctx->stream, name);
  });
}

// Whether a cycle's correction sweeps run as one launch (dc_sweeps_fused): a single context
// with one triangle group of at most dc_fuse_cells cells and weak Dirichlet conditions only.
static bool dc_fused_ok(rds_ctx *ctx)
{
  if (ctx->nprob > 0 || ctx->groups.size() != 1 || ctx->bcs.size() > (size_t)kFuseMaxBC ||
      ctx->no_bcs || ctx->grp_beg != 0 || ctx->grp_end >= 0 || !ctx->d_fbar ||
      (long long)ctx->groups[0].desc.ncells > ctx->dc_fuse_cells)
    return false;
  const HostBC *bcs[kFuseMaxBC];
  for (size_t k = 0; k < ctx->bcs.size(); ++k)
    bcs[k] = &ctx->bcs[k];
  return dc_fused_supported(ctx->groups[0], bcs, (int)ctx->bcs.size());
}

// `nsweeps` correction sweeps in one launch (after an exact sweep; see dc_sweeps_fused).
static rds_status enqueue_dc_fused(rds_ctx *ctx, int nsweeps)
{
  DcFusedArgs fa{};
  fa.cell = dc_cell_args(ctx, 0, ctx->d_stop);
  const HostBC *bcs[kFuseMaxBC];
  fa.nbc = (int)ctx->bcs.size();
  for (int k = 0; k < fa.nbc; ++k)
  {
    bcs[k]       = &ctx->bcs[k];
    fa.bc[k]     = bc_args(ctx, ctx->bcs[k], ctx->d_stop);
    fa.bc[k].c32 = ctx->d_c32;
  }
  fa.ga            = gather_args(ctx, 0.0, ctx->d_stop);
  fa.ga.c32        = ctx->d_c32;
  fa.ga.dres       = ctx->d_dres;
  fa.ga.dtv        = ctx->d_dtv;
  fa.ga.ur         = ctx->d_ur;
  fa.nsweeps       = nsweeps;
  fa.bar           = ctx->d_fbar;
  fa.status        = ctx->d_status;
  fa.wait_limit    = ctx->fuse_test_wait > 0 ? ctx->fuse_test_wait : 1 << 22;
  fa.test_extra    = ctx->fuse_test_wait > 0 ? 1 : 0;
  return launch(ctx, [&](const char **name) {
    bool ok             = false;
    const cudaError_t e = launch_dc_fused(ctx->groups[0], bcs, fa, ctx->stream, name, &ok);
    return ok ? e : cudaErrorNotSupported;
  });
}

// Defect-correction loop of the mixed form: cycles of one exact FP64 sweep and dc_m - 1 FP32
// correction sweeps (one launch for all of them on small meshes, dc_fused_ok), captured once (graph slot 6, several cycles per graph) and replayed until
// an exact sweep raises the stop flag. The stop test sees only exact FP64 norms, and the fixed
// point is the FP64 scheme's: at convergence the correction is zero and R64 = 0.
static rds_status run_loop_dc(rds_ctx *ctx, double cfl, int max_iter, double drop)
{
  rds_status st;
  const int m = ctx->dc_m;
  LoopParams lp{};
  lp.cfl      = cfl;
  lp.drop     = drop;
  lp.max_iter = max_iter;
  lp.dc_m     = m;
  if ((st = set_loop_params(ctx, lp)) != RDS_OK)
    return st;
  ctx->active_precision = RDS_FP64;
  const bool fused      = m > 1 && dc_fused_ok(ctx);
  if (ctx->timing)
  {
    for (int it = 0; it < max_iter; ++it)
    {
      if (fused && it % m == 1)
      {
        // the rest of the cycle in one launch (its sweeps end at max_iter at the latest)
        const int n = std::min(m - 1, max_iter - it);
        if ((st = enqueue_dc_fused(ctx, n)) != RDS_OK)
          return st;
        it += n - 1;
        continue;
      }
      if ((st = enqueue_dc_sweep(ctx, it % m == 0, cfl, max_iter, drop)) != RDS_OK)
        return st;
    }
    return RDS_OK;
  }
  const int cycles = std::max(1, 32 / m); // sweeps per graph launch: cycles x m
  auto cycle       = [&]() -> rds_status {
    for (int j = 0; j < m; ++j)
    {
      if (fused && j == 1)
        return enqueue_dc_fused(ctx, m - 1);
      const rds_status s2 = enqueue_dc_sweep(ctx, j == 0, cfl, max_iter, drop);
      if (s2 != RDS_OK)
        return s2;
    }
    return RDS_OK;
  };
  if ((st = capture_graph(ctx, 6, cycles, cycle)) != RDS_OK)
    return st;
  const long long per_sweep = (long long)ctx->groups.size() + (long long)ctx->bcs.size() + 1;
  const int per_graph       = cycles * m;
  const long long per_launch =
      fused ? (long long)cycles * (per_sweep + 1) : per_sweep * per_graph;
  return replay_chunks(ctx, 6, (max_iter + per_graph - 1) / per_graph, per_launch);
}

rds_status rds_iterate(rds_ctx *ctx, double cfl, int max_iter, double drop, int *it_done,
                       double *hist)
{
  if (!ctx || !ctx->finalized || max_iter <= 0)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_iterate: not finalized or max_iter <= 0")
               : RDS_ERR_INVALID;
  const int NEQ = ctx->desc.neq;
  rds_status st;
  if (max_iter > ctx->hist_cap)
  {
    if (ctx->d_hist)
      cudaFree(ctx->d_hist);
    ctx->d_hist = nullptr;
    if ((st = dalloc(ctx, &ctx->d_hist, (size_t)max_iter * NEQ)) != RDS_OK)
      return st;
    ctx->hist_cap = max_iter;
    release_graph(ctx);
  }
  RDS_CUDA(cudaMemsetAsync(ctx->d_iter, 0, sizeof(int), ctx->stream));
  RDS_CUDA(cudaMemsetAsync(ctx->d_stop, 0, sizeof(int), ctx->stream));
  RDS_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(unsigned), ctx->stream));

  if (ctx->desc.precision == RDS_MIXED && ctx->dc_ok && !ctx->blend_on && !ctx->av_on)
  {
    // mixed form, scalar physics: defect-correction loop (exact FP64 sweep every dc_m sweeps)
    if ((st = run_loop_dc(ctx, cfl, max_iter, drop)) != RDS_OK)
      return st;
  }
  else if (ctx->desc.precision == RDS_MIXED)
  {
    // mixed form: FP32 cell kernels until the relative residual reaches mixed_switch, then a
    // final FP64 phase of pseudo-time sweeps from that state to the requested drop; the
    // iteration counter, the initial norm and the history continue across the switch
    ctx->active_precision = RDS_MIXED;
    const double drop1    = std::max(drop, ctx->mixed_switch);
    if ((st = run_loop(ctx, cfl, max_iter, drop1)) != RDS_OK)
      return st;
    int done1 = 0;
    unsigned status1 = 0;
    RDS_CUDA(cudaMemcpyAsync(&done1, ctx->d_iter, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    RDS_CUDA(cudaMemcpyAsync(&status1, ctx->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost,
                             ctx->stream));
    RDS_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->active_precision = RDS_FP64;
    if (done1 < max_iter && status1 == 0)
    {
      RDS_CUDA(cudaMemsetAsync(ctx->d_stop, 0, sizeof(int), ctx->stream));
      if ((st = run_loop(ctx, cfl, max_iter, drop)) != RDS_OK)
        return st;
    }
  }
  else
  {
    ctx->active_precision = RDS_FP64;
    if ((st = run_loop(ctx, cfl, max_iter, drop)) != RDS_OK)
      return st;
  }
  ctx->active_precision = ctx->desc.precision;
  int done = 0;
  RDS_CUDA(cudaMemcpyAsync(&done, ctx->d_iter, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  if (it_done)
    *it_done = done;
  if (hist && done > 0)
  {
    RDS_CUDA(cudaMemcpy(hist, ctx->d_hist, (size_t)done * NEQ * sizeof(double),
                        cudaMemcpyDeviceToHost));
  }
  st = check_status(ctx);
  if (st != RDS_OK)
    return st;
  if (drop > 0.0)
  {
    std::vector<double> h((size_t)NEQ * 2);
    RDS_CUDA(cudaMemcpy(h.data(), ctx->d_norm, NEQ * sizeof(double), cudaMemcpyDeviceToHost));
    RDS_CUDA(cudaMemcpy(h.data() + NEQ, ctx->d_norm0, NEQ * sizeof(double), cudaMemcpyDeviceToHost));
    double rel = 0.0;
    for (int e = 0; e < NEQ; ++e)
      rel = std::max(rel, h[NEQ + e] > 0 ? h[e] / h[NEQ + e] : 0.0);
    if (rel > drop)
      return fail(ctx, RDS_ERR_ITER_CAP, "residual drop not reached within max_iter");
  }
  return RDS_OK;
}

rds_status rds_run(rds_ctx *ctx, double cfl, int n)
{
  if (!ctx || !ctx->finalized || n <= 0)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_run: not finalized or n <= 0") : RDS_ERR_INVALID;
  // plain launches (event timing, if enabled, brackets each kernel); the stop flag stays 0
  rds_status st;
  if (!ctx->d_hist)
  {
    if ((st = dalloc(ctx, &ctx->d_hist, (size_t)ctx->desc.neq)) != RDS_OK)
      return st;
    ctx->hist_cap = 1;
  }
  auto one = [&]() -> rds_status {
    rds_status s2 = launch_residual_kernels(ctx, ctx->d_zero);
    if (s2 != RDS_OK)
      return s2;
    GatherArgs ga = gather_args(ctx, cfl, ctx->d_zero);
    ga.loop       = ctx->d_loop;
    return launch(ctx, [&](const char **name) {
      return launch_gather(ga, 7, ctx->gblocks, ctx->stream, name);
    });
  };
  LoopParams lp{};
  lp.cfl = cfl;
  if ((st = set_loop_params(ctx, lp)) != RDS_OK)
    return st;
  if (ctx->timing)
  {
    for (int i = 0; i < n; ++i)
      if ((st = one()) != RDS_OK)
        return st;
    return RDS_OK;
  }
  // one iteration captured once (graph slot 3) and replayed n times: the launch sequence of an
  // iteration costs one graph launch
  const int gi = ctx->active_precision == RDS_MIXED ? 4 : 3;
  if ((st = capture_graph(ctx, gi, 1, one)) != RDS_OK)
    return st;
  const long long per_iter = (long long)ctx->groups.size() + (long long)ctx->bcs.size() + 1;
  for (int i = 0; i < n; ++i)
  {
    RDS_CUDA(cudaGraphLaunch(ctx->graph_exec[gi], ctx->stream));
    ctx->launches += per_iter;
  }
  return RDS_OK;
}

// One step of the third-order TVD Runge-Kutta stepper (solver/time/ExplicitTimeStepper.cpp:
// 66-100): the residual, wave speed and dt at u_n, then two more residual passes at the stage
// states u_1 and u_2 with the dt of the first. Each gather ends in the stage combination, so a
// stage costs one pass over the nodes. The later stages run the cell and boundary kernels on
// the stage state and write their residual to a separate buffer, the way the reference's
// stepper points the solver's solution and residuals at u_1 / u_2 and res_tmp; the first
// stage's residual and dt stay in the context for the norm.
static rds_status enqueue_rk3tvd(rds_ctx *ctx, double cfl)
{
  double *const u = ctx->d_u, *const res = ctx->d_res;
  auto stage = [&](int k) -> rds_status {
    rds_status st = launch_residual_kernels(ctx, ctx->d_zero);
    if (st != RDS_OK)
      return st;
    GatherArgs ga = gather_args(ctx, k == 1 ? cfl : 0.0, ctx->d_zero);
    ga.rk_first   = k == 1;
    ga.rk_un      = u;
    ga.rk_us      = ctx->d_u;
    ga.rk_out     = k == 1 ? ctx->d_rk_u1 : k == 2 ? ctx->d_rk_u2 : u;
    ga.rk_ca      = k == 2 ? 3. / 4. : 1. / 3.;
    ga.rk_cb      = k == 2 ? 1. / 4. : 2. / 3;
    ga.rk_cc      = k == 2 ? 1. / 4. : 2. / 3.;
    return launch(ctx, [&](const char **name) {
      return launch_gather(ga, k == 1 ? 17 : 16, ctx->gblocks, ctx->stream, name);
    });
  };
  rds_status st = stage(1);
  if (st == RDS_OK)
  {
    ctx->d_u   = ctx->d_rk_u1;
    ctx->d_res = ctx->d_rk_res;
    st         = stage(2);
  }
  if (st == RDS_OK)
  {
    ctx->d_u = ctx->d_rk_u2;
    st       = stage(3);
  }
  ctx->d_u   = u;
  ctx->d_res = res;
  return st;
}

// One Runge-Kutta stage of a batched RK3TVD step (enqueue_batch_iteration's gather ends in the
// stage combination instead of the update, norm and stop test)
struct RkStage
{
  int k;                  // 1, 2, 3
  const double *un, *us;  // u_n and the stage state
  double *out;            // u_1, u_2 or u_n+1
  double ca, cb, cc;
};

static rds_status enqueue_batch_iteration(rds_ctx *ctx, bool mixed, int dc = 0,
                                          const RkStage *rk = nullptr);

// One RK3TVD step of every problem of a batched context (the stages of enqueue_rk3tvd over the
// batch's persistent kernels, each problem with its own CFL).
static rds_status enqueue_rk3tvd_batch(rds_ctx *ctx)
{
  double *const u = ctx->d_u, *const res = ctx->d_res;
  auto stage = [&](int k) -> rds_status {
    RkStage rk{};
    rk.k   = k;
    rk.un  = u;
    rk.us  = ctx->d_u;
    rk.out = k == 1 ? ctx->d_rk_u1 : k == 2 ? ctx->d_rk_u2 : u;
    rk.ca  = k == 2 ? 3. / 4. : 1. / 3.;
    rk.cb  = k == 2 ? 1. / 4. : 2. / 3;
    rk.cc  = k == 2 ? 1. / 4. : 2. / 3.;
    return enqueue_batch_iteration(ctx, false, 0, &rk);
  };
  rds_status st = stage(1);
  if (st == RDS_OK)
  {
    ctx->d_u   = ctx->d_rk_u1;
    ctx->d_res = ctx->d_rk_res;
    st         = stage(2);
  }
  if (st == RDS_OK)
  {
    ctx->d_u = ctx->d_rk_u2;
    st       = stage(3);
  }
  ctx->d_u   = u;
  ctx->d_res = res;
  return st;
}

rds_status rds_advance_rk3tvd(rds_ctx *ctx, double cfl, int nsteps)
{
  if (!ctx || !ctx->finalized || nsteps <= 0)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_advance_rk3tvd: not finalized or nsteps <= 0")
               : RDS_ERR_INVALID;
  if (ctx->d_if_nodes)
    return fail(ctx, RDS_ERR_UNSUPPORTED,
                "rds_advance_rk3tvd: not in partitioned contexts");
  const bool batched = ctx->nprob > 0;
  // the stages run the FP64 cell kernels in every context (a mixed context's time steps equal
  // an FP64 context's)
  struct Fp64Stages
  {
    rds_ctx *c;
    int saved;
    ~Fp64Stages() { c->active_precision = saved; }
  } fp64{ctx, ctx->active_precision};
  ctx->active_precision = RDS_FP64;
  rds_status st;
  const size_t n = (size_t)ctx->desc.nnodes * ctx->desc.neq;
  for (double **p : {&ctx->d_rk_u1, &ctx->d_rk_u2, &ctx->d_rk_res})
    if (!*p && (st = dalloc(ctx, p, n)) != RDS_OK)
      return st;
  if (batched)
  {
    // every problem takes part (phase 1: FP64 cells; rds_iterate_batch resets the phases)
    const std::vector<int32_t> ph(ctx->nprob, 1);
    const int32_t one = 1;
    if ((st = upload(ctx, ctx->d_phase, ph.data(), ctx->nprob)) ||
        (st = upload(ctx, ctx->d_changed, &one, 1)))
      return st;
    RDS_CUDA(cudaMemsetAsync(ctx->d_stop, 0, sizeof(int), ctx->stream));
  }
  auto step = [&]() { return batched ? enqueue_rk3tvd_batch(ctx) : enqueue_rk3tvd(ctx, cfl); };
  if (ctx->timing)
  {
    for (int i = 0; i < nsteps; ++i)
      if ((st = step()) != RDS_OK)
        return st;
    return RDS_OK;
  }
  // one step captured once (graph slot 5, recaptured when the CFL changes; batched contexts use
  // their problems' own CFLs) and replayed
  const int gi = 5;
  if (ctx->graph_exec[gi] && !batched && ctx->rk_cfl != cfl)
  {
    cudaGraphExecDestroy(ctx->graph_exec[gi]);
    ctx->graph_exec[gi] = nullptr;
  }
  ctx->rk_cfl = cfl;
  if ((st = capture_graph(ctx, gi, 1, step)) != RDS_OK)
    return st;
  const long long per_step = 3 * ((long long)ctx->groups.size() + (long long)ctx->bcs.size() +
                                  (batched ? 2 : 1));
  for (int i = 0; i < nsteps; ++i)
  {
    RDS_CUDA(cudaGraphLaunch(ctx->graph_exec[gi], ctx->stream));
    ctx->launches += per_step;
  }
  return RDS_OK;
}

rds_status rds_set_option(rds_ctx *ctx, const char *key, double value)
{
  if (!ctx || !key)
    return RDS_ERR_INVALID;
  if (std::strcmp(key, "mixed_switch") == 0)
  {
    if (!(value > 0.0 && value < 1.0))
      return fail(ctx, RDS_ERR_INVALID, "mixed_switch must be in (0, 1)");
    ctx->mixed_switch = value;
    return RDS_OK;
  }
  if (std::strcmp(key, "tc_test_wait") == 0)
  {
    // test of the tensor-core kernel's bounded wait: each CTA first waits up to `value` tries on
    // a barrier nothing completes, so the call reports the timeout (0: off)
    if (!(value >= 0.0 && value <= 1048576.0))
      return fail(ctx, RDS_ERR_INVALID, "tc_test_wait must be in [0, 2^20]");
    ctx->tc_test_wait = (int)value;
    release_graph(ctx);
    return RDS_OK;
  }
  if (std::strcmp(key, "tensor_cores") == 0)
  {
    ctx->use_tc = value != 0.0;
    release_graph(ctx); // captured loops hold the previous choice
    return RDS_OK;
  }
  if (std::strcmp(key, "loop_pdl") == 0)
  {
    // programmatic dependent launch of the iteration's main-stream kernels (0 / 1)
    ctx->loop_pdl = value != 0.0 ? 1 : 0;
    release_graph(ctx);
    return RDS_OK;
  }
  if (std::strcmp(key, "mixed_refresh") == 0)
  {
    // defect-correction loop: an exact FP64 sweep every `value` sweeps
    if (!(value >= 1.0 && value <= 1024.0))
      return fail(ctx, RDS_ERR_INVALID, "mixed_refresh must be in [1, 1024]");
    if ((int)value != ctx->dc_m)
      for (int gi : {2, 6}) // the captured cycles hold the previous period
        if (ctx->graph_exec[gi])
        {
          cudaGraphExecDestroy(ctx->graph_exec[gi]);
          ctx->graph_exec[gi] = nullptr;
        }
    ctx->dc_m = (int)value;
    return RDS_OK;
  }
  if (std::strcmp(key, "fuse_test_wait") == 0)
  {
    // test of the fused sweeps' bounded barrier wait: > 0 makes every barrier of the next
    // fused launches wait for one arrival more than the grid has and give up after `value`
    // polls (the call then reports RDS_ERR_CUDA); 0 restores the normal barrier
    if (!(value >= 0.0 && value <= 1.0e6))
      return fail(ctx, RDS_ERR_INVALID, "fuse_test_wait must be in [0, 1e6]");
    ctx->fuse_test_wait = (int)value;
    for (int gi : {2, 6})
      if (ctx->graph_exec[gi])
      {
        cudaGraphExecDestroy(ctx->graph_exec[gi]);
        ctx->graph_exec[gi] = nullptr;
      }
    return RDS_OK;
  }
  if (std::strcmp(key, "mixed_fuse_cells") == 0)
  {
    // defect-correction loop: one launch for a cycle's correction sweeps on meshes of at most
    // `value` cells (0: one launch per kernel and sweep)
    if (!(value >= 0.0 && value <= 2.0e9))
      return fail(ctx, RDS_ERR_INVALID, "mixed_fuse_cells must be in [0, 2e9]");
    ctx->dc_fuse_cells = (long long)value;
    for (int gi : {2, 6})
      if (ctx->graph_exec[gi])
      {
        cudaGraphExecDestroy(ctx->graph_exec[gi]);
        ctx->graph_exec[gi] = nullptr;
      }
    return RDS_OK;
  }
  if (std::strcmp(key, "mixed_stall_min") == 0)
  {
    if (!(value >= 1.0 && value <= 2.0e9))
      return fail(ctx, RDS_ERR_INVALID, "mixed_stall_min must be in [1, 2e9]");
    ctx->stall_min = (int)value;
    return RDS_OK;
  }
  if (std::strcmp(key, "mixed_stall_mult") == 0)
  {
    if (!(value >= 0.0 && value <= 1.0e6))
      return fail(ctx, RDS_ERR_INVALID, "mixed_stall_mult must be in [0, 1e6]");
    ctx->stall_mult = value;
    return RDS_OK;
  }
  return fail(ctx, RDS_ERR_INVALID, std::string("unknown option ") + key);
}

rds_status rds_kernel_timing(rds_ctx *ctx, int enable)
{
  if (!ctx)
    return RDS_ERR_INVALID;
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  for (TimingRec &r : ctx->trecs)
  {
    ctx->ev_pool.push_back(r.a);
    ctx->ev_pool.push_back(r.b);
  }
  ctx->trecs.clear();
  ctx->timing = enable != 0;
  return RDS_OK;
}

int rds_kernel_times(rds_ctx *ctx, char (*names)[32], double *ms, int *launches, int max)
{
  if (!ctx)
    return 0;
  cudaStreamSynchronize(ctx->stream);
  std::vector<std::string> order;
  std::map<std::string, std::pair<double, int>> acc;
  for (TimingRec &r : ctx->trecs)
  {
    float t = 0.f;
    cudaEventElapsedTime(&t, r.a, r.b);
    if (!acc.count(r.name))
      order.push_back(r.name);
    acc[r.name].first += t;
    acc[r.name].second += 1;
  }
  int n = 0;
  for (const std::string &k : order)
  {
    if (n >= max)
      break;
    std::snprintf(names[n], 32, "%s", k.c_str());
    ms[n]       = acc[k].first;
    launches[n] = acc[k].second;
    ++n;
  }
  return n;
}

// ---- batched independent problems -----------------------------------------------------------

rds_status rds_set_problems(rds_ctx *ctx, int nproblems, const int32_t *node_offsets,
                            const double *cfl)
{
  if (!ctx)
    return RDS_ERR_INVALID;
  if (ctx->finalized || !ctx->groups.empty() || !ctx->bcs.empty() || ctx->nprob > 0)
    return fail(ctx, RDS_ERR_INVALID,
                "rds_set_problems: call once, before adding cell groups and conditions");
  if (ctx->desc.physics != RDS_ADVECTION_CONST && ctx->desc.physics != RDS_BURGERS2D)
    return fail(ctx, RDS_ERR_UNSUPPORTED, "batched problems: scalar 2D physics only");
  if (nproblems <= 0 || !node_offsets || !cfl || node_offsets[0] != 0 ||
      node_offsets[nproblems] != ctx->desc.nnodes)
    return fail(ctx, RDS_ERR_INVALID,
                "rds_set_problems: node offsets must run from 0 to nnodes over nproblems ranges");
  for (int p = 0; p < nproblems; ++p)
    if (node_offsets[p + 1] <= node_offsets[p] || !(cfl[p] > 0.0) || !std::isfinite(cfl[p]))
      return fail(ctx, RDS_ERR_INVALID, "rds_set_problems: problem " + std::to_string(p) +
                                            " has an empty node range or a CFL <= 0");
  ctx->nprob = nproblems;
  ctx->prob_nodes.assign(node_offsets, node_offsets + nproblems + 1);
  ctx->prob_cfl.assign(cfl, cfl + nproblems);
  return RDS_OK;
}

rds_status rds_add_batch_cell_group(rds_ctx *ctx, const rds_cell_group *g, int physics,
                                    int scheme, const int32_t *problem_cells)
{
  if (!ctx || !g)
    return RDS_ERR_INVALID;
  const int P = ctx->nprob;
  if (P == 0)
    return fail(ctx, RDS_ERR_INVALID, "rds_add_batch_cell_group: rds_set_problems first");
  if (physics != RDS_ADVECTION_CONST && physics != RDS_BURGERS2D)
    return fail(ctx, RDS_ERR_UNSUPPORTED, "batched problems: scalar 2D physics only");
  if (scheme < RDS_PGLDA || scheme > RDS_PGPSI || !problem_cells || !g->sol_conn ||
      g->ncells <= 0 || g->ndof <= 0 || problem_cells[0] != 0 || problem_cells[P] != g->ncells)
    return fail(ctx, RDS_ERR_INVALID,
                "rds_add_batch_cell_group: invalid scheme or problem cell offsets");
  if (scheme == RDS_PGPSI && ctx->desc.precision != RDS_FP64)
    return fail(ctx, RDS_ERR_UNSUPPORTED, "rds_add_batch_cell_group: the PSI scheme in FP64 "
                                          "contexts only");
  for (int p = 0; p < P; ++p)
  {
    if (problem_cells[p + 1] < problem_cells[p])
      return fail(ctx, RDS_ERR_INVALID, "rds_add_batch_cell_group: decreasing cell offsets");
    const int v0 = ctx->prob_nodes[p], v1 = ctx->prob_nodes[p + 1];
    for (size_t i = (size_t)problem_cells[p] * g->ndof; i < (size_t)problem_cells[p + 1] * g->ndof;
         ++i)
      if (g->sol_conn[i] < v0 || g->sol_conn[i] >= v1)
        return fail(ctx, RDS_ERR_INVALID, "rds_add_batch_cell_group: a cell of problem " +
                                              std::to_string(p) + " has a node of another problem");
  }
  const rds_status st = rds_add_cell_group(ctx, g);
  if (st != RDS_OK)
    return st;
  HostCellGroup &h = ctx->groups.back();
  h.physics        = physics;
  h.scheme         = scheme;
  h.pcells.assign(problem_cells, problem_cells + P + 1);
  return RDS_OK;
}

rds_status rds_add_batch_bc(rds_ctx *ctx, const rds_bc_group *b, int physics)
{
  if (!ctx)
    return RDS_ERR_INVALID;
  if (ctx->nprob == 0)
    return fail(ctx, RDS_ERR_INVALID, "rds_add_batch_bc: rds_set_problems first");
  if (physics != RDS_ADVECTION_CONST && physics != RDS_BURGERS2D)
    return fail(ctx, RDS_ERR_UNSUPPORTED, "batched problems: scalar 2D physics only");
  if (b && b->kind == RDS_BC_STRONG_DIRICHLET)
    return fail(ctx, RDS_ERR_UNSUPPORTED, "batched problems: weak boundary conditions only");
  const rds_status st = rds_add_bc(ctx, b);
  if (st == RDS_OK)
    ctx->bcs.back().physics = physics;
  return st;
}

// One batched iteration: rebuild of the active lists (only after a phase change), boundary
// facets of all problems on the side stream, persistent cell kernels over the active tiles of
// each group (FP32 tiles and FP64 tiles in the mixed form), persistent gather with the
// per-problem update, norm and stop test.
// dc: 0 plain iteration (FP32 tiles of the problems in phase 0 when mixed, FP64 tiles of those
// in phase 1); 1 exact sweep of the defect-correction loop (FP64 cells of every active problem,
// blending coefficients kept for the corrections); 2 correction sweep (FP32 cell changes).
static rds_status enqueue_batch_iteration(rds_ctx *ctx, bool mixed, int dc, const RkStage *rk)
{
  const rds_desc &d = ctx->desc;
  const int P = ctx->nprob, G = (int)ctx->groups.size();
  RebuildArgs r{};
  r.nprob       = P;
  r.ngroups     = G;
  r.phase       = ctx->d_phase;
  r.cbeg        = ctx->d_cbeg;
  r.cend        = ctx->d_cend;
  r.tile        = ctx->d_tile;
  r.tile_prefix = ctx->d_tile_prefix;
  r.node_off    = ctx->d_node_off;
  r.nb_prefix   = ctx->d_nb_prefix;
  r.changed     = ctx->d_changed;
  r.stop        = ctx->d_stop;
  rds_status st = launch(ctx, [&](const char **name) {
    return launch_batch_rebuild(r, ctx->stream, name);
  });
  if (st != RDS_OK)
    return st;
  const bool fork = !ctx->bcs.empty();
  if (fork && (st = fork_sides(ctx)) != RDS_OK)
    return st;
  for (size_t k = 0; k < ctx->bcs.size(); ++k)
  {
    const HostBC &b       = ctx->bcs[k];
    const cudaStream_t sk = side_stream(ctx, (int)k);
    BCArgs a              = bc_args(ctx, b, ctx->d_stop);
    if (dc == 2)
      a.c32 = ctx->d_c32; // the change since the exact sweep, in FP32
    if ((st = launch_on(ctx, sk, [&](const char **name) {
           return launch_bc(b, a, b.physics, d.dim, d.neq, sk, name);
         })) != RDS_OK)
      return st;
  }
  for (int gi = 0; gi < G; ++gi)
  {
    const HostCellGroup &g = ctx->groups[gi];
    if (dc == 2)
    {
      // correction sweep over the same active tiles as the exact sweep (phase 1)
      DcCellArgs da{};
      da.ncells     = g.desc.ncells;
      da.sol_conn   = g.d_sol_conn;
      da.geo_conn   = g.d_geo_conn;
      da.X          = ctx->d_X;
      da.ngeo_nodes = d.ngeo_nodes;
      da.u          = ctx->d_u;
      da.ur         = ctx->d_ur;
      da.c32        = ctx->d_c32;
      da.slot_base  = g.slot_base;
      da.theta      = ctx->d_dc_theta + ctx->dc_cell_base[gi];
      da.adv0       = d.adv[0];
      da.adv1       = d.adv[1];
      da.stop       = ctx->d_stop;
      da.bt         = {ctx->d_tile_prefix + ((size_t)gi * 2 + 1) * (P + 1), g.d_cbeg, g.d_cend, P};
      const int grid = g.tune_grid[1] > 0 ? g.tune_grid[1] : 4 * ctx->nsm;
      if ((st = launch(ctx, [&](const char **name) {
             bool ok             = false;
             const cudaError_t e = launch_cells_scalar_dc(g, da, grid, g.tune_tile[1],
                                                          ctx->stream, name, &ok);
             return ok ? e : cudaErrorNotSupported;
           })) != RDS_OK)
        return st;
      continue;
    }
    for (int ph = (mixed && dc == 0) ? 0 : 1; ph < 2; ++ph)
    {
      CellArgs a = cell_args(ctx, g, ctx->d_stop);
      a.bt       = {ctx->d_tile_prefix + ((size_t)gi * 2 + ph) * (P + 1), g.d_cbeg, g.d_cend, P};
      if (dc == 1 && g.scheme == RDS_PGB)
        a.theta = ctx->d_dc_theta + ctx->dc_cell_base[gi];
      const int grid = g.tune_grid[ph] > 0 ? g.tune_grid[ph] : 4 * ctx->nsm;
      const bool tc  = ph == 0 && ctx->use_tc && g.d_tc;
      if ((st = launch(ctx, [&](const char **name) {
             bool ok = false;
             cudaError_t e =
                 tc ? launch_cells_scalar_tc(g, a, true, grid, 0, ctx->stream, name, &ok)
                    : launch_cells_scalar_batch(g, a, ph == 0 ? RDS_MIXED : RDS_FP64, grid,
                                                g.tune_tile[ph], ctx->stream, name, &ok);
             return ok ? e : cudaErrorNotSupported;
           })) != RDS_OK)
        return st;
    }
  }
  if (fork && (st = join_sides(ctx)) != RDS_OK)
    return st;
  GatherArgs ga = gather_args(ctx, 0.0, ctx->d_stop);
  ga.status     = ctx->d_status;
  ga.loop       = ctx->d_loop;
  ga.c32        = ctx->d_c32;
  ga.dres       = ctx->d_dres;
  ga.dtv        = ctx->d_dtv;
  ga.ur         = ctx->d_ur;
  if (rk)
  {
    ga.rk_first = rk->k == 1;
    ga.rk_un    = rk->un;
    ga.rk_us    = rk->us;
    ga.rk_out   = rk->out;
    ga.rk_ca    = rk->ca;
    ga.rk_cb    = rk->cb;
    ga.rk_cc    = rk->cc;
  }
  BatchArgs b{};
  b.nprob     = P;
  b.node_off  = ctx->d_node_off;
  b.nb_base   = ctx->d_nb_base;
  b.nb_prefix = ctx->d_nb_prefix;
  b.cfl       = ctx->d_pcfl;
  b.pcount    = ctx->d_pcount;
  b.phase     = ctx->d_phase;
  b.iter      = ctx->d_piter;
  b.norm      = ctx->d_pnorm;
  b.norm0     = ctx->d_pnorm0;
  b.pstatus   = ctx->d_pstatus;
  b.changed   = ctx->d_changed;
  b.loop      = ctx->d_loop;
  b.stall     = ctx->d_pstall;
  return launch(ctx, [&](const char **name) {
    return launch_gather_batch(ga, b, ctx->batch_grid, ctx->stream, name, dc,
                               rk ? (rk->k == 1 ? 1 : 2) : 0);
  });
}

rds_status rds_iterate_batch(rds_ctx *ctx, int max_iter, double drop, int32_t *iters,
                             double *rel)
{
  if (!ctx || !ctx->finalized || ctx->nprob == 0 || max_iter <= 0)
    return ctx ? fail(ctx, RDS_ERR_INVALID,
                      "rds_iterate_batch: not a finalized batched context or max_iter <= 0")
               : RDS_ERR_INVALID;
  const int P = ctx->nprob, NEQ = ctx->desc.neq;
  const bool mixed = ctx->desc.precision == RDS_MIXED;
  // mixed form, scalar physics: the defect-correction loop, every problem in step with the
  // single-problem loop (exact FP64 sweep at sweeps 0, m, 2m, ..., FP32 corrections between)
  const bool dc    = mixed && ctx->dc_ok;
  const int m      = dc ? ctx->dc_m : 1;
  rds_status st;
  LoopParams lp{};
  lp.drop     = drop;
  lp.sw         = ctx->mixed_switch;
  lp.max_iter   = max_iter;
  lp.stall_min  = ctx->stall_min;
  lp.stall_mult = ctx->stall_mult;
  lp.dc_m       = dc ? m : 0;
  if ((st = set_loop_params(ctx, lp)) != RDS_OK)
    return st;
  const std::vector<int32_t> phase0(P, (mixed && !dc) ? 0 : 1);
  const int32_t one = 1;
  if ((st = upload(ctx, ctx->d_phase, phase0.data(), P)) ||
      (st = upload(ctx, ctx->d_changed, &one, 1)))
    return st;
  RDS_CUDA(cudaMemsetAsync(ctx->d_piter, 0, P * sizeof(int32_t), ctx->stream));
  RDS_CUDA(cudaMemsetAsync(ctx->d_pcount, 0, P * sizeof(unsigned), ctx->stream));
  RDS_CUDA(cudaMemsetAsync(ctx->d_pstatus, 0, P * sizeof(unsigned), ctx->stream));
  RDS_CUDA(cudaMemsetAsync(ctx->d_stop, 0, sizeof(int), ctx->stream));
  RDS_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(unsigned), ctx->stream));
  // every problem is done after max_iter iterations; one more raises the stop flag
  const int total_iter = max_iter + 1;
  if (dc)
  {
    const long long per_sweep = 2 + (long long)ctx->bcs.size() + (long long)ctx->groups.size();
    if (ctx->timing)
    {
      for (int it = 0; it < total_iter; ++it)
        if ((st = enqueue_batch_iteration(ctx, mixed, it % m == 0 ? 1 : 2)) != RDS_OK)
          return st;
    }
    else
    {
      const int cycles = std::max(1, 32 / m);
      auto cycle       = [&]() -> rds_status {
        for (int j = 0; j < m; ++j)
        {
          const rds_status s2 = enqueue_batch_iteration(ctx, mixed, j == 0 ? 1 : 2);
          if (s2 != RDS_OK)
            return s2;
        }
        return RDS_OK;
      };
      if ((st = capture_graph(ctx, 2, cycles, cycle)) != RDS_OK)
        return st;
      const int per_graph = cycles * m;
      if ((st = replay_chunks(ctx, 2, (total_iter + per_graph - 1) / per_graph,
                              per_sweep * per_graph)) != RDS_OK)
        return st;
    }
  }
  else if (ctx->timing)
  {
    for (int it = 0; it < total_iter; ++it)
      if ((st = enqueue_batch_iteration(ctx, mixed)) != RDS_OK)
        return st;
  }
  else
  {
    if ((st = capture_chunk(ctx, 2, [&] { return enqueue_batch_iteration(ctx, mixed); })) !=
        RDS_OK)
      return st;
    const long long per_iter =
        2 + (long long)ctx->bcs.size() + (long long)ctx->groups.size() * (mixed ? 2 : 1);
    if ((st = replay_chunks(ctx, 2, (total_iter + rds_ctx::kChunk - 1) / rds_ctx::kChunk,
                            per_iter * rds_ctx::kChunk)) != RDS_OK)
      return st;
  }
  std::vector<int32_t> it(P);
  std::vector<double> nrm((size_t)P * NEQ), nrm0((size_t)P * NEQ);
  std::vector<unsigned> pst(P);
  RDS_CUDA(cudaMemcpyAsync(it.data(), ctx->d_piter, P * sizeof(int32_t), cudaMemcpyDeviceToHost,
                           ctx->stream));
  RDS_CUDA(cudaMemcpyAsync(nrm.data(), ctx->d_pnorm, nrm.size() * sizeof(double),
                           cudaMemcpyDeviceToHost, ctx->stream));
  RDS_CUDA(cudaMemcpyAsync(nrm0.data(), ctx->d_pnorm0, nrm0.size() * sizeof(double),
                           cudaMemcpyDeviceToHost, ctx->stream));
  RDS_CUDA(cudaMemcpyAsync(pst.data(), ctx->d_pstatus, P * sizeof(unsigned),
                           cudaMemcpyDeviceToHost, ctx->stream));
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  int nonfinite = 0, capped = 0;
  for (int p = 0; p < P; ++p)
  {
    double r = 0.0;
    for (int e = 0; e < NEQ; ++e)
    {
      const double n0 = nrm0[(size_t)p * NEQ + e];
      const double x  = n0 > 0.0 ? nrm[(size_t)p * NEQ + e] / n0 : 0.0;
      if (!(x <= r)) // a NaN drop stays NaN in rel
        r = x;
    }
    if (iters)
      iters[p] = it[p];
    if (rel)
      rel[p] = r;
    nonfinite += (pst[p] & kFlagNonFinite) != 0;
    capped += (drop > 0.0 && !(r <= drop));
  }
  if (nonfinite)
    return fail(ctx, RDS_ERR_NONFINITE,
                std::to_string(nonfinite) + " problem(s) with a non-finite residual norm");
  if ((st = check_status(ctx)) != RDS_OK)
    return st;
  if (capped)
    return fail(ctx, RDS_ERR_ITER_CAP,
                std::to_string(capped) + " problem(s) did not reach the drop within max_iter");
  return RDS_OK;
}

// Autotuner: for every group and cell precision of the batch, time the persistent cell kernel
// over all problems for tiles of 64 / 128 cells per CTA and 1..16 resident CTAs per SM,
// and keep the fastest (tile, grid). Results per cell do not depend on the choice.
rds_status rds_autotune(rds_ctx *ctx, char *report, int len)
{
  if (!ctx || !ctx->finalized || ctx->nprob == 0)
    return ctx ? fail(ctx, RDS_ERR_INVALID, "rds_autotune: not a finalized batched context")
               : RDS_ERR_INVALID;
  static const int kTiles[] = {64, 128};
  static const int kPerSm[] = {1, 2, 3, 4, 5, 6, 8, 12, 16}; // capped at the kernel's occupancy
  const int P = ctx->nprob;
  const bool mixed = ctx->desc.precision == RDS_MIXED;
  rds_status st;
  int32_t *d_pre = nullptr;
  if ((st = dalloc(ctx, &d_pre, P + 1)) != RDS_OK)
    return st;
  ctx->extra.push_back(d_pre);
  cudaEvent_t e0 = get_event(ctx), e1 = get_event(ctx);
  std::string rep = "[";
  for (size_t gi = 0; gi < ctx->groups.size(); ++gi)
  {
    HostCellGroup &g = ctx->groups[gi];
    for (int ph = mixed ? 0 : 1; ph < 2; ++ph)
    {
      float best = 1e30f;
      int best_tile = 128, best_grid = 4 * ctx->nsm;
      const char *kname = "?";
      const bool tc     = ph == 0 && ctx->use_tc && g.d_tc; // tensor-core kernel: 128-cell tiles
      for (int tile : kTiles)
      {
        if (tc && tile != 128)
          continue;
        std::vector<int32_t> pre(P + 1, 0);
        for (int p = 0; p < P; ++p)
          pre[p + 1] = pre[p] + (g.pcells[p + 1] - g.pcells[p] + tile - 1) / tile;
        if ((st = upload(ctx, d_pre, pre.data(), P + 1)) != RDS_OK)
          return st;
        int last_grid = -1;
        for (int per_sm : kPerSm)
        {
          const int grid = std::max(1, std::min(per_sm * ctx->nsm, pre[P]));
          if (grid == last_grid)
            continue;
          last_grid  = grid;
          CellArgs a = cell_args(ctx, g, ctx->d_zero);
          a.bt       = {d_pre, g.d_cbeg, g.d_cend, P};
          const int prec = ph == 0 ? RDS_MIXED : RDS_FP64;
          bool ok        = false;
          for (int rep_i = 0; rep_i < 4; ++rep_i)
          {
            if (rep_i == 1)
              RDS_CUDA(cudaEventRecord(e0, ctx->stream));
            if (tc)
              RDS_CUDA(launch_cells_scalar_tc(g, a, true, grid, 0, ctx->stream, &kname, &ok));
            else
              RDS_CUDA(
                  launch_cells_scalar_batch(g, a, prec, grid, tile, ctx->stream, &kname, &ok));
            if (!ok)
              return fail(ctx, RDS_ERR_UNSUPPORTED,
                          "rds_autotune: no batched kernel for this cell group");
          }
          RDS_CUDA(cudaEventRecord(e1, ctx->stream));
          RDS_CUDA(cudaEventSynchronize(e1));
          float ms = 0.f;
          RDS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
          ms /= 3.f;
          if (ms < best)
          {
            best      = ms;
            best_tile = tile;
            best_grid = grid;
          }
        }
      }
      g.tune_tile[ph] = best_tile;
      g.tune_grid[ph] = best_grid;
      char buf[256];
      snprintf(buf, sizeof buf,
               "%s{\"group\": %zu, \"kernel\": \"%s\", \"ndof\": %d, \"nq\": %d, \"tile\": %d, "
               "\"grid\": %d, \"ms\": %.4f}",
               rep.size() > 1 ? ", " : "", gi, kname, g.desc.ndof, g.desc.nq, best_tile,
               best_grid, best);
      rep += buf;
    }
  }
  rep += "]";
  ctx->ev_pool.push_back(e0);
  ctx->ev_pool.push_back(e1);
  std::vector<int32_t> tile(ctx->groups.size() * 2);
  for (size_t gi = 0; gi < ctx->groups.size(); ++gi)
  {
    tile[gi * 2]     = ctx->groups[gi].tune_tile[0];
    tile[gi * 2 + 1] = ctx->groups[gi].tune_tile[1];
  }
  if ((st = upload(ctx, ctx->d_tile, tile.data(), tile.size())) != RDS_OK)
    return st;
  RDS_CUDA(cudaStreamSynchronize(ctx->stream));
  release_graph(ctx); // the captured batch loop holds the old grids
  ctx->tuned       = true;
  ctx->tune_report = rep;
  if (report && len > 0)
  {
    strncpy(report, rep.c_str(), (size_t)len - 1);
    report[len - 1] = '\0';
  }
  return RDS_OK;
}

rds_status rds_destroy(rds_ctx *ctx)
{
  if (!ctx)
    return RDS_OK;
  if (ctx->stream)
    cudaStreamSynchronize(ctx->stream);
  if (ctx->side)
    cudaStreamSynchronize(ctx->side);
  for (int k = 1; k < rds_ctx::kMaxSides; ++k)
    if (ctx->sides[k])
      cudaStreamSynchronize(ctx->sides[k]);
  release_graph(ctx);
  for (HostCellGroup &g : ctx->groups)
  {
    cudaFree(g.d_sol_conn);
    cudaFree(g.d_geo_conn);
  }
  for (HostBC &b : ctx->bcs)
  {
    cudaFree(b.d_sol_conn);
    cudaFree(b.d_geo_conn);
    cudaFree(b.d_gq);
  }
  cudaFree(ctx->d_bon);
  if (ctx->h_loop)
    cudaFreeHost(ctx->h_loop);
  if (ctx->ev_loop)
    cudaEventDestroy(ctx->ev_loop);
  cudaFree(ctx->d_if_nodes);
  cudaFree(ctx->d_if_slots);
  cudaFree(ctx->d_owned);
  cudaFree(ctx->d_jp_brow);
  cudaFree(ctx->d_jp_cnr);
  cudaFree(ctx->d_jp_cptr);
  cudaFree(ctx->d_jp_coff);
  cudaFree(ctx->d_jp_jac);
  cudaFree(ctx->d_theta);
  if (ctx->h_out)
    cudaStreamSynchronize(ctx->h_out);
  if (ctx->h_in)
    cudaStreamSynchronize(ctx->h_in);
  for (int k = 0; k < 2; ++k)
  {
    cudaFree(ctx->d_hin[k]);
    cudaFree(ctx->d_hout[k]);
    cudaFree(ctx->d_hnorm[k]);
    for (cudaEvent_t e : {ctx->ev_in_ready[k], ctx->ev_in_free[k], ctx->ev_out_ready[k],
                          ctx->ev_out_free[k]})
      if (e)
        cudaEventDestroy(e);
  }
  if (ctx->h_in)
    cudaStreamDestroy(ctx->h_in);
  if (ctx->h_out)
    cudaStreamDestroy(ctx->h_out);
  void *bufs[] = {ctx->d_X,     ctx->d_u,     ctx->d_res,     ctx->d_ws,       ctx->d_dt,
                  ctx->d_vol,   ctx->d_inv_vol, ctx->d_contrib, ctx->d_wsc,    ctx->d_stage,
                  ctx->d_row,   ctx->d_ent_slot, ctx->d_ent_ws, ctx->d_part,   ctx->d_norm,
                  ctx->d_norm0, ctx->d_hist,  ctx->d_iter,    ctx->d_stop,     ctx->d_zero,
                  ctx->d_status, ctx->d_counter, ctx->d_loop, ctx->d_rk_u1, ctx->d_rk_u2,
                  ctx->d_rk_res};
  for (void *p : ctx->extra)
    cudaFree(p);
  for (void *p : bufs)
    if (p)
      cudaFree(p);
  if (ctx->h_stop)
    cudaFreeHost(ctx->h_stop);
  for (TimingRec &r : ctx->trecs)
  {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (cudaEvent_t e : ctx->ev_pool)
    cudaEventDestroy(e);
  if (ctx->ev_fork)
    cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join)
    cudaEventDestroy(ctx->ev_join);
  if (ctx->side)
    cudaStreamDestroy(ctx->side);
  for (int k = 1; k < rds_ctx::kMaxSides; ++k)
  {
    if (ctx->sides[k])
      cudaStreamDestroy(ctx->sides[k]);
    if (ctx->ev_joins[k])
      cudaEventDestroy(ctx->ev_joins[k]);
  }
  if (ctx->own_stream && ctx->stream)
    cudaStreamDestroy(ctx->stream);
  delete ctx;
  return RDS_OK;
}

} // extern "C"
