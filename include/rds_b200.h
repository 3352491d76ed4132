/* rds_b200 -- B200 (sm_100a) implementation of pdekit's explicit continuous
 * residual-distribution (RDS) cell-residual + pseudo-time update path.
 *
 * C ABI: plain pointers and sizes, no exceptions, every call returns an rds_status.
 * Host arrays are owned by the caller and copied in/out; the context owns all device memory.
 * Nodal fields cross the ABI in the reference's AoS layout [node][neq]
 * (interpolation::VectorMeshFunction, src/interpolation/mesh_function/VectorMeshFunction.hpp:210-248);
 * the device keeps them as SoA [neq][node].
 *
 * Entry point -> reference interface it replaces (file:line in martinv/pdekit):
 *   rds_create / rds_add_cell_group / rds_finalize
 *       RDMethod::configure_mesh_data + initialize_work_data
 *       (src/solver/rdm/RDMethod.hpp:60-67,159-207; PGRDMethodExplicit.hpp:232-299)
 *   rds_add_bc            RDMethod::add_boundary_condition + set_expression
 *       (src/solver/rdm/RDMethod.hpp:230-243; bc/RDMBCBase.hpp:112-114)
 *   rds_set_state / rds_get_state
 *       set_vec_function(SolverVecFn::solution, ...) (src/solver/rdm/PGRDMethodExplicit.hpp:324-358)
 *   rds_assemble          PGRDMethodExplicit::assemble_lhs_and_rhs(CFL) (PGRDMethodExplicit.hpp:417-423)
 *   rds_assemble_rhs      PGRDMethodExplicit::assemble_rhs() (PGRDMethodExplicit.hpp:428-463)
 *   rds_update            PGRDMethodExplicit::solve() (PGRDMethodExplicit.hpp:468-477)
 *   rds_residual_norm     PGRDMethodExplicit::compute_residual_norm (PGRDMethodExplicit.hpp:482-514)
 *   rds_get_fields        residual / time-step / wave-speed / dual-volume mesh functions
 *       (RDMethod::vec_function, scal_function(SolverScalFn::time_step), RDTimeUpdate.hpp:30-40)
 *   rds_iterate           the examples' loop "assemble_lhs_and_rhs(CFL); solve()" run to a residual drop
 *       (examples/testcases-rdm/Advection-Continuous-RDS-2D-Explicit.cpp:133-174;
 *        src/solver/time/ExplicitTimeStepper.cpp:36-40)
 */
#ifndef RDS_B200_H
#define RDS_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define RDS_API __attribute__((visibility("default")))
#else
#define RDS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rds_ctx rds_ctx;

typedef enum
{
  RDS_OK                 = 0,
  RDS_ERR_INVALID        = 1, /* invalid descriptor / argument / call order */
  RDS_ERR_CUDA           = 2, /* CUDA runtime failure (message in rds_last_error) */
  RDS_ERR_NONFINITE      = 3, /* NaN/Inf in the residual or state */
  RDS_ERR_NEG_PRESSURE   = 4, /* non-positive pressure met (Euler) */
  RDS_ERR_ITER_CAP       = 5, /* rds_iterate reached max_iter without the requested drop */
  RDS_ERR_UNSUPPORTED    = 6, /* configuration not compiled into this library */
  RDS_ERR_TOO_LARGE      = 7  /* size above a documented limit */
} rds_status;

/* Physics: template argument of PGRDMethodExplicit<MeshConfig, Physics, Scheme>. */
typedef enum
{
  RDS_ADVECTION_CONST = 0, /* physics::RotationAdvection2D with a constant direction policy */
  RDS_BURGERS2D       = 1, /* physics::Burgers2D (src/physics/scalar/Burgers2D.hpp) */
  RDS_EULER2D         = 2, /* physics::Euler2DCons (src/physics/euler/Euler2DCons.hpp) */
  RDS_EULER3D         = 3  /* physics::Euler3DCons (src/physics/euler/Euler3DCons.hpp) */
} rds_physics;

/* Scheme: SchemeTraits tag (src/solver/rdm/cellsplitters/PGLDA.hpp:24, PGN.hpp:24, PGB.hpp:24). */
typedef enum
{
  RDS_PGLDA = 0,
  RDS_PGN   = 1,
  RDS_PGB   = 2,
  /* PSI: the N scheme's node residuals phi_n limited per cell with the reference's residual
   * limiter (solver/rdm/cellsplitters/LFResidualLimiter.hpp:37-110): where |phi| > 1e-14,
   * x_n = max(phi_n / phi, 0) + 1e-12 and phi_n <- x_n / sum x * phi (phi the cell residual).
   * The reference applies that limiter only to its Lax-Friedrichs schemes and has no PSI
   * scheme: this one has no reference to be pinned on. Scalar physics (the reference's limiter
   * is empty for systems), FP64 contexts, single and batched; no element Jacobians. */
  RDS_PGPSI = 3
} rds_scheme;

typedef enum
{
  RDS_FP64  = 0, /* plain path: FP64 everywhere (parity with the reference CPU path) */
  RDS_MIXED = 1  /* FP32 interpolation/flux/upwind arithmetic, FP64 accumulation, inverse and norms */
} rds_precision;

/* Element shapes, numbered as the reference's ElemShape (src/common/Constants.hpp:29-40). */
typedef enum
{
  RDS_LINE  = 2,
  RDS_TRIAG = 3,
  RDS_QUAD  = 4,
  RDS_TETRA = 10
} rds_shape;

typedef enum
{
  RDS_BC_WEAK_DIRICHLET  = 0, /* bc/WeakDirichletBC.hpp: gq = boundary state */
  RDS_BC_WEAK_WALL       = 1, /* bc/WeakWall.hpp (Euler) */
  RDS_BC_WEAK_SUB_INLET  = 2, /* bc/WeakSubInlet.hpp (Euler): params = total temperature, pressure */
  RDS_BC_WEAK_SUB_OUTLET = 3, /* bc/WeakSubOutlet.hpp (Euler): params[0] = outlet pressure */
  RDS_BC_WEAK_FARFIELD   = 4, /* bc/WeakFarfield.hpp:125-240 (Euler): gq = [neq] reference state
                               * (conservative variables, set_reference_state) */
  RDS_BC_STRONG_DIRICHLET = 5 /* bc/StrongDirichletBC.hpp:202-233: gq = [nfacets][nfdof][neq]
                               * values the facet dofs take, facet by facet (a dof on two facets
                               * keeps the later value); only sol_conn / nfacets / nfdof are
                               * read besides. Applied in condition order after the cells (the
                               * conditions added after it see the new state); the update then
                               * moves these dofs by -dt res like every other dof. Not in
                               * batched contexts. */,
  RDS_BC_WEAK_SUPER_INLET = 6, /* bc/WeakSuperInlet.hpp:62-160 (Euler): no residual, only the
                                * facet's wave speed (max eigenvalue magnitude on the facet) */
  RDS_BC_WEAK_SYMMETRY    = 7  /* bc/WeakSymmetry.hpp:100-190 (Euler): K-(n) (u_mirror - u), the
                                * mirror state with the momentum reflected about the facet */
} rds_bc_kind;

typedef struct
{
  int physics;   /* rds_physics */
  int scheme;    /* rds_scheme */
  int precision; /* rds_precision */
  int dim;       /* 2 or 3 */
  int neq;       /* 1 (scalar), 4 (Euler 2D), 5 (Euler 3D) */
  int nnodes;    /* number of solution nodes (dofs) */
  int ngeo_nodes;
  const double *geo_coords; /* [ngeo_nodes][dim] */
  double adv[3];            /* RDS_ADVECTION_CONST: advection direction */
  double gamma;             /* Euler: ratio of specific heats (1.4) */
} rds_desc;

/* One element type: connectivity and reference-element tables as the reference's FEValues /
 * FluxSpaceMetric hold them (src/interpolation/FEValues.hpp:45-114,
 * src/interpolation/FluxSpaceMetric.hpp:237-456). Row-major; derivative tables stacked
 * [dim][rows][cols]. */
typedef struct
{
  int shape;   /* rds_shape */
  int order;   /* solution polynomial order p */
  int ncells;
  int ndof;    /* solution dofs per cell */
  int ngeo;    /* geometry nodes per cell */
  int nq;      /* quadrature points */
  int nfl;     /* flux nodes (Lagrange order p+1) */
  const int32_t *sol_conn; /* [ncells][ndof], reference local dof order */
  const int32_t *geo_conn; /* [ncells][ngeo] */
  const double *w;     /* [nq]             quadrature weights */
  const double *V;     /* [nq][ndof]       solution basis at quadrature points */
  const double *dV;    /* [dim][nq][ndof]  reference derivatives of the solution basis */
  const double *dVgeo; /* [dim][nq][ngeo]  reference derivatives of the geometry basis */
  const double *dVf;   /* [dim][nq][nfl]   reference derivatives of the flux basis */
  const double *Vsf;   /* [nfl][ndof]      solution basis at the flux nodes */
  /* Optional rule for the dual (cell) volumes, sum_q wv_q detJ_q: the reference uses the Gauss
   * rule of the cell's own polynomial order (src/solver/rdm/RDTimeUpdate.hpp:85-150). nqv = 0
   * uses the rule above. */
  int nqv;
  const double *wv;      /* [nqv] */
  const double *dVgeo_v; /* [dim][nqv][ngeo] */
} rds_cell_group;

/* One weak boundary condition on a set of boundary facets, traversed in the given order
 * (src/solver/rdm/bc/WeakBC.hpp:227-360). 'gq' is the boundary state g(x) evaluated by the
 * caller at the facet quadrature points (the reference evaluates its expression pointer at the
 * same points, bc/WeakDirichletBC.hpp:225-228). */
typedef struct
{
  int kind; /* rds_bc_kind */
  int nfacets;
  int nfdof;
  int nfgeo;
  int nfq;
  const int32_t *sol_conn; /* [nfacets][nfdof] */
  const int32_t *geo_conn; /* [nfacets][nfgeo] */
  const double *fw;        /* [nfq] */
  const double *fV;        /* [nfq][nfdof] */
  const double *fdVgeo;    /* [dim-1][nfq][nfgeo] */
  const double *gq;        /* RDS_BC_WEAK_DIRICHLET: [nfacets][nfq][neq]; RDS_BC_WEAK_FARFIELD:
                            [neq]; RDS_BC_STRONG_DIRICHLET: [nfacets][nfdof][neq]; NULL
                            otherwise */
  int order;               /* polynomial order of the facet basis (WeakWall relaxation) */
  double params[4];        /* kind-specific parameters (set_parameter of the reference) */
} rds_bc_group;

/* Create a context on the current CUDA device. 'stream' is a cudaStream_t to run on, or NULL
 * for a stream owned by the context. */
RDS_API rds_status rds_create(rds_ctx **ctx, const rds_desc *desc, void *stream);
RDS_API rds_status rds_add_cell_group(rds_ctx *ctx, const rds_cell_group *group);
/* Boundary conditions are applied in the order they are added. */
RDS_API rds_status rds_add_bc(rds_ctx *ctx, const rds_bc_group *bc);
/* Build the node-centred gather lists and the dual volumes. Required before any solve call. */
RDS_API rds_status rds_finalize(rds_ctx *ctx);

RDS_API rds_status rds_set_state(rds_ctx *ctx, const double *u_aos);
RDS_API rds_status rds_get_state(rds_ctx *ctx, double *u_aos);
/* assemble_lhs_and_rhs(CFL): residual, wave speed and local time step. */
RDS_API rds_status rds_assemble(rds_ctx *ctx, double cfl);
/* assemble_rhs(): residual and wave speed only. */
RDS_API rds_status rds_assemble_rhs(rds_ctx *ctx);
/* solve(): u -= dt * res */
RDS_API rds_status rds_update(rds_ctx *ctx);
/* compute_residual_norm(): sqrt(sum_n (res_n dt_n)^2 / N) per equation, into norm[neq]. */
RDS_API rds_status rds_residual_norm(rds_ctx *ctx, double *norm);
/* Element Jacobians of the PGLDA, PGN and PGB schemes at the current state, as the reference's
 * Picard-linearised implicit solver assembles them (solver/rdm/cellsplitters/PGLDA.hpp:316-536,
 * PGN.hpp:296-440, PGB.hpp:505-690, called from
 * solver/rdm/assembly/PGRDMPicardJacCellAssemblyWorker.hpp:370):
 * PGLDA J_mn = sum_q w_q |J_q| K+_m (sum_k K+_k)^-1 K_n (K_n the unclipped upwind matrix);
 * PGN   J_mn = sum_q w_q |J_q| (delta_mn K+_m - K+_m (sum_k K-_k)^-1 K-_n) (the reference's
 *       implicit PGN is the plain N scheme);
 * PGB   J_mn = PGLDA + theta sum_q w_q |J_q| (delta_mn K+_m - K+_m (sum_k K+_k)^-1 K+_n), theta
 *       the cell's blending coefficient of the residual at the same state.
 * jac: device array [ncells][ndof*neq][ndof*neq] of cell group 'group' (row m*neq + i, column
 * n*neq + j), before the division by the dual volumes. Asynchronous on the context's stream
 * (for PGB the residual kernel runs first to get theta; the residual fields are not touched). */
RDS_API rds_status rds_element_jacobians(rds_ctx *ctx, int group, double *jac);

/* The same Jacobians assembled into a block-CSR matrix over the solution nodes, as the
 * reference's Picard worker hands them to its sparse matrix (PGRDMPicardJacCellAssemblyWorker.hpp:
 * 392-412): block (v, w) (neq x neq) = sum over the cells holding nodes v and w of the (v, w)
 * block of their element matrix, each entry divided by the dual volume of v. No Dirichlet rows
 * are removed and no boundary terms are added.
 *   rds_jacobian_pattern: nnzb (number of blocks) and, when not NULL, row_ptr [nnodes + 1] and
 *     col_idx [nnzb] (host arrays; columns ascending within a row). Built on the first call.
 *   rds_assemble_jacobian: values (device array [nnzb][neq][neq], row-major blocks) at the
 *     current state. Asynchronous on the context's stream. */
RDS_API rds_status rds_jacobian_pattern(rds_ctx *ctx, int64_t *nnzb, int32_t *row_ptr,
                                        int32_t *col_idx);
RDS_API rds_status rds_assemble_jacobian(rds_ctx *ctx, double *values);

/* Stabilisation fields (solver/rdm/RDMethod.hpp:79-85, read by the cell worker at
 * solver/rdm/assembly/PGRDMExplicitCellWorker.hpp:505-533). Both are nodal [nnodes] host
 * arrays, copied; NULL removes the field.
 *   rds_set_blending_coeff       (set_blending_coeff): PGB cells use theta_n = theta[dof(c,n)]
 *     instead of their own blending coefficient, res_n = lda_n + theta_n diss_n, and drop the
 *     N part when every theta_n < 1e-6 (solver/rdm/cellsplitters/PGB.hpp:141-148,467-477).
 *     Other schemes ignore it. rds_element_jacobians refuses PGB contexts that have one.
 *   rds_set_artificial_viscosity (set_artificial_viscosity): PGLDA cells add
 *     w_q detJ_q eps_q grad phi_n . grad u(q), eps_q = sum_n V(q,n) eps[dof(c,n)]
 *     (cellsplitters/PGLDA.hpp:245-256). Other schemes ignore it.
 * Not in batched contexts. */
RDS_API rds_status rds_set_blending_coeff(rds_ctx *ctx, const double *theta);
RDS_API rds_status rds_set_artificial_viscosity(rds_ctx *ctx, const double *eps);

/* Stabilisation operators on the current state (its first component), the producers of those
 * fields: solver/art_visc/ArtificialViscosity.hpp and solver/rdm/blending_coeff/ (the
 * RDBlendingCoeff types LF_Blend, ViscosityIndicator, WongJansen, Bonanni2D / Bonanni3D).
 *   rds_set_stab_tables (after rds_finalize), per cell group:
 *     nq, w [nq], Vn [nq][ndof], R [nq][ndof]: the smoothness sensor's rule (exact to degree
 *       2p on the reference element), the nodal basis there, and the map from nodal values to
 *       u - u_{p-1} there, u_{p-1} the reference's modal truncation (the L2 projection onto
 *       degree p - 1; at p = 1 the reference truncates to 0, R = Vn). nq = 0: no sensor.
 *     nvert, P1 [ndof][nvert]: the vertex interpolant at the cell's nodes (cell-to-node
 *       transfer).
 *   rds_compute_stabilisation: cell values of operator op (rds_stab_op), into cells_out
 *     [total cells, groups in order] when not NULL; their nodal field (every vertex the max of
 *     0 and its cells' values, every other node the vertex interpolant of the last cell holding
 *     it; interpolation/mesh_function/MeshFunctionTools.hpp:52-397) into nodes_out [nnodes]
 *     when not NULL; install != 0 makes the nodal field the context's artificial viscosity
 *     (RDS_STAB_ART_VISC) or blending coefficient (the blend operators), as
 *     rds_set_artificial_viscosity / rds_set_blending_coeff would, without a host copy.
 *     The sensor operators need sensor tables on every group, and on groups that are not
 *     affine simplices (bilinear quadrilaterals) the geometry tables of
 *     rds_set_stab_geo_tables.
 *   rds_set_stab_geo_tables (after rds_set_stab_tables with nq > 0): dVgeo [dim][nq][ngeo],
 *     the derivatives of the group's geometry basis (ngeo <= 4 nodes) at the sensor's points;
 *     the sensor then takes detJ at every point, as the reference's geometry metric does
 *     (ArtificialViscosity.hpp:388-426). Replaces the affine detJ of simplex groups. */
typedef enum
{
  RDS_STAB_ART_VISC          = 0, /* compute_artificial_viscosity; p0 = kappa, p1 = factor */
  RDS_STAB_INDICATOR         = 1, /* compute_indicator_normalized (cells only); p0 = kappa */
  RDS_STAB_BLEND_LF          = 2, /* "LF_Blend" */
  RDS_STAB_BLEND_VISC        = 3, /* "ViscosityIndicator"; p0 = kappa */
  RDS_STAB_BLEND_WONG_JANSEN = 4, /* "WongJansen"; p0 = u_inf */
  RDS_STAB_BLEND_BONANNI     = 5  /* "Bonanni2D" / "Bonanni3D" (Euler 2D / 3D); needs the tables
                                     of rds_set_bonanni_tables */
} rds_stab_op;
RDS_API rds_status rds_set_stab_tables(rds_ctx *ctx, int group, int nq, const double *w,
                                       const double *Vn, const double *R, int nvert,
                                       const double *P1);
RDS_API rds_status rds_set_stab_geo_tables(rds_ctx *ctx, int group, int ngeo,
                                           const double *dVgeo);
RDS_API rds_status rds_compute_stabilisation(rds_ctx *ctx, int op, double p0, double p1,
                                             int install, double *cells_out, double *nodes_out);

/* Bonanni's pressure-based blending coefficient (solver/rdm/blending_coeff/
 * BonanniBlendingCoeffImpl.hpp:171-392, selected as "Bonanni2D" / "Bonanni3D" by
 * RDBlendingCoeff.hpp:139-160): per cell c, with the reference's Gauss rule of order
 * max(p, geometry order), f_c = (v_c . gp_c) |v_c| where v_c, gp_c are the cell means of the
 * velocity and of grad p (p, V from the nodal states), and lc = |K_c|^(1/D); then
 * theta_c = min(1, max(f_c / ((p_max - p_min) |v_dom|^2), 0)^2 lc), p_min / p_max over the
 * nodal pressures and v_dom the mesh's mean velocity. rds_set_bonanni_tables (after
 * rds_finalize), per cell group: that rule's nq points, w [nq], the solution basis
 * V [nq][ndof] and its reference derivatives dV [dim][nq][ndof], the geometry basis derivatives
 * dVgeo [dim][nq][ngeo] (straight-sided cells: ngeo <= 4). */
RDS_API rds_status rds_set_bonanni_tables(rds_ctx *ctx, int group, int nq, const double *w,
                                          const double *V, const double *dV,
                                          const double *dVgeo);

/* One step on host buffers, pipelined: upload u_in ([nnodes][neq], pinned host memory for the
 * copies to overlap), one assemble_lhs_and_rhs + solve, residual norm into norm[neq] (may be
 * NULL) and the new state into u_out ([nnodes][neq], pinned). Returns without waiting; the
 * upload of the next call and the download of this one overlap the compute (two staging
 * buffers, separate copy streams), so consecutive calls keep both copy directions and the GPU
 * busy. u_in must stay unchanged and u_out / norm unread until rds_step_sync returns. The same
 * sequence as rds_set_state, rds_assemble, rds_update, rds_residual_norm, rds_get_state
 * (solver/rdm/PGRDMethodExplicit.hpp:417-514). */
RDS_API rds_status rds_step_host(rds_ctx *ctx, const double *u_in, double *u_out, double cfl,
                                 double *norm);
/* Waits for every issued rds_step_host and reports the status flags. */
RDS_API rds_status rds_step_sync(rds_ctx *ctx);

/* Partitioned single mesh (no counterpart call in the reference, whose explicit solver runs
 * one mesh per process): one context per rank holds a part of the cells and the nodes they
 * touch, renumbered; the ranks add their partial nodal sums at the nodes they share.
 * Per iteration: rds_assemble_rhs, rds_pack_interface, a sum of the buffers over the ranks
 * (e.g. an NCCL all-reduce on the context's stream), rds_unpack_interface, rds_finish, a sum
 * of 'sq' over the ranks; norm = sqrt(sum / total node count).
 *   rds_set_dual_volume: replaces the dual volumes [nnodes] (host) after rds_finalize, with the
 *     sums over all ranks' cells at the shared nodes.
 *   rds_set_interface: the n shared nodes (local numbers) and their slots in an exchange
 *     buffer of nslots x (neq + 1) doubles, and owned [nnodes] (host, 1 where this rank counts
 *     the node in the norm: every node is owned by exactly one rank).
 *   rds_pack_interface: zeroes the device buffer, then writes residual and wave speed of the
 *     shared nodes at their slots.
 *   rds_unpack_interface: the summed residual and wave speed back from the device buffer.
 *   rds_finish: dt = CFL V / ws, u -= dt res when update != 0, and sq[neq] (device) = sum over
 *     the owned nodes of (res dt)^2. Asynchronous; rds_check reports the status flags
 *     (non-finite values, non-positive pressure) raised by the work done so far. */
RDS_API rds_status rds_set_dual_volume(rds_ctx *ctx, const double *vol);
RDS_API rds_status rds_set_interface(rds_ctx *ctx, int n, const int32_t *nodes,
                                     const int32_t *slots, int nslots, const uint8_t *owned);
RDS_API rds_status rds_pack_interface(rds_ctx *ctx, double *buf);
RDS_API rds_status rds_unpack_interface(rds_ctx *ctx, const double *buf);
RDS_API rds_status rds_finish(rds_ctx *ctx, double cfl, int update, double *sq);

/* The assembly of rds_assemble_rhs in two parts, so that a partitioned iteration can send the
 * interface sums while the remaining cells run (local node numbering with the interface nodes
 * first, each cell group split into the cells touching an interface node and the rest):
 *   rds_assemble_rhs_cells: the cell kernels of groups [g0, g1) and, when with_bcs != 0, the
 *     weak boundary conditions; no nodal sums.
 *   rds_gather_rhs: the nodal sums of residual and wave speed of nodes [v0, v1) from the
 *     contribution slots (every cell and facet of those nodes must have run).
 * rds_assemble_rhs_cells(ctx, 0, ngroups, 1) then rds_gather_rhs(ctx, 0, nnodes) is
 * rds_assemble_rhs. Reference: the cell loop and nodal sums of PGRDMethodExplicit::assemble_rhs
 * (PGRDMethodExplicit.hpp:428-463, PGRDMExplicitCellWorker.hpp:549-567). */
RDS_API rds_status rds_assemble_rhs_cells(rds_ctx *ctx, int g0, int g1, int with_bcs);
RDS_API rds_status rds_gather_rhs(rds_ctx *ctx, int v0, int v1);

/* The finish of a partitioned iteration in two node ranges: the nodes whose sums are complete on
 * this rank finish right after their gather, the interface nodes after the exchange.
 *   rds_gather_finish: nodal sums of nodes [v0, v1), dt = CFL V / ws, u -= dt res, and their
 *     block sums of (res dt)^2 (all of them counted: nodes outside the interface are this
 *     rank's own); with sq (device, neq doubles) non-null, also their sum into sq (for a rank
 *     without interface nodes, which then needs no rds_finish_nodes).
 *   rds_finish_nodes: rds_finish for nodes [v0, v1) (owned ones in the norm); sq[neq] (device)
 *     = the sum of its and the preceding rds_gather_finish's block sums, in a fixed order (sq
 *     null: the block sums only, for a step whose norm is not needed).
 * rds_finish(ctx, cfl, update, sq) is rds_finish_nodes(ctx, cfl, update, 0, nnodes, sq) without
 * a preceding rds_gather_finish. */
RDS_API rds_status rds_gather_finish(rds_ctx *ctx, int v0, int v1, double cfl, double *sq);
RDS_API rds_status rds_finish_nodes(rds_ctx *ctx, double cfl, int update, int v0, int v1,
                                    double *sq);

/* RK3TVD in a partitioned context (RK3TVD::advance_in_time, solver/time/ExplicitTimeStepper.cpp:
 * 66-100, with the exchange in every stage): per stage k = 1, 2, 3
 *   rds_rk_stage_state(ctx, k): the following calls read the stage state (u_n, u_1, u_2) and
 *     write the stage residual (the context's own, then a scratch buffer), as the reference's
 *     stepper points its solver at them; rds_rk_stage_state(ctx, 0) restores the context's
 *     own state and residual (required before any other call); the first call allocates the
 *     stage buffers (make it outside a stream capture);
 *   the assembly of the partitioned iteration (rds_assemble_rhs_cells, rds_gather_rhs over the
 *     interface nodes, rds_pack_interface, the sum over the ranks, rds_unpack_interface);
 *   rds_gather_rk: the nodal sums of nodes [v0, v1) ending in the stage combination (stage 1:
 *     dt = CFL V / ws and u_1 = u_n - dt r; 2: u_2 = 3/4 u_n + 1/4 u_1 - 1/4 dt r; 3:
 *     u_n+1 = 1/3 u_n + 2/3 u_2 - 2/3 dt r, dt of stage 1), for the nodes complete on the rank;
 *   rds_combine_rk: the same combination for nodes [v0, v1) from their summed residual and wave
 *     speed (the interface nodes, after the exchange). */
RDS_API rds_status rds_rk_stage_state(rds_ctx *ctx, int stage);
RDS_API rds_status rds_gather_rk(rds_ctx *ctx, int v0, int v1, double cfl);
RDS_API rds_status rds_combine_rk(rds_ctx *ctx, int v0, int v1, double cfl);
RDS_API rds_status rds_check(rds_ctx *ctx);

/* Copy out any of: residual [node][neq], dt [node], nodal wave speed [node], dual volume [node]
 * (NULL skips). */
RDS_API rds_status rds_get_fields(rds_ctx *ctx, double *res_aos, double *dt, double *ws, double *vol);

/* Pseudo-time loop on the device: up to max_iter x (assemble_lhs_and_rhs(cfl) + solve()),
 * stopping after the first iteration whose norm satisfies max_eq norm/norm(iter 0) <= drop
 * (drop <= 0: run exactly max_iter). The loop is captured once in a CUDA graph and replayed.
 * it_done: iterations executed; hist (may be NULL): [max_iter][neq] norms. Returns
 * RDS_ERR_ITER_CAP when drop > 0 was not reached. */
RDS_API rds_status rds_iterate(rds_ctx *ctx, double cfl, int max_iter, double drop, int *it_done,
                       double *hist);

/* Options: "mixed_refresh" (default 24): with RDS_MIXED and scalar physics, rds_iterate and
 * rds_iterate_batch run the defect-correction loop: an exact FP64 sweep every mixed_refresh
 * sweeps, FP32 correction sweeps between (the change of every contribution computed from the
 * correction itself, the coefficients and time steps of the exact sweep's state); the loop
 * stops only at an exact sweep and converges to the FP64 scheme's fixed point. Longer periods
 * save exact sweeps but hold the time steps longer: at 32, three Burgers P1 N-scheme problems
 * at CFL 0.53 diverged (RDS_ERR_NONFINITE), none at 24.
 * "mixed_fuse_cells" (default 65536): in a single context with one triangle group of at most
 * that many cells and weak Dirichlet conditions only, the mixed_refresh - 1 correction sweeps
 * of a cycle run as one launch, a barrier between the cells-and-facets phase and the node
 * phase of every sweep: the same arithmetic as the separate launches, bit for bit, without
 * their launch latency. Meshes of up to two items a thread of a 16-CTA cluster run as one
 * thread-block cluster with its hardware barrier; larger ones as a grid of resident CTAs with
 * a bounded barrier in global memory. 0 keeps separate launches. A barrier wait that
 * gives up makes the call return RDS_ERR_CUDA ("bounded device wait"); "fuse_test_wait" (> 0,
 * a test option) forces that after the given number of polls.
 * "mixed_switch" (default 1e-6): with RDS_MIXED and Euler physics (or a stabilisation field
 * installed), rds_iterate runs FP32 cell kernels
 * until max_eq norm/norm(iter 0) <= mixed_switch, or, once that drop has halved at least
 * once, until it has not halved for max(mixed_stall_min, mixed_stall_mult x the last interval
 * between halvings) iterations (the problem's FP32 round-off floor; defaults 200 and 3), and
 * then finishes with FP64 sweeps to the requested drop.
 * "tensor_cores" (default 0): with RDS_MIXED, scalar physics on straight-sided P1-P3 triangles,
 * 1 runs the FP32 cell kernel with its basis contractions on the tensor cores (tcgen05,
 * 3xTF32); results agree with the CUDA-core FP32 kernel to FP32 accuracy. */
RDS_API rds_status rds_set_option(rds_ctx *ctx, const char *key, double value);

/* Enqueue n fused iterations (assemble_lhs_and_rhs(cfl) + solve()) on the context's stream and
 * return without waiting: no residual-drop test, no copies back. For timing with events on
 * rds_stream(); the norms of these iterations are not kept. */
RDS_API rds_status rds_run(rds_ctx *ctx, double cfl, int n);

/* nsteps x RK3TVD::advance_in_time(scheme, cfl) (src/solver/time/ExplicitTimeStepper.cpp:66-100):
 * per step the residual, wave speed and dt at u_n (assemble_lhs_and_rhs), u_1 = u_n - dt r,
 * the residual at u_1 (assemble_rhs; cells and conditions read u_1), u_2 = 3/4 u_n + 1/4 u_1 -
 * 1/4 dt r(u_1), the residual at u_2, u_n+1 = 1/3 u_n + 2/3 u_2 - 2/3 dt r(u_2). Afterwards the
 * context's residual and dt are those of the last step's first stage, as the reference's solver
 * holds them, so rds_residual_norm / rds_get_fields give what compute_residual_norm and the
 * solver's functions give after advance_in_time. One step is captured in a CUDA graph and
 * replayed; enqueued without waiting. The stages run the FP64 cell kernels in every context (a
 * mixed context's steps equal an FP64 context's). In a batched context every problem takes the
 * steps with its own CFL (cfl is ignored), bit for bit its single-problem steps; partitioned
 * contexts return RDS_ERR_UNSUPPORTED (their steps: rds_rk_stage_state, rds_gather_rk,
 * rds_combine_rk below). The three stage buffers are allocated on the first call. */
RDS_API rds_status rds_advance_rk3tvd(rds_ctx *ctx, double cfl, int nsteps);

/* Batched independent problems (no counterpart in the reference, which solves one problem per
 * solver object, src/solver/rdm/PGRDMethodExplicit.hpp:417-514). One context holds the disjoint
 * union of P problems of scalar 2D physics: problem p owns nodes [node_offsets[p],
 * node_offsets[p+1]) and runs at its own CFL. Call rds_set_problems right after rds_create,
 * then add each cell group with the per-problem cell offsets (cells of problem p are rows
 * [problem_cells[p], problem_cells[p+1]) of the group, and refer only to nodes of p) and its
 * physics / scheme (advection and Burgers groups may share the context), and the weak
 * conditions with their physics; then rds_finalize and rds_set_state as usual.
 * rds_iterate_batch iterates every problem until its own max_eq norm/norm(iter 0) <= drop or
 * max_iter: one persistent launch per group walks the tiles of the problems still iterating,
 * the gather updates and tests each problem separately, and the whole loop is one CUDA graph.
 * With RDS_MIXED every problem runs FP32 cell kernels down to max(drop, mixed_switch) (or to
 * its FP32 floor, as in rds_iterate) and then FP64 ones. Every problem's iterates equal those of its own single-problem context bit for
 * bit. iters[P] and rel[P] (may be NULL) receive the iterations done and the final
 * max_eq norm/norm(iter 0); RDS_ERR_ITER_CAP when a problem did not reach drop > 0.
 * rds_autotune times the persistent cell kernels for tiles of 64/128 cells per CTA and
 * 1-16 CTAs per SM and keeps the fastest per group and precision; report (may be NULL)
 * receives a JSON list of the choices. */
RDS_API rds_status rds_set_problems(rds_ctx *ctx, int nproblems, const int32_t *node_offsets,
                                    const double *cfl);
RDS_API rds_status rds_add_batch_cell_group(rds_ctx *ctx, const rds_cell_group *group,
                                            int physics, int scheme,
                                            const int32_t *problem_cells);
RDS_API rds_status rds_add_batch_bc(rds_ctx *ctx, const rds_bc_group *bc, int physics);
RDS_API rds_status rds_iterate_batch(rds_ctx *ctx, int max_iter, double drop, int32_t *iters,
                                     double *rel);
RDS_API rds_status rds_autotune(rds_ctx *ctx, char *report, int len);

/* Diagnostics. */
/* Measured CUDA-core FMA throughput of this GPU in TFLOP/s (precision: RDS_FP64 or RDS_MIXED
 * for FP32), the roofline denominator of the cell kernels. */
RDS_API rds_status rds_measure_peak(int precision, double *tflops);
RDS_API void *rds_stream(rds_ctx *ctx); /* the cudaStream_t the context launches on */
/* Per-kernel device time over the launches since the last reset (enable = 1 starts event
 * timing around every launch, 0 stops it). names: up to max entries of 32 chars. */
RDS_API rds_status rds_kernel_timing(rds_ctx *ctx, int enable);
RDS_API int rds_kernel_times(rds_ctx *ctx, char (*names)[32], double *ms, int *launches, int max);
/* Kernel launches issued by this context since creation. */
RDS_API long long rds_launch_count(rds_ctx *ctx);

/* Residual norm for callers that cannot allocate device memory (no counterpart in the
 * reference, whose norm runs on the host). For a solver whose device memory belongs to
 * another allocator, or a loop that cannot take the device-wide synchronisation of
 * cudaMalloc/cudaFree: the same result as rds_residual_norm, computed from caller-owned DEVICE
 * arrays, with no context and no allocation of any kind.
 *   res  [neq][nnodes] (SoA), dt [nnodes], norm [neq] output: device pointers
 *   stream: cudaStream_t to run on (NULL = default stream); the call only enqueues work.
 * Scratch is a fixed device array inside this library, sized for RDS_NOALLOC_MAX_NODES nodes
 * and 5 equations (1.25 MiB per GPU, held until the process exits); larger inputs get
 * RDS_ERR_TOO_LARGE. Its address is looked up in the first call on each device, so make that
 * first call before any stream capture. The address stays cached for the life of the process:
 * cudaDeviceReset invalidates it (as it invalidates every context of this library), so a process
 * that resets a device does not call this entry point on that device again. All calls share the
 * array: calls that overlap on the GPU race and must be serialised by the caller. */
#define RDS_NOALLOC_MAX_NODES (32768 * 256)
RDS_API rds_status rds_residual_norm_noalloc(const double *res, const double *dt, int nnodes,
                                             int neq, double *norm, void *stream);

RDS_API rds_status rds_destroy(rds_ctx *ctx);
RDS_API const char *rds_last_error(rds_ctx *ctx);
RDS_API const char *rds_version(void);

#ifdef __cplusplus
}
#endif

#endif
