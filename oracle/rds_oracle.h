/* CPU restatement of pdekit's explicit continuous RDS iteration -- TEST ORACLE ONLY.
 *
 * This library is test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load it, as the checker. The product path (pdekit_b200) never calls it.
 *
 * It restates, in plain C with FP64 arithmetic in the reference's operation order, the path
 *   PGRDMethodExplicit::assemble_lhs_and_rhs / solve / compute_residual_norm
 *     (src/solver/rdm/PGRDMethodExplicit.hpp:417-514)
 *   PGRDMExplicitCellWorker::assemble_lhs_and_rhs_impl
 *     (src/solver/rdm/assembly/PGRDMExplicitCellWorker.hpp:340-574)
 *   GeometryMetric / SolutionSpaceMetric / FluxSpaceMetric evaluation
 *     (src/interpolation/GeometryMetric.hpp:364-478, FluxSpaceMetric.hpp:545-746)
 *   PGLDA / PGN / PGB cell splitters
 *     (src/solver/rdm/cellsplitters/PGLDA.hpp:111-311, PGN.hpp:98-290, PGB.hpp:314-498);
 *     PSI, the N residuals limited with the reference's residual limiter
 *     (cellsplitters/LFResidualLimiter.hpp:37-110), which the reference applies only to its
 *     Lax-Friedrichs schemes: that scheme is unpinned (no reference counterpart)
 *   WeakBC::apply + WeakDirichletBC::compute_on_element_weak
 *     (src/solver/rdm/bc/WeakBC.hpp:227-360,786-832, WeakDirichletBC.hpp:159-265)
 *   RDTimeUpdate (src/solver/rdm/RDTimeUpdate.hpp:71-194, RDTimeUpdate.cpp:41-67).
 *
 * Parity of this restatement is pinned against golden vectors produced by the reference
 * itself (oracle/ref_harness.cpp, tests/golden/).
 *
 * Layouts: nodal fields are AoS [node][neq] as the reference's VectorMeshFunction; tables are
 * row-major [rows][cols]; derivative tables are stacked [dim][rows][cols].
 */
#ifndef RDS_ORACLE_H
#define RDS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum
{
  RDSO_ADVECTION_CONST = 0, /* RotationAdvection2D with a constant direction */
  RDSO_BURGERS2D       = 1,
  RDSO_EULER2D         = 2,
  RDSO_EULER3D         = 3
};

enum
{
  RDSO_LDA = 0,
  RDSO_N   = 1,
  RDSO_B   = 2,
  RDSO_PSI = 3 /* the N residuals limited with LFResidualLimiter.hpp:37-110 (scalar) */
};

enum
{
  RDSO_BC_WEAK_DIRICHLET  = 0, /* bc/WeakDirichletBC.hpp */
  RDSO_BC_WEAK_WALL       = 1, /* bc/WeakWall.hpp */
  RDSO_BC_WEAK_SUB_INLET  = 2, /* bc/WeakSubInlet.hpp, params: total temperature, pressure */
  RDSO_BC_WEAK_SUB_OUTLET = 3, /* bc/WeakSubOutlet.hpp, params: outlet pressure */
  RDSO_BC_WEAK_FARFIELD   = 4, /* bc/WeakFarfield.hpp, gq: [neq] reference state */
  RDSO_BC_STRONG_DIRICHLET = 5, /* bc/StrongDirichletBC.hpp, gq: [nfacets][nfdof][neq] values */
  RDSO_BC_WEAK_SUPER_INLET = 6, /* bc/WeakSuperInlet.hpp: wave speed only */
  RDSO_BC_WEAK_SYMMETRY    = 7  /* bc/WeakSymmetry.hpp: mirrored momentum */
};

typedef struct
{
  int physics;
  int scheme;
  int dim;
  int neq;
  double adv[3];   /* advection direction (RDSO_ADVECTION_CONST) */
  double gamma;    /* Euler: 1.4 */
  double gas_R;    /* Euler: 287.05 (temperature only, not on the residual path) */
} rdso_model;

typedef struct
{
  int ncells, ndof, ngeo, nq, nfl;
  const int *sol_conn; /* [ncells][ndof] */
  const int *geo_conn; /* [ncells][ngeo] */
  const double *w;     /* [nq] */
  const double *V;     /* [nq][ndof]         solution basis at quadrature points */
  const double *dV;    /* [dim][nq][ndof]    reference derivatives */
  const double *dVgeo; /* [dim][nq][ngeo]    geometry basis derivatives */
  const double *dVf;   /* [dim][nq][nfl]     flux (order p+1) basis derivatives */
  const double *Vsf;   /* [nfl][ndof]        solution basis at flux nodes */
  int nqv;              /* dual-volume rule (0: use the rule above) */
  const double *wv;     /* [nqv] */
  const double *dVgeo_v; /* [dim][nqv][ngeo] */
} rdso_cells;

typedef struct
{
  int kind;
  int nfacets, nfdof, nfgeo, nfq;
  const int *sol_conn;  /* [nfacets][nfdof] */
  const int *geo_conn;  /* [nfacets][nfgeo] */
  const double *fw;     /* [nfq] */
  const double *fV;     /* [nfq][nfdof] */
  const double *fdVgeo; /* [dim-1][nfq][nfgeo] */
  const double *gq;     /* WeakDirichlet: [nfacets][nfq][neq] boundary state at the facet
                         * quadrature points; WeakFarfield: [neq]; StrongDirichlet:
                         * [nfacets][nfdof][neq] values at the facet dofs */
  int order;            /* polynomial order of the facet's solution basis */
  double params[4];     /* kind-specific parameters */
} rdso_bc;

/* Dual volume: every dof of a cell receives the full cell volume sum_q w_q detJ_q. */
void rdso_dual_volume(const rdso_model *m, const rdso_cells *groups, int ngroups, int nnodes,
                      const double *geo_coords, double *vol);

/* One assemble_lhs_and_rhs(CFL): res, ws and dt from u; StrongDirichlet conditions overwrite
 * their dofs of u in place. Returns the number of non-positive-pressure evaluations seen
 * (Euler), 0 otherwise. */
int rdso_assemble(const rdso_model *m, const rdso_cells *groups, int ngroups, const rdso_bc *bcs,
                  int nbcs, int nnodes, const double *geo_coords, const double *vol,
                  double *u, double cfl, double *res, double *ws, double *dt);

/* solve(): u -= dt * res */
void rdso_update(int nnodes, int neq, const double *dt, const double *res, double *u);

/* compute_residual_norm(): sqrt(sum_n (res*dt)^2 / N) per equation */
void rdso_residual_norm(int nnodes, int neq, const double *res, const double *dt, double *norm);

/* Scheme residual of ONE cell from its nodal values (for kernel-level checks):
 * elem_res [ndof][neq], elem_ws [ndof]. */
void rdso_cell_residual(const rdso_model *m, const rdso_cells *g, const double *X /* [ngeo][dim] */,
                        const double *un /* [ndof][neq] */, double *elem_res, double *elem_ws);

/* Element Jacobian of ONE cell, PGLDA (PGLDA.hpp:316-536), PGN (PGN.hpp:296-440) or PGB
 * (PGB.hpp:505-690) after
 * the model's scheme, [ndof*neq][ndof*neq] row-major. */
void rdso_element_jacobian(const rdso_model *m, const rdso_cells *g, const double *X,
                           const double *un, double *jac);

#ifdef __cplusplus
}
#endif

#endif
