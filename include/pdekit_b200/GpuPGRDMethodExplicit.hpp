/* Drop-in GPU solver for pdekit's explicit continuous RDS method.
 *
 *   GpuPGRDMethodExplicit<MeshConfig, Physics, SchemeTag>
 *
 * replaces PGRDMethodExplicit<MeshConfig, Physics, SchemeTag>
 * (src/solver/rdm/PGRDMethodExplicit.hpp:25-93) where a pdekit program constructs it; it derives
 * from the same base, RDMethod<MeshConfig, Physics> (src/solver/rdm/RDMethod.hpp:33-139), and
 * keeps the call sequence of the reference's examples
 * (examples/testcases-rdm/Advection-Continuous-RDS-2D-Explicit.cpp:70-174):
 *
 *   configure_mesh_data(mesh, geo_dofs, sol_dofs)
 *   initialize_work_data(SFunc::Lagrange, PointSetID::Gauss, quad_order, nb_threads, nb_blocks)
 *   set_vec_function(SolverVecFn::solution / residuals, ...)
 *   add_boundary_condition(type, name, boundary)->set_expression(...) / set_parameter(...)
 *   loop: assemble_lhs_and_rhs(CFL); solve(); compute_residual_norm(norm)
 *
 * The work runs in librds_b200 (include/rds_b200.h) on the GPU. The reference-element tables
 * (quadrature, Lagrange bases and their derivatives, flux basis of order p+1, boundary facet
 * bases) are taken from the reference's own FEValues / StdPointSet / StdRegion classes, so the
 * GPU sees exactly the reference's tables. nb_threads and nb_blocks are accepted and ignored.
 *
 * Scope: physics Burgers2D, Euler2DCons, Euler3DCons and RotationAdvection2D with a constant
 * direction; schemes PGLDA, PGN, PGB; boundary conditions WeakDirichlet (expression of the
 * coordinates, evaluated once at the facet quadrature points), WeakWall, WeakSubInlet,
 * WeakSubOutlet, WeakFarfield (Euler; set_reference_state), WeakSuperInlet, WeakSymmetry
 * (Euler) and StrongDirichlet (expression at the facet dofs' coordinates). Anything else throws
 * std::runtime_error at set-up.
 *
 * Host fields stay the source of truth between calls: assemble_lhs_and_rhs uploads the
 * solution function, and downloads the residual and time-step functions; solve() downloads
 * the updated solution. iterate() runs the whole pseudo-time loop on the device.
 *
 * This header is compiled inside a pdekit build (the reference's src/ on the include path).
 */
#ifndef PDEKIT_B200_GPU_PGRD_METHOD_EXPLICIT_HPP
#define PDEKIT_B200_GPU_PGRD_METHOD_EXPLICIT_HPP

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "interpolation/FEValues.hpp"
#include "math/DenseConstVecView.hpp"
#include "math/DenseSVec.hpp"
#include "mesh/point_set/StdPointSet.hpp"
#include "mesh/std_region/StdRegion.hpp"
#include "physics/euler/Euler2DCons.hpp"
#include "physics/euler/Euler3DCons.hpp"
#include "physics/scalar/Burgers2D.hpp"
#include "physics/scalar/RotationAdvection2D.hpp"
#include "solver/rdm/RDMethod.hpp"
#include "solver/rdm/bc/RDMBCBase.hpp"
#include "solver/rdm/cellsplitters/CellSplitters.hpp"

#include "../rds_b200.hpp"

namespace pdekit
{

namespace solver
{

namespace rdm
{

/* Solvers that run RK3TVD steps on the device (GpuRK3TVD dispatches to them). */
class DeviceRK3TVDSolver
{
  public:
  virtual ~DeviceRK3TVDSolver() = default;
  virtual void advance_rk3tvd(const Real CFL, const Uint nsteps) = 0;
};

namespace gpu_detail
{

/* Physics -> rds_physics (and the constant advection direction). */
template <typename Physics>
struct PhysicsId;

template <>
struct PhysicsId<physics::Burgers2D>
{
  static constexpr int id = RDS_BURGERS2D;
  static void direction(double *)
  {
  }
};

template <>
struct PhysicsId<physics::Euler2DCons>
{
  static constexpr int id = RDS_EULER2D;
  static void direction(double *)
  {
  }
};

template <>
struct PhysicsId<physics::Euler3DCons>
{
  static constexpr int id = RDS_EULER3D;
  static void direction(double *)
  {
  }
};

template <typename Direction>
struct PhysicsId<physics::RotationAdvection2D<Direction>>
{
  static constexpr int id = RDS_ADVECTION_CONST;
  /* The GPU path takes one direction for the whole mesh: the policy is evaluated at two points
   * and must give the same vector. */
  static void direction(double *a)
  {
    math::DenseSVec<Real, 2> x0, x1, v0, v1;
    x0[0] = 0.1;
    x0[1] = 0.2;
    x1[0] = 0.9;
    x1[1] = -0.7;
    Direction::rotation_vector(x0, v0);
    Direction::rotation_vector(x1, v1);
    if (v0[0] != v1[0] || v0[1] != v1[1])
      throw std::runtime_error("GpuPGRDMethodExplicit: the advection direction must be constant");
    a[0] = v0[0];
    a[1] = v0[1];
    a[2] = 0.0;
  }
};

template <typename SchemeTag>
struct SchemeId;
template <>
struct SchemeId<PGLDA>
{
  static constexpr int id = RDS_PGLDA;
};
template <>
struct SchemeId<PGN>
{
  static constexpr int id = RDS_PGN;
};
template <>
struct SchemeId<PGB>
{
  static constexpr int id = RDS_PGB;
};

inline int shape_id(ElemShape s)
{
  switch (s)
  {
  case ElemShape::Line:
    return RDS_LINE;
  case ElemShape::Triag:
    return RDS_TRIAG;
  case ElemShape::Quad:
    return RDS_QUAD;
  case ElemShape::Tetra:
    return RDS_TETRA;
  default:
    throw std::runtime_error("GpuPGRDMethodExplicit: element shape not supported on the GPU");
  }
}

inline std::vector<double> rows(const math::DenseDMat<Real> &m)
{
  std::vector<double> v(m.rows() * m.cols());
  for (Uint r = 0; r < m.rows(); ++r)
    for (Uint c = 0; c < m.cols(); ++c)
      v[r * m.cols() + c] = m(r, c);
  return v;
}

inline void append(std::vector<double> &dst, const std::vector<double> &src)
{
  dst.insert(dst.end(), src.begin(), src.end());
}

/* Lagrange basis of order p on an element shape, evaluated at points. */
inline void fill_fe(interpolation::FEValues &fe, ElemShape shape, Uint p,
                    const math::DenseDMat<Real> &pts, const math::DenseDVec<Real> &w)
{
  fe.configure(mesh::PointSetTag(shape, p, PointSetID::Equidist),
               mesh::sf::SFTag(shape, SFunc::Lagrange, p, ModalBasis::Modal));
  fe.fill_Vandermonde(pts, w);
}

} // namespace gpu_detail

/* Boundary condition record: what the user configures on the object returned by
 * add_boundary_condition. The GPU applies the condition; apply() is not used. */
template <typename MeshConfig, typename Physics>
class GpuRDMBC : public RDMBCBase<MeshConfig, Physics, Physics::DIM - 1>
{
  public:
  using expr_type = Real (*)(const math::DenseConstVecView<Real> &,
                             const interpolation::VectorMeshFunction<Real>::const_entry_type &,
                             const Uint);

  GpuRDMBC(const std::string &type, const std::string &name, const std::string &boundary)
      : RDMBCBase<MeshConfig, Physics, Physics::DIM - 1>(name), m_type(type), m_boundary(boundary)
  {
  }

  void set_expression(expr_type e) override
  {
    m_expr = e;
  }
  void set_parameter(const std::string &param_name, const Real value) override
  {
    m_params[param_name] = value;
  }
  /* WeakFarfield: the reference state in conservative variables */
  void set_reference_state(const math::DenseDVec<Real> &state) override
  {
    m_state.assign(state.size(), 0.0);
    for (Uint i = 0; i < state.size(); ++i)
      m_state[i] = state[i];
  }
  RDMBCType bc_type() const override
  {
    return m_type == "StrongDirichlet" ? BC_TYPE_STRONG : BC_TYPE_WEAK;
  }
  void apply(RDTimeUpdate &) override
  {
    throw std::runtime_error("GpuRDMBC::apply: the condition is applied on the GPU");
  }

  const std::string &type() const
  {
    return m_type;
  }
  const std::string &boundary() const
  {
    return m_boundary;
  }
  expr_type expression() const
  {
    return m_expr;
  }
  const std::vector<Real> &reference_state() const
  {
    return m_state;
  }
  Real parameter(const std::string &n) const
  {
    const auto it = m_params.find(n);
    if (it == m_params.end())
      throw std::runtime_error("boundary condition '" + this->name() + "': parameter '" + n +
                               "' not set");
    return it->second;
  }

  private:
  std::string m_type, m_boundary;
  expr_type m_expr = nullptr;
  std::vector<Real> m_state;
  std::map<std::string, Real> m_params;
};

template <typename MeshConfig, typename Physics, typename SchemeTag>
class GpuPGRDMethodExplicit : public RDMethod<MeshConfig, Physics>, public DeviceRK3TVDSolver
{
  using base           = RDMethod<MeshConfig, Physics>;
  using mesh_type      = typename base::mesh_type;
  using cell_dofs      = typename base::cell_dofs;
  using bc_base_type   = typename base::bc_base_type;
  using bc_type        = GpuRDMBC<MeshConfig, Physics>;
  using vec_fn         = interpolation::VectorMeshFunction<Real>;
  static constexpr Uint D   = MeshConfig::GDIM;
  static constexpr Uint NEQ = Physics::NEQ;

  public:
  explicit GpuPGRDMethodExplicit(int precision = RDS_FP64) : m_precision(precision)
  {
  }
  ~GpuPGRDMethodExplicit() override = default;

  bool is_continuous() const override
  {
    return true;
  }
  bool is_explicit() const override
  {
    return true;
  }

  void initialize_work_data(const SFunc sf_type, const PointSetID quad_type,
                            const Uint quadrature_order, const Uint nb_threads,
                            const Uint nb_blocks) override
  {
    base::initialize_work_data(sf_type, quad_type, quadrature_order, nb_threads, nb_blocks);
    if (sf_type != SFunc::Lagrange || quad_type != PointSetID::Gauss)
      throw std::runtime_error("GpuPGRDMethodExplicit: Lagrange bases and Gauss rules only");
    m_ctx.reset();
  }

  void compute_node_reordering(const mesh_type &, const cell_dofs &, std::vector<Int> &) override
  {
  }
  void compute_cell_reordering(const mesh_type &, const cell_dofs &, std::vector<Int> &) override
  {
  }

  std::shared_ptr<bc_base_type> add_boundary_condition(const std::string &bc_type_name,
                                                       const std::string &condition_name,
                                                       const std::string &boundary_name) override
  {
    if (bc_type_name != "WeakDirichlet" && bc_type_name != "WeakWall" &&
        bc_type_name != "WeakSubInlet" && bc_type_name != "WeakSubOutlet" &&
        bc_type_name != "WeakFarfield" && bc_type_name != "StrongDirichlet" &&
        bc_type_name != "WeakSuperInlet" && bc_type_name != "WeakSymmetry")
      throw std::runtime_error("GpuPGRDMethodExplicit: boundary condition '" + bc_type_name +
                               "' not supported on the GPU");
    auto bc             = std::make_shared<bc_type>(bc_type_name, condition_name, boundary_name);
    m_bcs[condition_name] = bc;
    m_ctx.reset();
    return bc;
  }
  std::shared_ptr<bc_base_type> boundary_condition(const std::string &condition_name) const override
  {
    const auto it = m_bcs.find(condition_name);
    return it == m_bcs.end() ? nullptr : it->second;
  }
  void remove_boundary_condition(const std::string &condition_name) override
  {
    m_bcs.erase(condition_name);
    m_ctx.reset();
  }
  void remove_all_boundary_conditions() override
  {
    m_bcs.clear();
    m_ctx.reset();
  }

  /* Residual, wave speed and local time step at the current solution (PGRDMethodExplicit.hpp:
   * 417-423); the residual and time-step functions receive the results. */
  void assemble_lhs_and_rhs(const Real CFL) override
  {
    ensure_context();
    upload_solution();
    m_ctx->assemble(CFL);
    m_cfl_set = true;
    download_fields();
    download_strong_state();
  }
  void assemble_rhs() override
  {
    ensure_context();
    if (!m_cfl_set)
      throw std::runtime_error("GpuPGRDMethodExplicit: assemble_rhs before assemble_lhs_and_rhs");
    upload_solution();
    m_ctx->assemble_rhs();
    download_fields();
    download_strong_state();
  }
  /* u -= dt * res (PGRDMethodExplicit.hpp:468-477). */
  void solve(std::vector<SolverOption> const & = {}) override
  {
    ensure_context();
    m_ctx->update();
    download_solution();
  }
  void compute_residual_norm(math::DenseDVec<Real> &norm_L2) const override
  {
    if (!m_ctx)
      throw std::runtime_error("GpuPGRDMethodExplicit: no residual assembled yet");
    const std::vector<double> n = m_ctx->residual_norm();
    norm_L2.resize(NEQ);
    for (Uint e = 0; e < NEQ; ++e)
      norm_L2[e] = n[e];
  }

  /* The pseudo-time loop on the device (graph-captured), to max_iter iterations or to
   * max_eq norm / norm(iteration 0) <= drop; the solution function receives the result. */
  rds_b200::Context::IterateResult iterate(const Real CFL, const Uint max_iter, const Real drop,
                                           const bool throw_on_cap = true)
  {
    ensure_context();
    upload_solution();
    rds_b200::Context::IterateResult r = m_ctx->iterate(CFL, int(max_iter), drop, throw_on_cap);
    download_solution();
    return r;
  }

  /* nsteps of the reference's RK3TVD::advance_in_time(*this, CFL) (solver/time/
   * ExplicitTimeStepper.cpp:66-100) with the stages on the device: one upload before, the
   * solution, residual and time-step functions refreshed after (the residual and dt of the
   * last step's first stage, as the reference's stepper leaves them). */
  void advance_rk3tvd(const Real CFL, const Uint nsteps = 1) override
  {
    ensure_context();
    upload_solution();
    m_ctx->advance_rk3tvd(CFL, int(nsteps));
    m_cfl_set = true;
    download_solution();
    download_fields();
  }

  rds_b200::Context &context()
  {
    ensure_context();
    return *m_ctx;
  }

  private:
  /* Builds the device context from the mesh, the reference's tables and the conditions. */
  void ensure_context()
  {
    if (m_ctx)
      return;
    if (!base::m_tria || base::m_sol_dofs.is_null() || base::m_geo_dofs.is_null())
      throw std::runtime_error("GpuPGRDMethodExplicit: configure_mesh_data first");
    const mesh_type &tria = *base::m_tria;
    const cell_dofs &sol  = *base::m_sol_dofs;
    const cell_dofs &geo  = *base::m_geo_dofs;
    const Uint quad_order = base::m_quad_order;

    // geometry node coordinates, indexed by geometry dof
    const Uint ngeo_nodes = geo.nb_nodes();
    m_coords.assign(ngeo_nodes * D, 0.0);
    const Uint ncells = sol.nb_active_cells();
    struct Group
    {
      ElemShape shape;
      Uint p, pg;
      std::vector<int32_t> sconn, gconn;
      Uint ndof = 0, ngeo = 0;
    };
    std::map<std::pair<int, int>, Group> groups;
    for (Uint c = 0; c < ncells; ++c)
    {
      const mesh::MeshEntity sc = sol.active_cell(mesh::ActiveIdx(c));
      const mesh::MeshEntity gc = geo.active_cell(mesh::ActiveIdx(c));
      const auto coords         = tria.active_cell(mesh::ActiveIdx(c)).coordinates();
      for (Uint v = 0; v < gc.nb_vert(); ++v)
      {
        const auto node = coords.const_node_view(v);
        for (Uint d = 0; d < D; ++d)
          m_coords[gc.vertex(v) * D + d] = node[d];
      }
      const ElemShape shape = sc.pt_set_id().elem_shape();
      const Uint p          = sc.pt_set_id().poly_order();
      Group &g = groups[std::make_pair(int(shape), int(p))];
      g.shape  = shape;
      g.p      = p;
      g.pg     = gc.pt_set_id().poly_order();
      g.ndof   = sc.nb_vert();
      g.ngeo   = gc.nb_vert();
      for (Uint n = 0; n < sc.nb_vert(); ++n)
        g.sconn.push_back(int32_t(sc.vertex(n)));
      for (Uint n = 0; n < gc.nb_vert(); ++n)
        g.gconn.push_back(int32_t(gc.vertex(n)));
    }

    rds_desc desc{};
    desc.physics    = gpu_detail::PhysicsId<Physics>::id;
    desc.scheme     = gpu_detail::SchemeId<SchemeTag>::id;
    desc.precision  = m_precision;
    desc.dim        = int(D);
    desc.neq        = int(NEQ);
    desc.nnodes     = int(sol.nb_nodes());
    desc.ngeo_nodes = int(ngeo_nodes);
    desc.geo_coords = m_coords.data();
    desc.gamma      = 1.4; // Euler2DProperties / Euler3DProperties heat capacity ratio
    gpu_detail::PhysicsId<Physics>::direction(desc.adv);
    std::unique_ptr<rds_b200::Context> ctx(new rds_b200::Context(desc));

    for (auto &kv : groups)
      add_group(*ctx, kv.second.shape, kv.second.p, kv.second.pg, kv.second.ndof, kv.second.ngeo,
                kv.second.sconn, kv.second.gconn, quad_order);
    // weak conditions in the manager's order (by condition name, RDMBCManager.hpp:146)
    for (const auto &kv : m_bcs)
      add_condition(*ctx, *kv.second, quad_order);
    ctx->finalize();
    m_ctx = std::move(ctx);
    m_cfl_set = false;
  }

  void add_group(rds_b200::Context &ctx, ElemShape shape, Uint p, Uint pg, Uint ndof, Uint ngeo,
                 const std::vector<int32_t> &sconn, const std::vector<int32_t> &gconn,
                 Uint quad_order)
  {
    using namespace gpu_detail;
    mesh::StdPointSet quad;
    quad.change_type(shape, quad_order, PointSetID::Gauss);
    const math::DenseDMat<Real> &qp = quad.get().coordinates();
    const math::DenseDVec<Real> &qw = quad.get().weights();
    interpolation::FEValues fe_sol, fe_geo, fe_flux, fe_sol_at_flux, fe_vgeo;
    fill_fe(fe_sol, shape, p, qp, qw);
    fill_fe(fe_geo, shape, pg, qp, qw);
    fill_fe(fe_flux, shape, p + 1, qp, qw);
    // solution basis at the nodes of the order p+1 flux basis (FluxSpaceMetric.hpp:316-327)
    mesh::StdRegion flux_region;
    flux_region.change_type(mesh::PointSetTag(shape, p + 1, PointSetID::Equidist));
    const math::DenseDMat<Real> &flux_nodes = flux_region.get().coordinates();
    math::DenseDVec<Real> ones(flux_nodes.rows());
    ones.fill(1.0);
    fill_fe(fe_sol_at_flux, shape, p, flux_nodes, ones);
    // dual volumes use the Gauss rule of the cell's own order (RDTimeUpdate.hpp:85-150)
    mesh::StdPointSet vquad;
    vquad.change_type(shape, p, PointSetID::Gauss);
    fill_fe(fe_vgeo, shape, pg, vquad.get().coordinates(), vquad.get().weights());

    Tables t;
    t.w.assign(qw.size(), 0.0);
    for (Uint q = 0; q < qw.size(); ++q)
      t.w[q] = qw[q];
    t.V   = rows(fe_sol.Vandermonde());
    t.Vsf = rows(fe_sol_at_flux.Vandermonde());
    for (Uint d = 0; d < D; ++d)
    {
      append(t.dV, rows(fe_sol.deriv_Vandermonde(d)));
      append(t.dVgeo, rows(fe_geo.deriv_Vandermonde(d)));
      append(t.dVf, rows(fe_flux.deriv_Vandermonde(d)));
      append(t.dVgeo_v, rows(fe_vgeo.deriv_Vandermonde(d)));
    }
    const math::DenseDVec<Real> &vw = vquad.get().weights();
    t.wv.assign(vw.size(), 0.0);
    for (Uint q = 0; q < vw.size(); ++q)
      t.wv[q] = vw[q];
    const Tables &tb = t; // rds_add_cell_group copies the tables and connectivity

    rds_cell_group g{};
    g.shape    = shape_id(shape);
    g.order    = int(p);
    g.ncells   = int(sconn.size() / ndof);
    g.ndof     = int(ndof);
    g.ngeo     = int(ngeo);
    g.nq       = int(tb.w.size());
    g.nfl      = int(flux_nodes.rows());
    g.sol_conn = sconn.data();
    g.geo_conn = gconn.data();
    g.w        = tb.w.data();
    g.V        = tb.V.data();
    g.dV       = tb.dV.data();
    g.dVgeo    = tb.dVgeo.data();
    g.dVf      = tb.dVf.data();
    g.Vsf      = tb.Vsf.data();
    g.nqv      = int(tb.wv.size());
    g.wv       = tb.wv.data();
    g.dVgeo_v  = tb.dVgeo_v.data();
    ctx.add_cell_group(g);
  }

  void add_condition(rds_b200::Context &ctx, const bc_type &bc, Uint quad_order)
  {
    using namespace gpu_detail;
    using dof_it = typename mesh::BoundaryFacets<MeshConfig, MeshConfig::TDIM - 1>::const_dof_iterator_typed;
    const mesh_type &tria = *base::m_tria;
    const auto bdry_ptr   = tria.all_boundaries().domain(bc.boundary());
    if (!bdry_ptr)
      throw std::runtime_error("GpuPGRDMethodExplicit: no mesh boundary '" + bc.boundary() + "'");
    std::vector<common::IteratorRange<dof_it>> sranges, granges;
    (*bdry_ptr).all_bdry_dof_ranges(*base::m_sol_dofs, sranges);
    (*bdry_ptr).all_bdry_dof_ranges(*base::m_geo_dofs, granges);
    std::vector<int32_t> fsol, fgeo;
    Uint nfdof = 0, nfgeo = 0, pf = 1, pgf = 1;
    ElemShape fshape = ElemShape::Line;
    for (Uint r = 0; r < sranges.size(); ++r)
    {
      auto git = granges[r].begin();
      for (auto it = sranges[r].begin(); it != sranges[r].end(); ++it, ++git)
      {
        const mesh::MeshEntity se = it->mesh_entity();
        const mesh::MeshEntity ge = git->mesh_entity();
        fshape                    = se.pt_set_id().elem_shape();
        pf                        = se.pt_set_id().poly_order();
        pgf                       = ge.pt_set_id().poly_order();
        nfdof                     = se.nb_vert();
        nfgeo                     = ge.nb_vert();
        for (Uint n = 0; n < se.nb_vert(); ++n)
          fsol.push_back(int32_t(se.vertex(n)));
        for (Uint n = 0; n < ge.nb_vert(); ++n)
          fgeo.push_back(int32_t(ge.vertex(n)));
      }
    }
    const Uint nf = nfdof ? Uint(fsol.size() / nfdof) : 0;
    if (nf == 0)
      throw std::runtime_error("GpuPGRDMethodExplicit: boundary '" + bc.boundary() + "' is empty");

    // facet quadrature of order cell order + 1 (RDMethod.hpp:261-263)
    mesh::StdPointSet fquad;
    fquad.change_type(fshape, quad_order + 1, PointSetID::Gauss);
    const math::DenseDMat<Real> &fqp = fquad.get().coordinates();
    const math::DenseDVec<Real> &fqw = fquad.get().weights();
    interpolation::FEValues fe_fsol, fe_fgeo;
    fill_fe(fe_fsol, fshape, pf, fqp, fqw);
    fill_fe(fe_fgeo, fshape, pgf, fqp, fqw);
    const Uint nfq = fqw.size();

    Tables t;
    t.w.assign(nfq, 0.0);
    for (Uint q = 0; q < nfq; ++q)
      t.w[q] = fqw[q];
    t.V = rows(fe_fsol.Vandermonde());
    for (Uint d = 0; d + 1 < D; ++d)
      append(t.dVgeo, rows(fe_fgeo.deriv_Vandermonde(d)));
    const math::DenseDMat<Real> &fVgeo = fe_fgeo.Vandermonde();

    rds_bc_group b{};
    b.nfacets = int(nf);
    b.nfdof   = int(nfdof);
    b.nfgeo   = int(nfgeo);
    b.nfq     = int(nfq);
    b.order   = int(pf);
    if (bc.type() == "WeakDirichlet")
    {
      if (!bc.expression())
        throw std::runtime_error("boundary condition '" + bc.name() + "': no expression set");
      // boundary state at the facet quadrature points; the expression is a function of the
      // coordinates (the state argument is a zero state)
      vec_fn zero("", "zero");
      zero.resize(NEQ, 1);
      zero.fill(0.0);
      t.gq.assign(size_t(nf) * nfq * NEQ, 0.0);
      for (Uint f = 0; f < nf; ++f)
        for (Uint q = 0; q < nfq; ++q)
        {
          Real x[3] = {0.0, 0.0, 0.0};
          for (Uint g = 0; g < nfgeo; ++g)
            for (Uint d = 0; d < D; ++d)
              x[d] += fVgeo(q, g) * m_coords[size_t(fgeo[f * nfgeo + g]) * D + d];
          const math::DenseConstVecView<Real> xv(x, D);
          for (Uint e = 0; e < NEQ; ++e)
            t.gq[(size_t(f) * nfq + q) * NEQ + e] = bc.expression()(xv, zero.const_value(0), e);
        }
      b.kind = RDS_BC_WEAK_DIRICHLET;
    }
    else if (bc.type() == "WeakFarfield")
    {
      if (bc.reference_state().size() != NEQ)
        throw std::runtime_error("boundary condition '" + bc.name() +
                                 "': set_reference_state with " + std::to_string(NEQ) +
                                 " values first");
      t.gq.assign(bc.reference_state().begin(), bc.reference_state().end());
      b.kind = RDS_BC_WEAK_FARFIELD;
    }
    else if (bc.type() == "StrongDirichlet")
    {
      if (!bc.expression())
        throw std::runtime_error("boundary condition '" + bc.name() + "': no expression set");
      // values at the facet dofs (StrongDirichletBC::compute_Dirichlet_data): the expression
      // at the dof's coordinates, with the current state as its state argument. The reference
      // takes the coordinates from the facet geometry's nodes; for the dofs past the geometry
      // nodes of P2 / P3 facets it reads beyond them, here they are the dof coordinates (the
      // facet geometry at the dof's reference point).
      const vec_fn::ptr u = this->vec_function(SolverVecFn::solution);
      if (!u)
        throw std::runtime_error("GpuPGRDMethodExplicit: solution function not set");
      for (const int32_t v : fsol)
        if (Uint(v) >= u->nb_entries())
          throw std::runtime_error("GpuPGRDMethodExplicit: solution function too short");
      mesh::StdRegion fsol_region;
      Uint f0 = 0;
      t.gq.assign(size_t(nf) * nfdof * NEQ, 0.0);
      for (Uint r = 0; r < sranges.size(); ++r)
        for (auto it = sranges[r].begin(); it != sranges[r].end(); ++it, ++f0)
        {
          const mesh::MeshEntity se = it->mesh_entity();
          fsol_region.change_type(se.pt_set_id());
          const math::DenseDMat<Real> &rc = fsol_region.get().coordinates();
          math::DenseDVec<Real> ones(rc.rows());
          ones.fill(1.0);
          interpolation::FEValues fe_at_dofs;
          fill_fe(fe_at_dofs, fshape, pgf, rc, ones);
          const math::DenseDMat<Real> &Vd = fe_at_dofs.Vandermonde();
          for (Uint n = 0; n < nfdof; ++n)
          {
            Real x[3] = {0.0, 0.0, 0.0};
            for (Uint g = 0; g < nfgeo; ++g)
              for (Uint d = 0; d < D; ++d)
                x[d] += Vd(n, g) * m_coords[size_t(fgeo[f0 * nfgeo + g]) * D + d];
            const math::DenseConstVecView<Real> xv(x, D);
            for (Uint e = 0; e < NEQ; ++e)
              t.gq[(size_t(f0) * nfdof + n) * NEQ + e] =
                  bc.expression()(xv, u->const_value(fsol[f0 * nfdof + n]), e);
          }
        }
      b.kind = RDS_BC_STRONG_DIRICHLET;
    }
    else if (bc.type() == "WeakWall")
      b.kind = RDS_BC_WEAK_WALL;
    else if (bc.type() == "WeakSuperInlet")
      b.kind = RDS_BC_WEAK_SUPER_INLET;
    else if (bc.type() == "WeakSymmetry")
      b.kind = RDS_BC_WEAK_SYMMETRY;
    else if (bc.type() == "WeakSubInlet")
    {
      b.kind      = RDS_BC_WEAK_SUB_INLET;
      b.params[0] = bc.parameter("total_temperature");
      b.params[1] = bc.parameter("total_pressure");
    }
    else
    {
      b.kind      = RDS_BC_WEAK_SUB_OUTLET;
      b.params[0] = bc.parameter("total_pressure");
    }
    const Tables &tb = t; // rds_add_bc copies the tables, connectivity and boundary data
    b.sol_conn = fsol.data();
    b.geo_conn = fgeo.data();
    b.fw       = tb.w.data();
    b.fV       = tb.V.data();
    b.fdVgeo   = tb.dVgeo.data();
    b.gq       = tb.gq.empty() ? nullptr : tb.gq.data();
    ctx.add_bc(b);
  }

  /* The state, and the stabilisation fields handed over through the reference's
   * set_blending_coeff / set_artificial_viscosity (RDMethod.hpp:79-85): the reference's cell
   * worker reads their current values at every assembly (PGRDMExplicitCellWorker.hpp:505-533),
   * so they travel with the state. */
  void upload_solution()
  {
    const vec_fn::ptr u = this->vec_function(SolverVecFn::solution);
    if (!u || u->nb_entries() != Uint(m_ctx->nnodes()))
      throw std::runtime_error("GpuPGRDMethodExplicit: solution function not set or wrong size");
    m_ctx->set_state(&u->value(0)[0]);
    upload_field(base::m_blending_coeff, m_blend_sent, &rds_b200::Context::set_blending_coeff);
    upload_field(base::m_art_viscosity, m_av_sent, &rds_b200::Context::set_artificial_viscosity);
  }
  void upload_field(const interpolation::ScalarMeshFunction<Real>::ptr &f, bool &sent,
                    void (rds_b200::Context::*set)(const double *))
  {
    if (f)
    {
      if (f->nb_entries() != Uint(m_ctx->nnodes()))
        throw std::runtime_error("GpuPGRDMethodExplicit: stabilisation field of wrong size");
      ((*m_ctx).*set)(&(*f)[0]);
      sent = true;
    }
    else if (sent)
    {
      ((*m_ctx).*set)(nullptr);
      sent = false;
    }
  }
  void download_solution()
  {
    const vec_fn::ptr u = this->vec_function(SolverVecFn::solution);
    if (u && u->nb_entries() == Uint(m_ctx->nnodes()))
      m_ctx->get_state(&u->value(0)[0]);
  }
  /* StrongDirichlet conditions overwrite their dofs in the solution function during the
   * assembly (StrongDirichletBC::apply, bc/StrongDirichletBC.hpp:202-233); a caller that combines
   * states on the host (a Runge-Kutta stepper) reads them there. */
  void download_strong_state()
  {
    for (const auto &kv : m_bcs)
      if (kv.second->type() == "StrongDirichlet")
      {
        download_solution();
        return;
      }
  }
  void download_fields()
  {
    const vec_fn::ptr res = this->vec_function(SolverVecFn::residuals);
    interpolation::ScalarMeshFunction<Real>::ptr dt = this->scal_function(SolverScalFn::time_step);
    const Uint n = Uint(m_ctx->nnodes());
    double *pres = (res && res->nb_entries() == n) ? &res->value(0)[0] : nullptr;
    if (dt && dt->nb_entries() != n)
      dt->resize(n);
    m_ctx->get_fields(pres, dt ? &(*dt)[0] : nullptr, nullptr, nullptr);
  }

  struct Tables
  {
    std::vector<double> w, V, dV, dVgeo, dVf, Vsf, wv, dVgeo_v, gq;
  };

  int m_precision;
  bool m_cfl_set = false;
  bool m_blend_sent = false, m_av_sent = false;
  std::map<std::string, std::shared_ptr<bc_type>> m_bcs;
  std::vector<double> m_coords;
  std::unique_ptr<rds_b200::Context> m_ctx;
};

} // namespace rdm

} // namespace solver

} // namespace pdekit

#endif
