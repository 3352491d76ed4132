// Test-oracle driver around the reference's own explicit RDS solver.
//
// Linked against the reference sources compiled in place (oracle/Makefile). It is our code,
// written against the reference's public API exactly the way its examples drive it
// (examples/testcases-rdm/Advection-Continuous-RDS-2D-Explicit.cpp:37-174):
//   GmshReader -> DofMap::clone_continuous -> PGRDMethodExplicit<MeshConfig, Physics, Scheme>
//   configure_mesh_data / initialize_work_data / set_vec_function / add_boundary_condition
//   assemble_lhs_and_rhs(CFL) + solve()                 (src/solver/rdm/PGRDMethodExplicit.hpp:417-477)
//
// Two jobs:
//   dump  -- write golden inputs (mesh arrays, reference-element tables, boundary facets,
//            initial state) and outputs (nodal residual, wave speed, dt, dual volume, states
//            after k iterations, residual norms, two steps of the reference's RK3TVD stepper)
//            as raw little-endian arrays + meta.json.
//   time  -- time K explicit iterations (the CPU baseline), print one JSON line.
//
// Usage:
//   rds_ref_harness dump|time <physics> <scheme> <p> <quad> <mesh.msh> <outdir|-> <iters> <cfl>
//                   <init> <bcspec> [threads] [stab]
//     physics: advconst (a = (0.5,1)/|(0.5,1)|) | burgers | euler2d | euler3d
//     scheme : lda | n | b
//     init   : name of an initial-state function of the node coordinates (see init_state)
//     bcspec : comma-separated Type:condition_name:boundary:expr, or "none"
//     stab   : "none" | "av:<kappa>:<factor>" | "blend:<type>:<param>" -- a stabilisation field
//              computed at the initial state by the reference's own operators and handed to the
//              solver the way examples/testcases-rdm/Burgers-RDS-2D.cpp:121-176 does:
//              ArtificialViscosity (solver/art_visc/ArtificialViscosity.hpp) ->
//              set_artificial_viscosity, or RDBlendingCoeff of <type> (LF_Blend,
//              ViscosityIndicator, WongJansen; <param> = kappa or u_inf) -> set_blending_coeff.
//              "avcells:<kappa>:<factor>" / "blendcells:<type>:<param>": the cellwise values
//              only (the reference's cell-to-node transfer crashes on tetrahedral meshes);
//              "avfield:<file>" / "blendfield:<file>": a nodal field read from a raw array of
//              nsol doubles, handed to the solver.
//
// The only addition to the reference is the constant-direction advection policy below: the
// reference's ConstAdvection2D is hard-wired to a = (0,1) (physics/scalar/RotationAdvection2D.hpp:17-30),
// and RotationAdvection2D takes the direction as a template policy, so a new policy class is
// plugged in without editing the reference.

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "interpolation/FEValues.hpp"
#include "mesh/io/gmsh/GmshReader.hpp"
#include "mesh/point_set/StdPointSet.hpp"
#include "mesh/std_region/StdRegion.hpp"
#include "physics/euler/Euler2DCons.hpp"
#include "physics/euler/Euler3DCons.hpp"
#include "physics/scalar/Burgers2D.hpp"
#include "physics/scalar/RotationAdvection2D.hpp"
#include "solver/art_visc/ArtificialViscosity.hpp"
#include "solver/rdm/PGRDMethodExplicit.hpp"
#include "solver/rdm/assembly/PGRDMPicardJacCellAssemblyWorker.hpp"
#include "solver/rdm/blending_coeff/RDBlendingCoeff.hpp"
#include "solver/rdm/cellsplitters/CellSplitters.hpp"
#include "solver/time/ExplicitTimeStepper.hpp"

#include "ref_common.hpp"

using namespace pdekit;
using namespace pdekit::mesh;
using namespace pdekit::solver;

using vec_fn    = interpolation::VectorMeshFunction<Real>;
using namespace rds_oracle;

// ----------------------------------------------------------------------------
// Raw array output
// ----------------------------------------------------------------------------

struct Dumper
{
  std::string dir;
  std::ostringstream manifest;
  bool first = true;

  template <typename T>
  void put(const std::string &name, const std::vector<T> &v, const std::vector<Uint> &shape)
  {
    const std::string path = dir + "/" + name + (sizeof(T) == 8 ? ".f64" : ".i32");
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char *>(v.data()), v.size() * sizeof(T));
    manifest << (first ? "" : ",\n") << "  \"" << name << "\": [";
    for (Uint i = 0; i < shape.size(); ++i)
      manifest << (i ? ", " : "") << shape[i];
    manifest << "]";
    first = false;
  }
};

static std::vector<Real> mat_to_vec(const math::DenseDMat<Real> &m)
{
  std::vector<Real> v(m.rows() * m.cols());
  for (Uint r = 0; r < m.rows(); ++r)
    for (Uint c = 0; c < m.cols(); ++c)
      v[r * m.cols() + c] = m(r, c);
  return v;
}

// ----------------------------------------------------------------------------
// Probe subclass: the reference keeps the time-update object protected in RDMethod.
// ----------------------------------------------------------------------------

template <typename MC, typename Phys, typename Scheme>
class ProbeSolver : public rdm::PGRDMethodExplicit<MC, Phys, Scheme>
{
  public:
  const rdm::RDTimeUpdate &time_update() const
  {
    return this->m_rd_time_update;
  }
};

struct Args
{
  std::string mode, physics, scheme, mesh, outdir, init, bcspec, stab = "none";
  Uint p = 1, quad = 1, iters = 1, threads = 1;
  Real cfl = 0.5;
};

static ElemShape facet_shape_of(ElemShape s)
{
  if (s == ElemShape::Triag || s == ElemShape::Quad)
    return ElemShape::Line;
  return ElemShape::Triag;
}

template <typename MC, typename Phys, typename Scheme>
int run(const Args &a)
{
  using MeshType  = Tria<MC>;
  constexpr Uint D   = MC::GDIM;
  constexpr Uint NEQ = Phys::NEQ;

  auto mesh = std::make_shared<MeshType>("mesh");
  gmsh::GmshReader reader;
  reader.read_mesh_from_file(a.mesh, *mesh, "geo_dofs");
  auto geo = mesh->dof_storage("geo_dofs");
  auto sol = mesh->create_dof_storage("sol_dofs");
  MeshType::dof_storage_type::clone_continuous(*mesh, *geo, *sol, static_cast<PolyOrderID>(a.p),
                                               PointSetID::Equidist);

  const Uint nsol   = (*sol).nb_nodes();
  const Uint ncells = (*sol).nb_active_cells();

  auto u   = std::make_shared<vec_fn>("", "solution");
  auto res = std::make_shared<vec_fn>("", "residual");
  u->resize(NEQ, nsol);
  res->resize(NEQ, nsol);

  auto solver = std::make_shared<ProbeSolver<MC, Phys, Scheme>>();
  solver->configure_mesh_data(mesh, geo, sol);
  solver->initialize_work_data(SFunc::Lagrange, PointSetID::Gauss, a.quad, a.threads, 100);
  solver->set_vec_function(SolverVecFn::solution, u);
  solver->set_vec_function(SolverVecFn::residuals, res);

  // ---- boundary conditions: "Type:cond_name:boundary:expr,..."
  struct BCDesc
  {
    std::string type, name, boundary, expr;
  };
  std::vector<BCDesc> bcs;
  if (a.bcspec != "none")
  {
    std::stringstream ss(a.bcspec);
    std::string item;
    while (std::getline(ss, item, ','))
    {
      BCDesc b;
      std::stringstream is(item);
      std::getline(is, b.type, ':');
      std::getline(is, b.name, ':');
      std::getline(is, b.boundary, ':');
      std::getline(is, b.expr, ':');
      bcs.push_back(b);
    }
  }
  for (const BCDesc &b : bcs)
  {
    auto bc = solver->add_boundary_condition(b.type, b.name, b.boundary);
    if (b.expr.rfind("state=", 0) == 0)
    {
      // "state=v0|v1|..." : the reference state of WeakFarfield (set_reference_state)
      std::vector<Real> vals;
      std::stringstream vs(b.expr.substr(6));
      std::string v;
      while (std::getline(vs, v, '|'))
        vals.push_back(std::atof(v.c_str()));
      math::DenseDVec<Real> st(vals.size());
      for (Uint i = 0; i < vals.size(); ++i)
        st[i] = vals[i];
      bc->set_reference_state(st);
    }
    else if (b.expr.find('=') != std::string::npos)
    {
      // parameters "name=value;name=value" (WeakSubInlet / WeakSubOutlet)
      std::stringstream ps(b.expr);
      std::string kv;
      while (std::getline(ps, kv, ';'))
      {
        const size_t eq = kv.find('=');
        bc->set_parameter(kv.substr(0, eq), std::atof(kv.substr(eq + 1).c_str()));
      }
    }
    else if (!b.expr.empty() && b.expr != "-")
      bc->set_expression(find_expr(b.expr));
  }

  // ---- element types: (solution point set, geometry point set) pairs in order of first
  // appearance among the active cells; every type keeps its cells in ascending active-cell
  // order (mixed meshes, e.g. triangles + quadrilaterals, dump one table set per type)
  struct CellType
  {
    PointSetTag sol_tag, geo_tag;
    std::vector<Uint> cells;
  };
  std::vector<CellType> types;
  for (Uint c = 0; c < ncells; ++c)
  {
    const PointSetTag st = (*sol).active_cell(ActiveIdx(c)).pt_set_id();
    const PointSetTag gt = (*geo).active_cell(ActiveIdx(c)).pt_set_id();
    Uint k               = 0;
    while (k < types.size() && (types[k].sol_tag != st || types[k].geo_tag != gt))
      ++k;
    if (k == types.size())
      types.push_back({st, gt, {}});
    types[k].cells.push_back(c);
  }
  const ElemShape shape  = types[0].sol_tag.elem_shape();
  const Uint geo_order   = types[0].geo_tag.poly_order();
  const ElemShape fshape = facet_shape_of(shape);
  for (const CellType &t : types)
    if (facet_shape_of(t.sol_tag.elem_shape()) != fshape || t.geo_tag.poly_order() != geo_order)
    {
      std::cerr << "dump mode needs one facet shape and one geometry order" << std::endl;
      return 2;
    }

  // ---- geometry nodes (coordinates indexed by geometry dof id)
  const Uint ngeo_nodes = (*geo).nb_nodes();
  std::vector<Real> geo_coords(ngeo_nodes * D, 0.0);
  for (Uint c = 0; c < ncells; ++c)
  {
    const MeshEntity gc = (*geo).active_cell(ActiveIdx(c));
    const auto coords   = mesh->active_cell(ActiveIdx(c)).coordinates();
    for (Uint v = 0; v < gc.nb_vert(); ++v)
    {
      const auto node = coords.const_node_view(v);
      for (Uint d = 0; d < D; ++d)
        geo_coords[gc.vertex(v) * D + d] = node[d];
    }
  }

  // Facet tables (boundary quadrature order = cell quadrature order + 1,
  // solver/rdm/bc/RDMBCBase.hpp:261-263)
  StdPointSet fquad;
  fquad.change_type(fshape, a.quad + 1, PointSetID::Gauss);
  const math::DenseDMat<Real> &fqp = fquad.get().coordinates();
  const math::DenseDVec<Real> &fqw = fquad.get().weights();
  interpolation::FEValues fe_fsol, fe_fgeo;
  fe_fsol.configure(PointSetTag(fshape, a.p, PointSetID::Equidist),
                    sf::SFTag(fshape, SFunc::Lagrange, a.p, ModalBasis::Modal));
  fe_fsol.fill_Vandermonde(fqp, fqw);
  fe_fgeo.configure(PointSetTag(fshape, geo_order, PointSetID::Equidist),
                    sf::SFTag(fshape, SFunc::Lagrange, geo_order, ModalBasis::Modal));
  fe_fgeo.fill_Vandermonde(fqp, fqw);

  // ---- initial state from coordinates of solution dofs (geometry basis at the solution nodes
  // of each cell, so mixed meshes work too)
  const std::vector<Real> sol_coords = solution_node_coords(*mesh, *geo, *sol, D);
  std::vector<Real> u0(nsol * NEQ);
  for (Uint i = 0; i < nsol; ++i)
  {
    init_state(a.init, &sol_coords[i * D], D, NEQ, &u0[i * NEQ]);
    auto e = u->value(i);
    for (Uint k = 0; k < NEQ; ++k)
      e[k] = u0[i * NEQ + k];
  }

  auto grab = [&](const vec_fn &f) {
    std::vector<Real> v(nsol * NEQ);
    for (Uint i = 0; i < nsol; ++i)
    {
      const auto e = f.const_value(i);
      for (Uint k = 0; k < NEQ; ++k)
        v[i * NEQ + k] = e[k];
    }
    return v;
  };
  auto grab_scalar = [&](const interpolation::ScalarMeshFunction<Real> &f) {
    std::vector<Real> v(nsol);
    for (Uint i = 0; i < nsol; ++i)
      v[i] = f[i];
    return v;
  };

  // ---- stabilisation field at u0 (optional)
  using scal_fn = interpolation::ScalarMeshFunction<Real>;
  std::vector<std::pair<std::string, std::vector<Real>>> stab_arrays;
  std::shared_ptr<scal_fn> stab_nodal;
  auto cells_of = [&](const scal_fn &f) {
    std::vector<Real> v(ncells);
    for (Uint c = 0; c < ncells; ++c)
      v[c] = f[c];
    return v;
  };
  if (a.stab != "none")
  {
    std::vector<std::string> tok;
    std::stringstream ts(a.stab);
    std::string t;
    while (std::getline(ts, t, ':'))
      tok.push_back(t);
    const bool field = tok.size() == 2 && (tok[0] == "avfield" || tok[0] == "blendfield");
    const bool ok3   = tok.size() == 3 && (tok[0] == "av" || tok[0] == "blend" ||
                                         tok[0] == "avcells" || tok[0] == "blendcells");
    if (!field && !ok3)
    {
      std::cerr << "bad stab spec " << a.stab << std::endl;
      return 2;
    }
    stab_nodal = std::make_shared<scal_fn>("", "stab_nodal");
    stab_nodal->resize(nsol);
    scal_fn cellwise("", "cellwise");
    cellwise.resize(ncells);
    if (field)
    {
      std::ifstream fin(tok[1], std::ios::binary);
      std::vector<Real> vals(nsol);
      fin.read(reinterpret_cast<char *>(vals.data()), nsol * sizeof(Real));
      if (!fin)
      {
        std::cerr << "cannot read " << nsol << " values from " << tok[1] << std::endl;
        return 2;
      }
      for (Uint i = 0; i < nsol; ++i)
        (*stab_nodal)[i] = vals[i];
      if (tok[0] == "avfield")
      {
        stab_arrays.push_back({"av_nodal", vals});
        solver->set_artificial_viscosity(stab_nodal);
      }
      else
      {
        stab_arrays.push_back({"blend_nodal", vals});
        solver->set_blending_coeff(stab_nodal);
      }
    }
    else if (tok[0] == "av" || tok[0] == "avcells")
    {
      const Real kappa = std::atof(tok[1].c_str()), factor = std::atof(tok[2].c_str());
      solver::ArtificialViscosity<MC> op;
      op.prepare_indicator_operators(*sol);
      op.compute_artificial_viscosity(*sol, *u, cellwise, kappa, factor);
      stab_arrays.push_back({"av_cell", cells_of(cellwise)});
      op.compute_indicator_normalized(*sol, *u, cellwise, kappa);
      stab_arrays.push_back({"indicator", cells_of(cellwise)});
      if (tok[0] == "av")
      {
          op.compute_artificial_viscosity_nodal(*mesh, *sol, *u, *stab_nodal, kappa, factor);
        stab_arrays.push_back({"av_nodal", grab_scalar(*stab_nodal)});
        solver->set_artificial_viscosity(stab_nodal);
      }
    }
    else
    {
      solver::rdm::RDBlendingCoeff<MC> op;
      op.setup(*sol, tok[1]);
      op.set_param(tok[1] == "WongJansen" ? "u_inf" : "kappa", std::atof(tok[2].c_str()));
      op.calculate_in_cells(*mesh, *sol, *u, cellwise);
      stab_arrays.push_back({"blend_cell", cells_of(cellwise)});
      if (tok[0] == "blend")
      {
        op.calculate(*mesh, *sol, *u, *stab_nodal);
        stab_arrays.push_back({"blend_nodal", grab_scalar(*stab_nodal)});
        solver->set_blending_coeff(stab_nodal);
      }
    }
  }

  if (a.mode == "time")
  {
    solver->assemble_lhs_and_rhs(a.cfl); // warm-up
    const auto t0 = std::chrono::steady_clock::now();
    for (Uint it = 0; it < a.iters; ++it)
    {
      solver->assemble_lhs_and_rhs(a.cfl);
      solver->solve({});
    }
    const double s =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    math::DenseDVec<Real> nrm(NEQ);
    solver->compute_residual_norm(nrm);
    std::printf("{\"cells\": %u, \"nodes\": %u, \"iters\": %u, \"threads\": %u, \"seconds\": %.9g, "
                "\"cell_updates_per_s\": %.9g, \"norm0\": %.17g}\n",
                ncells, nsol, a.iters, a.threads, s, double(ncells) * a.iters / s, nrm[0]);
    return 0;
  }

  // ---- dump mode
  mkdir(a.outdir.c_str(), 0755);
  Dumper out;
  out.dir = a.outdir;

  out.put("geo_coords", geo_coords, {ngeo_nodes, D});
  out.put("sol_coords", sol_coords, {nsol, D});

  // ---- per element type: connectivity (reference dof order) and the reference-element tables,
  // built through the reference's own classes. A single-type mesh keeps the plain array names;
  // the types of a mixed mesh get the suffix _t<k> and are listed under "groups" in meta.json.
  std::ostringstream groupmeta;
  Uint nq = 0, nfl = 0, ndof = 0, ngeo = 0;
  for (Uint k = 0; k < types.size(); ++k)
  {
    const CellType &t       = types[k];
    const std::string sfx   = types.size() > 1 ? "_t" + std::to_string(k) : "";
    const ElemShape tshape  = t.sol_tag.elem_shape();
    const Uint tcells       = t.cells.size();
    const Uint tndof        = (*sol).active_cell(ActiveIdx(t.cells[0])).nb_vert();
    const Uint tngeo        = (*geo).active_cell(ActiveIdx(t.cells[0])).nb_vert();
    std::vector<int> gconn(tcells * tngeo), sconn(tcells * tndof);
    for (Uint i = 0; i < tcells; ++i)
    {
      const MeshEntity gc = (*geo).active_cell(ActiveIdx(t.cells[i]));
      const MeshEntity sc = (*sol).active_cell(ActiveIdx(t.cells[i]));
      for (Uint v = 0; v < tngeo; ++v)
        gconn[i * tngeo + v] = gc.vertex(v);
      for (Uint n = 0; n < tndof; ++n)
        sconn[i * tndof + n] = sc.vertex(n);
    }
    out.put("geo_conn" + sfx, gconn, {tcells, tngeo});
    out.put("sol_conn" + sfx, sconn, {tcells, tndof});

    StdPointSet quad;
    quad.change_type(tshape, a.quad, PointSetID::Gauss);
    const math::DenseDMat<Real> &qp = quad.get().coordinates();
    const math::DenseDVec<Real> &qw = quad.get().weights();
    const Uint tnq                  = qp.rows();

    interpolation::FEValues fe_sol, fe_geo, fe_flux, fe_sol_at_flux, fe_geo_at_flux;
    fe_sol.configure(PointSetTag(tshape, a.p, PointSetID::Equidist),
                     sf::SFTag(tshape, SFunc::Lagrange, a.p, ModalBasis::Modal));
    fe_sol.fill_Vandermonde(qp, qw);
    fe_geo.configure(PointSetTag(tshape, geo_order, PointSetID::Equidist),
                     sf::SFTag(tshape, SFunc::Lagrange, geo_order, ModalBasis::Modal));
    fe_geo.fill_Vandermonde(qp, qw);
    fe_flux.configure(PointSetTag(tshape, a.p + 1, PointSetID::Equidist),
                      sf::SFTag(tshape, SFunc::Lagrange, a.p + 1, ModalBasis::Modal));
    fe_flux.fill_Vandermonde(qp, qw);

    StdRegion flux_region;
    flux_region.change_type(PointSetTag(tshape, a.p + 1, PointSetID::Equidist));
    const math::DenseDMat<Real> &flux_nodes = flux_region.get().coordinates();
    const Uint tnfl                         = flux_nodes.rows();
    math::DenseDVec<Real> dummy_w(tnfl);
    dummy_w.fill(1.0);
    fe_sol_at_flux.configure(PointSetTag(tshape, a.p, PointSetID::Equidist),
                             sf::SFTag(tshape, SFunc::Lagrange, a.p, ModalBasis::Modal));
    fe_sol_at_flux.fill_Vandermonde(flux_nodes, dummy_w);
    fe_geo_at_flux.configure(PointSetTag(tshape, geo_order, PointSetID::Equidist),
                             sf::SFTag(tshape, SFunc::Lagrange, geo_order, ModalBasis::Modal));
    fe_geo_at_flux.fill_Vandermonde(flux_nodes, dummy_w);

    StdRegion sol_region;
    sol_region.change_type(PointSetTag(tshape, a.p, PointSetID::Equidist));
    const math::DenseDMat<Real> &sol_nodes = sol_region.get().coordinates();

    out.put("qp" + sfx, mat_to_vec(qp), {tnq, qp.cols()});
    std::vector<Real> w(tnq);
    for (Uint q = 0; q < tnq; ++q)
      w[q] = qw[q];
    out.put("w" + sfx, w, {tnq});
    out.put("V" + sfx, mat_to_vec(fe_sol.Vandermonde()), {tnq, tndof});
    out.put("Vgeo" + sfx, mat_to_vec(fe_geo.Vandermonde()), {tnq, tngeo});
    out.put("Vf" + sfx, mat_to_vec(fe_flux.Vandermonde()), {tnq, tnfl});
    out.put("Vsf" + sfx, mat_to_vec(fe_sol_at_flux.Vandermonde()), {tnfl, tndof});
    out.put("Vgf" + sfx, mat_to_vec(fe_geo_at_flux.Vandermonde()), {tnfl, tngeo});
    for (Uint d = 0; d < D; ++d)
    {
      const std::string s = std::to_string(d);
      out.put("dV" + s + sfx, mat_to_vec(fe_sol.deriv_Vandermonde(d)), {tnq, tndof});
      out.put("dVgeo" + s + sfx, mat_to_vec(fe_geo.deriv_Vandermonde(d)), {tnq, tngeo});
      out.put("dVf" + s + sfx, mat_to_vec(fe_flux.deriv_Vandermonde(d)), {tnq, tnfl});
      out.put("dVgf" + s + sfx, mat_to_vec(fe_geo_at_flux.deriv_Vandermonde(d)), {tnfl, tngeo});
      out.put("dVsf" + s + sfx, mat_to_vec(fe_sol_at_flux.deriv_Vandermonde(d)), {tnfl, tndof});
    }
    out.put("flux_nodes" + sfx, mat_to_vec(flux_nodes), {tnfl, flux_nodes.cols()});
    out.put("sol_nodes" + sfx, mat_to_vec(sol_nodes), {tndof, sol_nodes.cols()});

    // dual-volume rule: Gauss rule of the cell's own order (RDTimeUpdate.hpp:85-150)
    StdPointSet vquad;
    vquad.change_type(tshape, a.p, PointSetID::Gauss);
    const math::DenseDMat<Real> &vqp = vquad.get().coordinates();
    const math::DenseDVec<Real> &vqw = vquad.get().weights();
    interpolation::FEValues fe_vgeo;
    fe_vgeo.configure(PointSetTag(tshape, geo_order, PointSetID::Equidist),
                      sf::SFTag(tshape, SFunc::Lagrange, geo_order, ModalBasis::Modal));
    fe_vgeo.fill_Vandermonde(vqp, vqw);
    std::vector<Real> vw(vqp.rows());
    for (Uint q = 0; q < vqp.rows(); ++q)
      vw[q] = vqw[q];
    out.put("vqp" + sfx, mat_to_vec(vqp), {vqp.rows(), vqp.cols()});
    out.put("vw" + sfx, vw, {vqp.rows()});
    for (Uint d = 0; d < D; ++d)
      out.put("vdVgeo" + std::to_string(d) + sfx, mat_to_vec(fe_vgeo.deriv_Vandermonde(d)),
              {vqp.rows(), tngeo});

    const char *tname = tshape == ElemShape::Triag   ? "triag"
                        : tshape == ElemShape::Quad  ? "quad"
                        : tshape == ElemShape::Tetra ? "tetra"
                                                     : "other";
    groupmeta << (k ? ", " : "") << "{\"shape\": \"" << tname << "\", \"suffix\": \"" << sfx
              << "\", \"ncells\": " << tcells << ", \"ndof\": " << tndof << ", \"ngeo\": "
              << tngeo << ", \"nq\": " << tnq << ", \"nfl\": " << tnfl << "}";
    if (k == 0)
    {
      nq   = tnq;
      nfl  = tnfl;
      ndof = tndof;
      ngeo = tngeo;
    }
  }

  const Uint nfq = fqp.rows();
  out.put("fqp", mat_to_vec(fqp), {nfq, fqp.cols()});
  std::vector<Real> fw(nfq);
  for (Uint q = 0; q < nfq; ++q)
    fw[q] = fqw[q];
  out.put("fw", fw, {nfq});
  out.put("fV", mat_to_vec(fe_fsol.Vandermonde()), {nfq, fe_fsol.nb_nodes()});
  out.put("fVgeo", mat_to_vec(fe_fgeo.Vandermonde()), {nfq, fe_fgeo.nb_nodes()});
  for (Uint d = 0; d + 1 < D; ++d)
    out.put("fdVgeo" + std::to_string(d), mat_to_vec(fe_fgeo.deriv_Vandermonde(d)),
            {nfq, fe_fgeo.nb_nodes()});

  // ---- boundary facets in the order the weak BCs traverse them (WeakBC.hpp:227-360)
  std::ostringstream bcmeta;
  for (Uint ib = 0; ib < bcs.size(); ++ib)
  {
    const auto &bdry = *(mesh->all_boundaries().domain(bcs[ib].boundary));
    using dof_it     = typename BoundaryFacets<MC, D - 1>::const_dof_iterator_typed;
    std::vector<common::IteratorRange<dof_it>> sranges, granges;
    bdry.all_bdry_dof_ranges(*sol, sranges);
    bdry.all_bdry_dof_ranges(*geo, granges);
    std::vector<int> fsol, fgeo;
    Uint nfsol = 0, nfgeo = 0, nfac = 0;
    for (Uint r = 0; r < sranges.size(); ++r)
    {
      auto git = granges[r].begin();
      for (auto it = sranges[r].begin(); it != sranges[r].end(); ++it, ++git)
      {
        const MeshEntity se = it->mesh_entity();
        const MeshEntity ge = git->mesh_entity();
        nfsol               = se.nb_vert();
        nfgeo               = ge.nb_vert();
        for (Uint n = 0; n < se.nb_vert(); ++n)
          fsol.push_back(se.vertex(n));
        for (Uint n = 0; n < ge.nb_vert(); ++n)
          fgeo.push_back(ge.vertex(n));
        nfac++;
      }
    }
    out.put("bc" + std::to_string(ib) + "_sol", fsol, {nfac, nfsol});
    out.put("bc" + std::to_string(ib) + "_geo", fgeo, {nfac, nfgeo});
    bcmeta << (ib ? ", " : "") << "{\"type\": \"" << bcs[ib].type << "\", \"name\": \""
           << bcs[ib].name << "\", \"boundary\": \"" << bcs[ib].boundary << "\", \"expr\": \""
           << bcs[ib].expr << "\", \"nfacets\": " << nfac << "}";
  }

  out.put("u0", u0, {nsol, NEQ});
  for (const auto &sa : stab_arrays)
    out.put(sa.first, sa.second, {Uint(sa.second.size())});

  // ---- (RDS_HARNESS_JACOBIAN set) the reference's Picard-linearised implicit assembly at u0:
  // its cell worker (solver/rdm/assembly/PGRDMPicardJacCellAssemblyWorker.hpp:120-490) computes
  // every cell's residual and element Jacobian with the scheme's compute_adv_res_and_jacobian
  // (PGLDA.hpp:316-536, PGN.hpp:296, PGB.hpp:503-819) and adds J(m, n) / V(m) to the system
  // matrix and -res(m) / V(m) to the right-hand side; the recording classes of
  // oracle/shim_jac/linear_system/TpetraFwd.hpp keep the summed entries. No Dirichlet rows.
  if (std::getenv("RDS_HARNESS_JACOBIAN"))
  {
    rdm::RDTimeUpdate tu;
    tu.setup(*mesh, *sol);
    rdm::detail::PGRDMPicardJacCellAssemblyWorker<MC, Phys, Scheme> worker(0);
    worker.configure_cell_spaces(*mesh, *sol, 0, ncells - 1, 100, SFunc::Lagrange,
                                 PointSetID::Gauss, a.quad);
    const std::vector<bool> no_dirichlet(nsol * NEQ, false);
    ls::TpetraCrsMatrix<Real> mat;
    ls::TpetraMultiVector<Real> rhs;
    rhs.values.assign(nsol * NEQ, 0.0);
    worker.assemble_mat_and_rhs_part(*mesh, *sol, *u, tu, no_dirichlet, mat, rhs);
    std::vector<int> jrow, jcol;
    std::vector<Real> jval;
    for (const auto &e : mat.entries)
    {
      jrow.push_back(int(e.first.first));
      jcol.push_back(int(e.first.second));
      jval.push_back(e.second);
    }
    out.put("jac_row", jrow, {Uint(jrow.size())});
    out.put("jac_col", jcol, {Uint(jcol.size())});
    out.put("jac_val", jval, {Uint(jval.size())});
    out.put("jac_rhs", rhs.values, {nsol, NEQ});
  }

  // first iteration: residual, wave speed, dt, dual volume at u0
  solver->assemble_lhs_and_rhs(a.cfl);
  out.put("res1", grab(*res), {nsol, NEQ});
  // the state the update starts from: StrongDirichlet conditions overwrite their facet dofs
  // during assemble (bc/StrongDirichletBC.hpp:202-233)
  out.put("ua1", grab(*u), {nsol, NEQ});
  out.put("ws1", grab_scalar(solver->time_update().nodal_wave_speed()), {nsol});
  out.put("dt1", grab_scalar(*solver->scal_function(SolverScalFn::time_step)), {nsol});
  out.put("dual_volume", grab_scalar(solver->time_update().nodal_dual_volume()), {nsol});
  math::DenseDVec<Real> nrm(NEQ);
  solver->compute_residual_norm(nrm);
  std::vector<Real> norms;
  for (Uint k = 0; k < NEQ; ++k)
    norms.push_back(nrm[k]);
  solver->solve({});
  out.put("u1", grab(*u), {nsol, NEQ});

  for (Uint it = 1; it < a.iters; ++it)
  {
    solver->assemble_lhs_and_rhs(a.cfl);
    solver->compute_residual_norm(nrm);
    for (Uint k = 0; k < NEQ; ++k)
      norms.push_back(nrm[k]);
    solver->solve({});
  }
  out.put("uK", grab(*u), {nsol, NEQ});
  out.put("norms", norms, {Uint(norms.size() / NEQ), NEQ});

  // two steps of the reference's third-order TVD Runge-Kutta stepper from u0
  // (solver/time/ExplicitTimeStepper.cpp:66-100): the state, the residual of the last step's
  // first stage, the time step of that stage and the residual norm after each step
  // (left out when RDS_HARNESS_NO_RK3 is set: six more assemblies on large meshes)
  const bool with_rk3 = std::getenv("RDS_HARNESS_NO_RK3") == nullptr;
  for (Uint i = 0; i < nsol && with_rk3; ++i)
  {
    auto e = u->value(i);
    for (Uint k = 0; k < NEQ; ++k)
      e[k] = u0[i * NEQ + k];
  }
  if (with_rk3)
  {
    time::RK3TVD rk3;
    rk3.setup(NEQ, nsol);
    std::vector<Real> rk_norms;
    for (Uint step = 0; step < 2; ++step)
    {
      rk3.advance_in_time(*solver, a.cfl);
      solver->compute_residual_norm(nrm);
      for (Uint k = 0; k < NEQ; ++k)
        rk_norms.push_back(nrm[k]);
    }
    out.put("u_rk3", grab(*u), {nsol, NEQ});
    out.put("res_rk3", grab(*res), {nsol, NEQ});
    out.put("dt_rk3", grab_scalar(*solver->scal_function(SolverScalFn::time_step)), {nsol});
    out.put("norms_rk3", rk_norms, {2, NEQ});
  }

  const char *shape_name = shape == ElemShape::Triag   ? "triag"
                           : shape == ElemShape::Quad  ? "quad"
                           : shape == ElemShape::Tetra ? "tetra"
                                                       : "other";
  std::ofstream meta(a.outdir + "/meta.json");
  meta.precision(17);
  meta << "{\n \"physics\": \"" << a.physics << "\", \"scheme\": \"" << a.scheme
       << "\", \"p\": " << a.p << ", \"quad\": " << a.quad << ", \"shape\": \"" << shape_name
       << "\", \"dim\": " << D << ", \"neq\": " << NEQ << ",\n \"ncells\": " << ncells
       << ", \"nsol\": " << nsol << ", \"ngeo_nodes\": " << ngeo_nodes << ", \"ndof\": " << ndof
       << ", \"ngeo\": " << ngeo << ", \"nq\": " << nq << ", \"nfl\": " << nfl
       << ", \"nfq\": " << nfq << ",\n \"iters\": " << a.iters << ", \"cfl\": " << a.cfl
       << ", \"init\": \"" << a.init << "\", \"stab\": \"" << a.stab
       << "\",\n \"groups\": [" << groupmeta.str() << "]"
       << ",\n \"bcs\": [" << bcmeta.str()
       << "],\n \"arrays\": {\n"
       << out.manifest.str() << "\n }\n}\n";
  return 0;
}

int main(int argc, char **argv)
{
  if (argc < 12)
  {
    std::fprintf(stderr, "usage: %s dump|time physics scheme p quad mesh outdir iters cfl init "
                         "bcspec [threads] [stab]\n",
                 argv[0]);
    return 2;
  }
  Args a;
  a.mode    = argv[1];
  a.physics = argv[2];
  a.scheme  = argv[3];
  a.p       = std::atoi(argv[4]);
  a.quad    = std::atoi(argv[5]);
  a.mesh    = argv[6];
  a.outdir  = argv[7];
  a.iters   = std::atoi(argv[8]);
  a.cfl     = std::atof(argv[9]);
  a.init    = argv[10];
  a.bcspec  = argv[11];
  a.threads = argc > 12 ? std::atoi(argv[12]) : 1;
  if (argc > 13)
    a.stab = argv[13];

  using Adv   = physics::RotationAdvection2D<ConstDirection2D>;
  using Burg  = physics::Burgers2D;
  using Eul2D = physics::Euler2DCons;
  using Eul3D = physics::Euler3DCons;

#define DISPATCH(PHYS_NAME, MC, PHYS)                                                              \
  if (a.physics == PHYS_NAME)                                                                      \
  {                                                                                                \
    if (a.scheme == "lda")                                                                         \
      return run<MC, PHYS, solver::rdm::PGLDA>(a);                                                 \
    if (a.scheme == "n")                                                                           \
      return run<MC, PHYS, solver::rdm::PGN>(a);                                                   \
    if (a.scheme == "b")                                                                           \
      return run<MC, PHYS, solver::rdm::PGB>(a);                                                   \
  }

  DISPATCH("advconst", Cart2D, Adv)
  DISPATCH("burgers", Cart2D, Burg)
  DISPATCH("euler2d", Cart2D, Eul2D)
  DISPATCH("euler3d", Cart3D, Eul3D)
#undef DISPATCH

  std::fprintf(stderr, "unknown physics/scheme %s/%s\n", a.physics.c_str(), a.scheme.c_str());
  return 2;
}
