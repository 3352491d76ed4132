// Side-by-side check of the drop-in GPU solver against the reference's own CPU solver.
//
// Builds the same mesh, dofs, weak conditions and initial state for
//   PGRDMethodExplicit<MeshConfig, Physics, Scheme>      (reference, CPU, one thread)
//   GpuPGRDMethodExplicit<MeshConfig, Physics, Scheme>   (include/pdekit_b200, librds_b200 on the GPU)
// through the same public calls (configure_mesh_data, initialize_work_data, set_vec_function,
// add_boundary_condition + set_expression / set_parameter, assemble_lhs_and_rhs, solve,
// compute_residual_norm), runs K iterations of each and prints one JSON line with the largest
// differences: residual and time step after the first assembly (normalised by the reference's
// largest magnitude), the state after K iterations, the state after the drop-in's device loop
// (iterate), the residual norms, and the state after two RK3TVD steps (device stages, and the
// reference's own stepper class driving the drop-in, and the drop-in stepper GpuRK3TVD).
//
// usage: dropin_test <advconst|burgers|euler2d|euler3d> <lda|n|b> <p> <quad> <mesh.msh> <iters>
//                    <cfl> <init> <bcspec> [stab]
//   stab: "av:<kappa>:<factor>" / "blend:<type>:<param>" -- each solver gets a nodal
//   stabilisation field (set_artificial_viscosity / set_blending_coeff) that the reference's own
//   operator recomputes in place from that solver's state before the first and every second
//   iteration, as examples/testcases-rdm/Burgers-RDS-2D.cpp:224-229 does (the device loop is
//   then not compared: its field stays fixed).
// Test infrastructure: linked with the reference sources compiled in place (oracle/Makefile).

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <functional>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "mesh/io/gmsh/GmshReader.hpp"
#include "solver/art_visc/ArtificialViscosity.hpp"
#include "solver/rdm/PGRDMethodExplicit.hpp"
#include "solver/rdm/blending_coeff/RDBlendingCoeff.hpp"
#include "solver/time/ExplicitTimeStepper.hpp"

#include "pdekit_b200/GpuRK3TVD.hpp"

#include "pdekit_b200/GpuPGRDMethodExplicit.hpp"
#include "ref_common.hpp"

using namespace pdekit;
using namespace pdekit::mesh;
using namespace pdekit::solver;
using namespace rds_oracle;

using vec_fn = interpolation::VectorMeshFunction<Real>;

struct Args
{
  std::string physics, scheme, mesh, init, bcspec, stab = "none";
  Uint p = 1, quad = 1, iters = 1;
  Real cfl = 0.5;
};

template <typename Solver>
void add_bcs(Solver &s, const std::string &spec)
{
  if (spec == "none")
    return;
  std::stringstream ss(spec);
  std::string item;
  while (std::getline(ss, item, ','))
  {
    std::string type, name, boundary, expr;
    std::stringstream is(item);
    std::getline(is, type, ':');
    std::getline(is, name, ':');
    std::getline(is, boundary, ':');
    std::getline(is, expr, ':');
    auto bc = s.add_boundary_condition(type, name, boundary);
    if (expr.rfind("state=", 0) == 0)
    {
      // WeakFarfield reference state "state=v0|v1|..."
      std::vector<double> vals;
      std::stringstream vs(expr.substr(6));
      std::string v;
      while (std::getline(vs, v, '|'))
        vals.push_back(std::atof(v.c_str()));
      math::DenseDVec<Real> st(vals.size());
      for (Uint i = 0; i < vals.size(); ++i)
        st[i] = vals[i];
      bc->set_reference_state(st);
    }
    else if (expr.find('=') != std::string::npos)
    {
      std::stringstream ps(expr);
      std::string kv;
      while (std::getline(ps, kv, ';'))
      {
        const size_t eq = kv.find('=');
        bc->set_parameter(kv.substr(0, eq), std::atof(kv.substr(eq + 1).c_str()));
      }
    }
    else if (!expr.empty() && expr != "-")
      bc->set_expression(find_expr(expr));
  }
}

static double max_abs(const std::vector<double> &a)
{
  double m = 0.0;
  for (double x : a)
    m = std::max(m, std::fabs(x));
  return m;
}

static double max_diff(const std::vector<double> &a, const std::vector<double> &b)
{
  double m = 0.0;
  for (size_t i = 0; i < a.size(); ++i)
    m = std::max(m, std::fabs(a[i] - b[i]));
  return m;
}

template <typename MC, typename Phys, typename Scheme>
int run(const Args &a)
{
  using MeshType     = Tria<MC>;
  constexpr Uint D   = MC::GDIM;
  constexpr Uint NEQ = Phys::NEQ;

  auto mesh = std::make_shared<MeshType>("mesh");
  gmsh::GmshReader reader;
  reader.read_mesh_from_file(a.mesh, *mesh, "geo_dofs");
  auto geo = mesh->dof_storage("geo_dofs");
  auto sol = mesh->create_dof_storage("sol_dofs");
  MeshType::dof_storage_type::clone_continuous(*mesh, *geo, *sol, static_cast<PolyOrderID>(a.p),
                                               PointSetID::Equidist);
  const Uint nsol = (*sol).nb_nodes();

  auto u_ref = std::make_shared<vec_fn>("", "solution");
  auto r_ref = std::make_shared<vec_fn>("", "residual");
  auto u_gpu = std::make_shared<vec_fn>("", "solution");
  auto r_gpu = std::make_shared<vec_fn>("", "residual");
  for (auto f : {u_ref, r_ref, u_gpu, r_gpu})
    f->resize(NEQ, nsol);

  const std::vector<Real> xy = solution_node_coords(*mesh, *geo, *sol, D);
  std::vector<Real> u0(nsol * NEQ);
  for (Uint i = 0; i < nsol; ++i)
    init_state(a.init, &xy[i * D], D, NEQ, &u0[i * NEQ]);
  auto load = [&](vec_fn &f) {
    for (Uint i = 0; i < nsol; ++i)
      for (Uint e = 0; e < NEQ; ++e)
        f.value(i)[e] = u0[i * NEQ + e];
  };
  auto grab = [&](const vec_fn &f) {
    std::vector<double> v(nsol * NEQ);
    for (Uint i = 0; i < nsol; ++i)
      for (Uint e = 0; e < NEQ; ++e)
        v[i * NEQ + e] = f.const_value(i)[e];
    return v;
  };
  load(*u_ref);
  load(*u_gpu);

  rdm::PGRDMethodExplicit<MC, Phys, Scheme> ref;
  rdm::GpuPGRDMethodExplicit<MC, Phys, Scheme> gpu;
  ref.configure_mesh_data(mesh, geo, sol);
  gpu.configure_mesh_data(mesh, geo, sol);
  ref.initialize_work_data(SFunc::Lagrange, PointSetID::Gauss, a.quad, 1, 100);
  gpu.initialize_work_data(SFunc::Lagrange, PointSetID::Gauss, a.quad, 1, 100);
  ref.set_vec_function(SolverVecFn::solution, u_ref);
  ref.set_vec_function(SolverVecFn::residuals, r_ref);
  gpu.set_vec_function(SolverVecFn::solution, u_gpu);
  gpu.set_vec_function(SolverVecFn::residuals, r_gpu);
  add_bcs(ref, a.bcspec);
  add_bcs(gpu, a.bcspec);

  // stabilisation field per solver, recomputed in place by the reference's operator
  using scal_fn = interpolation::ScalarMeshFunction<Real>;
  auto f_ref    = std::make_shared<scal_fn>("", "stab");
  auto f_gpu    = std::make_shared<scal_fn>("", "stab");
  f_ref->resize(nsol);
  f_gpu->resize(nsol);
  std::function<void(const vec_fn &, scal_fn &)> compute;
  std::shared_ptr<solver::ArtificialViscosity<MC>> av_op;
  std::shared_ptr<solver::rdm::RDBlendingCoeff<MC>> bl_op;
  if (a.stab != "none")
  {
    std::vector<std::string> tok;
    std::stringstream ts(a.stab);
    std::string t;
    while (std::getline(ts, t, ':'))
      tok.push_back(t);
    if (tok.size() != 3)
      return 2;
    const Real p0 = std::atof(tok[1].c_str()), p1 = std::atof(tok[2].c_str());
    if (tok[0] == "av")
    {
      av_op = std::make_shared<solver::ArtificialViscosity<MC>>();
      av_op->prepare_indicator_operators(*sol);
      compute = [&, p0, p1](const vec_fn &u, scal_fn &f) {
        av_op->compute_artificial_viscosity_nodal(*mesh, *sol, u, f, p0, p1);
      };
      ref.set_artificial_viscosity(f_ref);
      gpu.set_artificial_viscosity(f_gpu);
    }
    else
    {
      bl_op = std::make_shared<solver::rdm::RDBlendingCoeff<MC>>();
      bl_op->setup(*sol, tok[1]);
      bl_op->set_param(tok[1] == "WongJansen" ? "u_inf" : "kappa", std::atof(tok[2].c_str()));
      compute = [&](const vec_fn &u, scal_fn &f) { bl_op->calculate(*mesh, *sol, u, f); };
      ref.set_blending_coeff(f_ref);
      gpu.set_blending_coeff(f_gpu);
    }
    compute(*u_ref, *f_ref);
    compute(*u_gpu, *f_gpu);
  }

  // first assembly
  ref.assemble_lhs_and_rhs(a.cfl);
  gpu.assemble_lhs_and_rhs(a.cfl);
  const std::vector<double> res_r = grab(*r_ref), res_g = grab(*r_gpu);
  std::vector<double> dt_r(nsol), dt_g(nsol);
  for (Uint i = 0; i < nsol; ++i)
  {
    dt_r[i] = (*ref.scal_function(SolverScalFn::time_step))[i];
    dt_g[i] = (*gpu.scal_function(SolverScalFn::time_step))[i];
  }
  math::DenseDVec<Real> n_r(NEQ), n_g(NEQ);
  ref.compute_residual_norm(n_r);
  gpu.compute_residual_norm(n_g);
  double norm_diff = 0.0;
  for (Uint e = 0; e < NEQ; ++e)
    norm_diff = std::max(norm_diff, std::fabs(n_r[e] - n_g[e]) / std::fabs(n_r[e]));
  ref.solve({});
  gpu.solve({});
  for (Uint it = 1; it < a.iters; ++it)
  {
    if (compute && it % 2 == 0)
    {
      compute(*u_ref, *f_ref);
      compute(*u_gpu, *f_gpu);
    }
    ref.assemble_lhs_and_rhs(a.cfl);
    ref.solve({});
    gpu.assemble_lhs_and_rhs(a.cfl);
    gpu.solve({});
  }
  const std::vector<double> uK_r = grab(*u_ref), uK_g = grab(*u_gpu);

  // the drop-in's device loop from the same initial state (without a recomputed field)
  std::vector<double> uL_g = uK_r;
  if (!compute)
  {
    load(*u_gpu);
    gpu.iterate(a.cfl, a.iters, 0.0);
    uL_g = grab(*u_gpu);
  }

  // two RK3TVD steps from the initial state (solver/time/ExplicitTimeStepper.cpp:66-100): the
  // reference's stepper on the reference solver, the drop-in's device stages, and the
  // reference's stepper driving the drop-in through the solver interface
  double rk3 = 0.0, rk3_class = 0.0;
  if (!compute)
  {
    load(*u_ref);
    time::RK3TVD rk_ref;
    rk_ref.setup(NEQ, nsol);
    rk_ref.advance_in_time(ref, a.cfl);
    rk_ref.advance_in_time(ref, a.cfl);
    const std::vector<double> uR = grab(*u_ref);
    load(*u_gpu);
    gpu.advance_rk3tvd(a.cfl, 2);
    const std::vector<double> uG = grab(*u_gpu);
    load(*u_gpu);
    time::RK3TVD rk_gpu;
    rk_gpu.setup(NEQ, nsol);
    rk_gpu.advance_in_time(gpu, a.cfl);
    rk_gpu.advance_in_time(gpu, a.cfl);
    const std::vector<double> uC = grab(*u_gpu);
    // the drop-in stepper class, through the stepper base class
    load(*u_gpu);
    std::unique_ptr<time::ExplicitTimeStepperBase> stepper(new time::GpuRK3TVD());
    stepper->setup(NEQ, nsol);
    stepper->advance_in_time(gpu, a.cfl);
    stepper->advance_in_time(gpu, a.cfl);
    const std::vector<double> uS = grab(*u_gpu);
    const double sr = std::max(max_abs(uR), 1e-300);
    rk3             = std::max(max_diff(uR, uG), max_diff(uR, uS)) / sr;
    rk3_class       = max_diff(uR, uC) / sr;
  }

  const double su = std::max(max_abs(uK_r), 1e-300);
  std::printf("{\"nodes\": %u, \"cells\": %u, \"iters\": %u, \"res1\": %.3e, \"dt1\": %.3e, "
              "\"norm1\": %.3e, \"uK\": %.3e, \"uK_loop\": %.3e, \"rk3\": %.3e, "
              "\"rk3_class\": %.3e, \"max_res\": %.6e}\n",
              nsol, (*sol).nb_active_cells(), a.iters,
              max_diff(res_r, res_g) / std::max(max_abs(res_r), 1e-300),
              max_diff(dt_r, dt_g) / std::max(max_abs(dt_r), 1e-300), norm_diff,
              max_diff(uK_r, uK_g) / su, max_diff(uK_r, uL_g) / su, rk3, rk3_class,
              max_abs(res_r));
  return 0;
}

int main(int argc, char **argv)
{
  if (argc < 10)
  {
    std::fprintf(stderr, "usage: %s physics scheme p quad mesh iters cfl init bcspec\n", argv[0]);
    return 2;
  }
  Args a;
  a.physics = argv[1];
  a.scheme  = argv[2];
  a.p       = std::atoi(argv[3]);
  a.quad    = std::atoi(argv[4]);
  a.mesh    = argv[5];
  a.iters   = std::atoi(argv[6]);
  a.cfl     = std::atof(argv[7]);
  a.init    = argv[8];
  a.bcspec  = argv[9];
  if (argc > 10)
    a.stab = argv[10];

  using Adv   = physics::RotationAdvection2D<ConstDirection2D>;
  using Burg  = physics::Burgers2D;
  using Eul2D = physics::Euler2DCons;
  using Eul3D = physics::Euler3DCons;
  try
  {
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
  }
  catch (const std::exception &e)
  {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  std::fprintf(stderr, "unknown physics/scheme %s/%s\n", a.physics.c_str(), a.scheme.c_str());
  return 2;
}
