// Definitions shared by the oracle harness (ref_harness.cpp) and the drop-in comparison
// program (tests/cpp/dropin_test.cpp): the constant-direction advection policy, the named
// boundary expressions and the named initial states of the benchmark configurations.
// Test infrastructure, compiled against the reference's headers.
#ifndef RDS_ORACLE_REF_COMMON_HPP
#define RDS_ORACLE_REF_COMMON_HPP

#include <cmath>
#include <cstdlib>
#include <iostream>
#include <string>

#include <vector>

#include "interpolation/FEValues.hpp"
#include "interpolation/mesh_function/VectorMeshFunction.hpp"
#include "mesh/std_region/StdRegion.hpp"
#include "math/DenseConstVecView.hpp"

namespace rds_oracle
{

using namespace pdekit;
using coord_v = math::DenseConstVecView<Real>;
using state_v = interpolation::VectorMeshFunction<Real>::const_entry_type;

// ----------------------------------------------------------------------------
// Constant advection direction a = (0.5, 1) / |(0.5, 1)|
// ----------------------------------------------------------------------------

class ConstDirection2D
{
  public:
  template <typename V1, typename V2>
  inline static void rotation_vector(const V1 &, V2 &adv_vector)
  {
    const Real inv_norm = 1.0 / std::sqrt(0.5 * 0.5 + 1.0 * 1.0);
    adv_vector[X0]      = 0.5 * inv_norm;
    adv_vector[X1]      = 1.0 * inv_norm;
  }
};

// ----------------------------------------------------------------------------
// Boundary expressions (our definitions of the configs' inflow data)
// ----------------------------------------------------------------------------

inline Real bc_zero(const coord_v &, const state_v &, const Uint)
{
  return 0.0;
}
inline Real bc_sin2pix(const coord_v &x, const state_v &, const Uint)
{
  return std::sin(2.0 * M_PI * x[0]);
}
inline Real bc_burgers_inlet(const coord_v &x, const state_v &, const Uint)
{
  return 1.5 - 2.0 * x[0];
}
inline Real bc_const_1p5(const coord_v &, const state_v &, const Uint)
{
  return 1.5;
}
inline Real bc_const_m0p5(const coord_v &, const state_v &, const Uint)
{
  return -0.5;
}

using expr_fn = Real (*)(const coord_v &, const state_v &, const Uint);

inline expr_fn find_expr(const std::string &name)
{
  if (name == "zero")
    return &bc_zero;
  if (name == "sin2pix")
    return &bc_sin2pix;
  if (name == "burgers_inlet")
    return &bc_burgers_inlet;
  if (name == "c1.5")
    return &bc_const_1p5;
  if (name == "c-0.5")
    return &bc_const_m0p5;
  std::cerr << "unknown expression " << name << std::endl;
  std::exit(2);
}

// ----------------------------------------------------------------------------
// Initial states as functions of physical coordinates (so that a different node numbering
// of the same mesh reproduces the same state). Each writes NEQ values.
// ----------------------------------------------------------------------------

inline void init_state(const std::string &name, const Real *x, Uint dim, Uint neq, Real *u)
{
  if (name == "zero")
  {
    for (Uint e = 0; e < neq; ++e)
      u[e] = 0.0;
  }
  else if (name == "smooth")
  {
    // scalar: smooth field with both signs and O(1) gradients
    u[0] = 0.3 * std::sin(3.1 * x[0] + 1.7 * x[1]) + 0.2 * std::cos(5.3 * x[0] * x[1]) +
           0.1 * x[0] - 0.05;
  }
  else if (name == "burgers")
  {
    // inflow profile 1.5 - 2x with a smooth perturbation
    u[0] = 1.5 - 2.0 * x[0] + 0.1 * std::sin(7.0 * x[0] + 3.0 * x[1]) * x[1];
  }
  else if (name == "steep")
  {
    // scalar: a steep front (width 0.04) from 1.5 to -0.5 across x = 0.5 + 0.15 y, the
    // profile the Burgers inflow/outflow values build up to
    u[0] = 0.5 - std::tanh((x[0] - 0.5 - 0.15 * x[1]) / 0.04);
  }
  else if (name == "bump2d" || name == "bump3d" || name == "bump2d_jump" ||
           name == "bump3d_jump")
  {
    // Freestream of the reference's bump case (examples/testcases-rdm/Bump-RDS-2D-Explicit.cpp:
    // 100-131): total temperature / pressure 307.6488978 K / 120195.4453 Pa, R = 287.046,
    // Mach 0.5 (2D) or 0.6 (3D) along x, with a +-1% perturbation of density and pressure that
    // is a fixed pseudo-random function of the coordinates.
    const Real gamma = 1.4, R = 287.046, Ttot = 307.6488978, Ptot = 120195.4453;
    const bool d2 = name == "bump2d" || name == "bump2d_jump";
    const Real M  = d2 ? 0.5 : 0.6;
    const Real f  = 1. + 0.5 * (gamma - 1.) * M * M;
    const Real T  = Ttot / f, p0 = Ptot / std::pow(f, gamma / (gamma - 1.));
    const Real z  = dim == 3 ? x[2] : 0.0;
    auto hash     = [](Real a, Real b, Real c) {
      const Real s = std::sin(12.9898 * a + 78.233 * b + 37.719 * c) * 43758.5453;
      return 2.0 * (s - std::floor(s)) - 1.0;
    };
    // "_jump": density and pressure raised by up to 30% across a steep front (width 0.05) at
    // x = 0.2 + 0.1 y
    const Real jump = name.size() > 6 ? 1. + 0.15 * (1. + std::tanh((x[0] - 0.2 - 0.1 * x[1]) / 0.05))
                                      : 1.;
    const Real rho = jump * p0 / (R * T) * (1. + 0.01 * hash(x[0], x[1], z));
    const Real p   = jump * p0 * (1. + 0.01 * hash(x[1], z, x[0]));
    const Real ux  = M * std::sqrt(gamma * R * T);
    u[0]           = rho;
    u[1]           = rho * ux;
    for (Uint d = 1; d < dim; ++d)
      u[1 + d] = 0.0;
    u[dim + 1] = p / (gamma - 1.) + 0.5 * rho * ux * ux;
  }
  else if (name == "euler2d")
  {
    // freestream M = 0.5 along x with a smooth O(1%) perturbation
    const Real gamma = 1.4, rho = 1.0 + 0.01 * std::sin(4.0 * x[0] + 3.0 * x[1]);
    const Real p = 1.0 / gamma * (1.0 + 0.01 * std::cos(5.0 * x[0] - 2.0 * x[1]));
    const Real c = std::sqrt(gamma * p / rho), ux = 0.5 * c, uy = 0.01 * std::sin(6.0 * x[1]);
    u[0] = rho;
    u[1] = rho * ux;
    u[2] = rho * uy;
    u[3] = p / (gamma - 1.0) + 0.5 * rho * (ux * ux + uy * uy);
  }
  else if (name == "euler3d")
  {
    const Real gamma = 1.4, rho = 1.0 + 0.01 * std::sin(4.0 * x[0] + 3.0 * x[1] - x[2]);
    const Real p  = 1.0 / gamma * (1.0 + 0.01 * std::cos(5.0 * x[0] - 2.0 * x[2]));
    const Real c  = std::sqrt(gamma * p / rho), ux = 0.6 * c;
    const Real uy = 0.01 * std::sin(6.0 * x[1]), uz = 0.01 * std::cos(5.0 * x[2]);
    u[0] = rho;
    u[1] = rho * ux;
    u[2] = rho * uy;
    u[3] = rho * uz;
    u[4] = p / (gamma - 1.0) + 0.5 * rho * (ux * ux + uy * uy + uz * uz);
  }
  else
  {
    std::cerr << "unknown init " << name << std::endl;
    std::exit(2);
  }
  (void)dim;
}


// Coordinates of the solution dofs [nsol][dim] through the geometry basis of each cell
// evaluated at the cell's solution nodes (the reference's equidistant point sets).
template <typename MeshType, typename DofMap>
std::vector<Real> solution_node_coords(const MeshType &mesh, const DofMap &geo, const DofMap &sol,
                                       Uint dim)
{
  std::vector<Real> xy(sol.nb_nodes() * dim, 0.0);
  for (Uint c = 0; c < sol.nb_active_cells(); ++c)
  {
    const mesh::MeshEntity gc = geo.active_cell(mesh::ActiveIdx(c));
    const mesh::MeshEntity sc = sol.active_cell(mesh::ActiveIdx(c));
    const auto coords         = mesh.active_cell(mesh::ActiveIdx(c)).coordinates();
    const ElemShape shape     = sc.pt_set_id().elem_shape();
    mesh::StdRegion sol_region;
    sol_region.change_type(
        mesh::PointSetTag(shape, sc.pt_set_id().poly_order(), PointSetID::Equidist));
    const math::DenseDMat<Real> &nodes = sol_region.get().coordinates();
    math::DenseDVec<Real> ones(nodes.rows());
    ones.fill(1.0);
    interpolation::FEValues fe;
    const Uint pg = gc.pt_set_id().poly_order();
    fe.configure(mesh::PointSetTag(shape, pg, PointSetID::Equidist),
                 mesh::sf::SFTag(shape, SFunc::Lagrange, pg, ModalBasis::Modal));
    fe.fill_Vandermonde(nodes, ones);
    const math::DenseDMat<Real> &Vgs = fe.Vandermonde();
    for (Uint n = 0; n < sc.nb_vert(); ++n)
      for (Uint d = 0; d < dim; ++d)
      {
        Real x = 0.0;
        for (Uint g = 0; g < gc.nb_vert(); ++g)
          x += Vgs(n, g) * coords.const_node_view(g)[d];
        xy[sc.vertex(n) * dim + d] = x;
      }
  }
  return xy;
}

} // namespace rds_oracle

#endif
