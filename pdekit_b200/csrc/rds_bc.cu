// Weak boundary-condition kernels: one thread per boundary facet.
//
// Per facet quadrature point a ghost flux is formed and distributed to the facet dofs with the
// facet basis, V(q,n) w_q |J_q| (ghost flux), and summed into the facet total; the dof
// residuals are then rescaled so that they sum to the facet total (src/solver/rdm/bc/
// WeakBC.hpp:786-832). The facet's wave speed is max_q max(1e-9, |lambda|) for every dof and
// enters the nodal wave speed multiplied by the dual volume (WeakBC.hpp:315-352).
//   WeakDirichlet (bc/WeakDirichletBC.hpp:159-265): K-(n) (g - u_q).
//   WeakWall (bc/WeakWall.hpp:93-250): F(u_mirror).n - F(u_q).n, u_mirror with the normal
//     velocity removed, same density and pressure; the dof part is scaled by 1/(3p) for p > 1.
//   WeakSubInlet (bc/WeakSubInlet.hpp:113-215): K-(n) (u_in - u_q), u_in from the total
//     temperature and pressure at the local Mach number (gas constant 287.046 as there).
//   WeakSubOutlet (bc/WeakSubOutlet.hpp:105-190): K-(n) (u_out - u_q), u_out = u_q with the
//     energy of the outlet pressure.
//   WeakFarfield (bc/WeakFarfield.hpp:125-240, the active branch): K-(n) (u_ref - u_q) with the
//     reference state u_ref, lambda floor 1e-8.
//   WeakSuperInlet (bc/WeakSuperInlet.hpp:62-160): no residual; only the facet's wave speed.
//   WeakSymmetry (bc/WeakSymmetry.hpp:100-190): K-(n) (u_mirror - u_q), u_mirror with the same
//     density and energy and the momentum rho (V - 2 (V.n) n).
// StrongDirichletBC::apply (bc/StrongDirichletBC.hpp:202-233) has its own kernel: the listed
// dofs take their values (one thread per distinct dof, the value of the last facet naming it).
// Facet normals are (dy/dxi, -dx/dxi)/|.| in 2D and the normalised cross product of the two
// tangents in 3D, with |J| the length / area factor (src/interpolation/GeometryMetric.hpp:560-660).

#include "rds_bc_facet.cuh"
#include "rds_internal.h"
#include "rds_physics.cuh"

namespace rds
{

namespace
{

template <int KIND, int PHYS, int D, int NEQ, int NFDOF, int NFQ, int NFGEO>
__global__ void __launch_bounds__(kBlock)
    bc_weak(const BCArgs a, const FacetTables<double, D, NFDOF, NFQ, NFGEO> tb)
{
  if (*a.stop)
    return;
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= a.nfacets)
    return;
  bc_weak_facet<KIND, PHYS, D, NEQ, NFDOF, NFQ, NFGEO>(a, tb, f);
}

template <int KIND, int PHYS, int D, int NEQ, int NFDOF, int NFQ, int NFGEO>
cudaError_t launch_weak(const HostBC &b, const BCArgs &a, cudaStream_t s)
{
  FacetTables<double, D, NFDOF, NFQ, NFGEO> tb;
  for (int q = 0; q < NFQ; ++q)
  {
    tb.fw[q] = b.fw[q];
    for (int n = 0; n < NFDOF; ++n)
      tb.fV[q][n] = b.fV[q * NFDOF + n];
    for (int xi = 0; xi < D - 1; ++xi)
      for (int g = 0; g < NFGEO; ++g)
        tb.fdVgeo[xi][q][g] = b.fdVgeo[(xi * NFQ + q) * NFGEO + g];
  }
  const int grid = (a.nfacets + kBlock - 1) / kBlock;
  bc_weak<KIND, PHYS, D, NEQ, NFDOF, NFQ, NFGEO><<<grid, kBlock, 0, s>>>(a, tb);
  return cudaGetLastError();
}

// Facet types: 2D lines P1-P3 with 3-5 point Gauss rules; 3D P1 triangles with 4 points and P2
// triangles with 7 or 12.
template <int KIND, int PHYS, int D, int NEQ>
cudaError_t dispatch_facets(const HostBC &b, const BCArgs &a, cudaStream_t s, bool *ok)
{
  const rds_bc_group &d = b.desc;
  *ok                   = true;
  if constexpr (D == 2)
  {
    if (d.nfgeo == 2)
    {
#define RDS_WEAK(NFDOF, NFQ)                                                                       \
  if (d.nfdof == NFDOF && d.nfq == NFQ)                                                            \
    return launch_weak<KIND, PHYS, D, NEQ, NFDOF, NFQ, 2>(b, a, s);
      RDS_WEAK(2, 3)
      RDS_WEAK(2, 4)
      RDS_WEAK(3, 3)
      RDS_WEAK(3, 4)
      RDS_WEAK(4, 5)
      RDS_WEAK(4, 4)
#undef RDS_WEAK
    }
  }
  else
  {
    if (d.nfgeo == 3 && d.nfdof == 6 && d.nfq == 12)
      return launch_weak<KIND, PHYS, D, NEQ, 6, 12, 3>(b, a, s);
    if (d.nfgeo == 3 && d.nfdof == 3 && d.nfq == 4)
      return launch_weak<KIND, PHYS, D, NEQ, 3, 4, 3>(b, a, s);
    if (d.nfgeo == 3 && d.nfdof == 6 && d.nfq == 7)
      return launch_weak<KIND, PHYS, D, NEQ, 6, 7, 3>(b, a, s);
  }
  *ok = false;
  return cudaSuccess;
}

template <int PHYS, int D, int NEQ>
cudaError_t dispatch_kind(const HostBC &b, const BCArgs &a, cudaStream_t s, bool *ok)
{
  *ok = false;
  switch (b.desc.kind)
  {
  case RDS_BC_WEAK_DIRICHLET:
    return dispatch_facets<RDS_BC_WEAK_DIRICHLET, PHYS, D, NEQ>(b, a, s, ok);
  case RDS_BC_WEAK_WALL:
    if constexpr (NEQ > 1)
      return dispatch_facets<RDS_BC_WEAK_WALL, PHYS, D, NEQ>(b, a, s, ok);
    break;
  case RDS_BC_WEAK_SUB_INLET:
    if constexpr (NEQ > 1)
      return dispatch_facets<RDS_BC_WEAK_SUB_INLET, PHYS, D, NEQ>(b, a, s, ok);
    break;
  case RDS_BC_WEAK_SUB_OUTLET:
    if constexpr (NEQ > 1)
      return dispatch_facets<RDS_BC_WEAK_SUB_OUTLET, PHYS, D, NEQ>(b, a, s, ok);
    break;
  case RDS_BC_WEAK_FARFIELD:
    if constexpr (NEQ > 1)
      return dispatch_facets<RDS_BC_WEAK_FARFIELD, PHYS, D, NEQ>(b, a, s, ok);
    break;
  case RDS_BC_WEAK_SUPER_INLET:
    if constexpr (NEQ > 1)
      return dispatch_facets<RDS_BC_WEAK_SUPER_INLET, PHYS, D, NEQ>(b, a, s, ok);
    break;
  case RDS_BC_WEAK_SYMMETRY:
    if constexpr (NEQ > 1)
      return dispatch_facets<RDS_BC_WEAK_SYMMETRY, PHYS, D, NEQ>(b, a, s, ok);
    break;
  default:
    break;
  }
  return cudaSuccess;
}

const char *bc_name(int kind)
{
  switch (kind)
  {
  case RDS_BC_WEAK_WALL:
    return "bc_weak_wall";
  case RDS_BC_WEAK_SUB_INLET:
    return "bc_weak_sub_inlet";
  case RDS_BC_WEAK_SUB_OUTLET:
    return "bc_weak_sub_outlet";
  case RDS_BC_WEAK_FARFIELD:
    return "bc_weak_farfield";
  case RDS_BC_WEAK_SUPER_INLET:
    return "bc_weak_super_inlet";
  case RDS_BC_WEAK_SYMMETRY:
    return "bc_weak_symmetry";
  case RDS_BC_STRONG_DIRICHLET:
    return "bc_strong_dirichlet";
  default:
    return "bc_weak_dirichlet";
  }
}

// Strong Dirichlet: ndofs distinct dofs, their values SoA [neq][ndofs].
__global__ void __launch_bounds__(kBlock)
    bc_strong(int ndofs, int neq, int nnodes, const int32_t *__restrict__ dofs,
              const double *__restrict__ vals, double *__restrict__ u, const int *stop)
{
  if (*stop)
    return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ndofs)
    return;
  const int v = dofs[i];
  for (int e = 0; e < neq; ++e)
    u[(size_t)e * nnodes + v] = vals[(size_t)e * ndofs + i];
}

} // namespace

cudaError_t launch_bc(const HostBC &b, const BCArgs &a, int physics, int dim, int neq,
                      cudaStream_t s, const char **name)
{
  bool ok         = false;
  cudaError_t err = cudaSuccess;
  *name           = bc_name(b.desc.kind);
  if (b.desc.kind == RDS_BC_STRONG_DIRICHLET)
  {
    if (a.nfacets > 0)
      bc_strong<<<(a.nfacets + kBlock - 1) / kBlock, kBlock, 0, s>>>(
          a.nfacets, neq, a.nnodes, a.sol_conn, a.gq, a.u_strong, a.stop);
    return cudaGetLastError();
  }
  if (physics == RDS_ADVECTION_CONST && dim == 2 && neq == 1)
    err = dispatch_kind<RDS_ADVECTION_CONST, 2, 1>(b, a, s, &ok);
  else if (physics == RDS_BURGERS2D && dim == 2 && neq == 1)
    err = dispatch_kind<RDS_BURGERS2D, 2, 1>(b, a, s, &ok);
  else if (physics == RDS_EULER2D && dim == 2 && neq == 4)
    err = dispatch_kind<RDS_EULER2D, 2, 4>(b, a, s, &ok);
  else if (physics == RDS_EULER3D && dim == 3 && neq == 5)
    err = dispatch_kind<RDS_EULER3D, 3, 5>(b, a, s, &ok);
  if (!ok)
    return cudaErrorNotSupported;
  return err;
}

} // namespace rds
