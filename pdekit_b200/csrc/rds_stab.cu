// Stabilisation operators either side of the cell residual: the shock sensor and blending
// coefficients that produce nodal fields, the cell-to-node transfer, and the artificial
// viscosity term that PGLDA adds to its nodal residuals.
//
//   viscous    PGLDA cells with a nodal artificial viscosity eps: at every quadrature point
//              eps_q = sum_n V(q,n) eps_n and, when eps_q != 0,
//              res_n += w_q detJ_q eps_q grad phi_n . grad u_e(q)  for every equation e
//              (src/solver/rdm/cellsplitters/PGLDA.hpp:245-256, the viscosity interpolated as
//              in assembly/PGRDMExplicitCellWorker.hpp:519-533). Runs after the cell kernel of
//              the group and adds to its contribution slots; G lanes per cell, on the points
//              to form the gradient terms, then on the nodes to contract them (shared memory).
//   sensor     the Persson-Peraire smoothness sensor of the first state component
//              (src/solver/art_visc/ArtificialViscosity.hpp:300-455,
//              blending_coeff/ArtViscIndicatorCoeffImpl.hpp:261-425), one thread per affine
//              simplex: Se = sum_q wj (R u)_q^2 / sum_q wj (Vn u)_q^2 (0 if the denominator is
//              <= 1e-10), R mapping nodal values to u - u_{p-1} at the points (u_{p-1} the
//              modal truncation of the reference, an L2 projection because its simplex bases
//              are orthogonal; the host builds R), se = log10 Se, s0 = 1/p^4, value 0 / eps0 /
//              0.5 eps0 (1 + sin(pi (se - s0) / (2 kappa))) below / above / within
//              s0 -+ kappa, eps0 = factor h / p (h = |K|^(1/D)) or 1 for the blending form.
//   blend      LF_Blend (blending_coeff/LFBlendingCoeffImpl.hpp:76-126): per cell
//              ksi = max_n |u_n - u_avg| / (|u_n| + |u_avg| + 1e-12), per node the max over its
//              cells (node-parallel over the gather lists), per cell 1 - max over its nodes;
//              Wong-Jansen (WongJansenBlendingCoeffImpl.hpp:80-116): per cell
//              sum_n t_n / (u_inf^4 + sum_n t_n), t_n = (u_n^2 - u_avg^2)^2.
//   bonanni    Bonanni's pressure-based coefficient (blending_coeff/BonanniBlendingCoeffImpl.hpp:
//              171-392, Euler 2D / 3D): per cell, with the coefficient's own Gauss rule, the
//              volume |K|, the integrals of the velocity and of grad p (p and V from the nodal
//              states), f = (v_m . gp_m) |v_m| with v_m, gp_m those integrals over |K|, and
//              lc = |K|^(1/D); over the mesh p_min, p_max of the nodal pressures and the mean
//              velocity v_dom = sum int V / sum |K|; then per cell
//              theta = min(1, max(f / ((p_max - p_min) |v_dom|^2), 0)^2 lc), min and max with
//              std::min / std::max's comparisons (so a NaN or infinite quotient ends as there).
//              Mesh sums over block sums in a fixed order.
//   transfer   cell values -> nodal field (interpolation/mesh_function/MeshFunctionTools.hpp:
//              52-397, no adaptation): every vertex node max(0, max over its cells), every
//              other node the vertex interpolant of the last cell (in cell order) holding it.
//              Node-parallel over the gather lists, which hold each node's cells in ascending
//              order, so the result does not depend on scheduling.

#include "rds_internal.h"

namespace rds
{

namespace
{

constexpr double kPi = 3.14159265358979323846;

template <int D>
__device__ __forceinline__ double invert(const double J[D][D], double iJ[D][D])
{
  if constexpr (D == 2)
  {
    const double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    const double r   = 1.0 / det;
    iJ[0][0]         = r * J[1][1];
    iJ[1][1]         = r * J[0][0];
    iJ[0][1]         = -r * J[0][1];
    iJ[1][0]         = -r * J[1][0];
    return det;
  }
  else
  {
    const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
    const double r   = 1.0 / det;
    iJ[0][0]         = r * c00;
    iJ[1][0]         = r * c01;
    iJ[2][0]         = r * c02;
    iJ[0][1]         = r * (J[0][2] * J[2][1] - J[0][1] * J[2][2]);
    iJ[1][1]         = r * (J[0][0] * J[2][2] - J[0][2] * J[2][0]);
    iJ[2][1]         = r * (J[0][1] * J[2][0] - J[0][0] * J[2][1]);
    iJ[0][2]         = r * (J[0][1] * J[1][2] - J[0][2] * J[1][1]);
    iJ[1][2]         = r * (J[0][2] * J[1][0] - J[0][0] * J[1][2]);
    iJ[2][2]         = r * (J[0][0] * J[1][1] - J[0][1] * J[1][0]);
    return det;
  }
}

// J[k][i] = d x_i / d xi_k at point q of cell c (every lane of the group computes it)
template <int D>
__device__ __forceinline__ void jacobian_at(const ViscArgs &a, int c, int q, double J[D][D])
{
#pragma unroll
  for (int k = 0; k < D; ++k)
#pragma unroll
    for (int i = 0; i < D; ++i)
      J[k][i] = 0.0;
  for (int g = 0; g < a.ngeo; ++g)
  {
    const int v = __ldg(a.geo_conn + (size_t)g * a.ncells + c);
#pragma unroll
    for (int k = 0; k < D; ++k)
    {
      const double d = __ldg(a.dVgeo + ((size_t)k * a.nq + q) * a.ngeo + g);
#pragma unroll
      for (int i = 0; i < D; ++i)
        J[k][i] += d * __ldg(a.X + (size_t)i * a.ngeo_nodes + v);
    }
  }
}

// Shared memory of viscous_cells: the tables (V, dV) once per block, then per cell the nodal
// values (eps, u) and the point values S'_q[e][a] = sum_i invJ_q[i][a] w_q detJ_q eps_q du_e/dx_i.
template <int D, int NEQ>
struct ViscSmem
{
  __host__ __device__ static size_t tables(int nq, int ndof) { return (size_t)nq * ndof * (1 + D); }
  __host__ __device__ static size_t cell(int nq, int ndof)
  {
    return (size_t)ndof * (NEQ + 1) + (size_t)nq * NEQ * D;
  }
  static size_t bytes(int nq, int ndof, int cpb)
  {
    return sizeof(double) * (tables(nq, ndof) + (size_t)cpb * cell(nq, ndof));
  }
};

// Two phases per cell, through shared memory: lanes on points form S' (the physical gradient
// of u, the viscosity at the point and the test function's invJ folded in, so the same form
// holds on curved cells), then lanes on nodes contract it with the reference gradients:
//   res_n,e += sum_q sum_a dV[a][q][n] S'_q[e][a]
//            = sum_q w_q detJ_q eps_q grad phi_n(q) . grad u_e(q).
// The sum over the points runs in a different order than the reference's (rounding only).
template <int D, int NEQ, int G>
__global__ void __launch_bounds__(kBlock) viscous_cells(const ViscArgs a)
{
  if (a.stop && *a.stop)
    return; // uniform over the grid
  extern __shared__ double smem[];
  const int nq = a.nq, ndof = a.ndof;
  double *sV   = smem;                            // [nq][ndof]
  double *sdV  = sV + (size_t)nq * ndof;          // [D][nq][ndof]
  const int cl = threadIdx.x / G, lane = threadIdx.x % G;
  double *cell = smem + ViscSmem<D, NEQ>::tables(nq, ndof) + (size_t)cl * ViscSmem<D, NEQ>::cell(nq, ndof);
  double *seps = cell;                            // [ndof]
  double *su   = seps + ndof;                     // [ndof][NEQ]
  double *sS   = su + (size_t)ndof * NEQ;         // [nq][NEQ][D]
  const int c     = blockIdx.x * (blockDim.x / G) + cl;
  const bool live = c < a.ncells;

  for (int i = threadIdx.x; i < nq * ndof; i += blockDim.x)
    sV[i] = __ldg(a.V + i);
  for (int i = threadIdx.x; i < D * nq * ndof; i += blockDim.x)
    sdV[i] = __ldg(a.dV + i);
  if (live)
    for (int n = lane; n < ndof; n += G)
    {
      const int v = __ldg(a.sol_conn + (size_t)n * a.ncells + c);
      seps[n]     = __ldg(a.eps + v);
#pragma unroll
      for (int e = 0; e < NEQ; ++e)
        su[n * NEQ + e] = __ldg(a.u + (size_t)e * a.nnodes + v);
    }
  __syncthreads();

  // phase 1: lanes on points
  if (live)
    for (int q = lane; q < nq; q += G)
    {
      double J[D][D], iJ[D][D];
      jacobian_at<D>(a, c, a.affine ? 0 : q, J);
      const double det = invert<D>(J, iJ);
      double eq = 0.0, gx[NEQ][D];
#pragma unroll
      for (int e = 0; e < NEQ; ++e)
#pragma unroll
        for (int k = 0; k < D; ++k)
          gx[e][k] = 0.0;
      for (int n = 0; n < ndof; ++n)
      {
        eq += sV[q * ndof + n] * seps[n];
        double gr[D];
#pragma unroll
        for (int k = 0; k < D; ++k)
          gr[k] = sdV[((size_t)k * nq + q) * ndof + n];
#pragma unroll
        for (int e = 0; e < NEQ; ++e)
        {
          const double un = su[n * NEQ + e];
#pragma unroll
          for (int k = 0; k < D; ++k)
            gx[e][k] += gr[k] * un;
        }
      }
      const double f = __ldg(a.w + q) * det * eq;
      double *S      = sS + (size_t)q * NEQ * D;
#pragma unroll
      for (int e = 0; e < NEQ; ++e)
      {
        double gp[D]; // f du_e/dx_i
#pragma unroll
        for (int i = 0; i < D; ++i)
        {
          double t = iJ[i][0] * gx[e][0];
#pragma unroll
          for (int k = 1; k < D; ++k)
            t += iJ[i][k] * gx[e][k];
          gp[i] = f * t;
        }
#pragma unroll
        for (int k = 0; k < D; ++k)
        {
          double t = iJ[0][k] * gp[0];
#pragma unroll
          for (int i = 1; i < D; ++i)
            t += iJ[i][k] * gp[i];
          S[e * D + k] = t;
        }
      }
    }
  __syncthreads();

  // phase 2: lanes on nodes
  if (live)
    for (int n = lane; n < ndof; n += G)
    {
      double acc[NEQ];
#pragma unroll
      for (int e = 0; e < NEQ; ++e)
        acc[e] = 0.0;
      for (int q = 0; q < nq; ++q)
      {
        double gr[D];
#pragma unroll
        for (int k = 0; k < D; ++k)
          gr[k] = sdV[((size_t)k * nq + q) * ndof + n];
        const double *S = sS + (size_t)q * NEQ * D;
#pragma unroll
        for (int e = 0; e < NEQ; ++e)
#pragma unroll
          for (int k = 0; k < D; ++k)
            acc[e] += gr[k] * S[e * D + k];
      }
      const long long slot = a.slot_base + (long long)n * a.ncells + c;
#pragma unroll
      for (int e = 0; e < NEQ; ++e)
        a.contrib[e * a.S + slot] += acc[e];
    }
}

template <int D, int NEQ>
cudaError_t launch_viscous_g(const ViscArgs &a, cudaStream_t s, const char **name)
{
  if (name)
    *name = "viscous_cells";
  // lanes per cell: the smallest power of two >= the nodes (phase 2) and >= 4
  int G = 4;
  while (G < a.ndof)
    G *= 2;
  if (G > 32)
    return cudaErrorInvalidValue;
  const int cpb       = kBlock / G;
  const size_t smem   = ViscSmem<D, NEQ>::bytes(a.nq, a.ndof, cpb);
  if (smem > 48 * 1024)
    return cudaErrorInvalidValue;
  const int grid = (a.ncells + cpb - 1) / cpb;
  switch (G)
  {
  case 4:
    viscous_cells<D, NEQ, 4><<<grid, kBlock, smem, s>>>(a);
    break;
  case 8:
    viscous_cells<D, NEQ, 8><<<grid, kBlock, smem, s>>>(a);
    break;
  case 16:
    viscous_cells<D, NEQ, 16><<<grid, kBlock, smem, s>>>(a);
    break;
  default:
    viscous_cells<D, NEQ, 32><<<grid, kBlock, smem, s>>>(a);
  }
  return cudaGetLastError();
}

__global__ void __launch_bounds__(kBlock) sensor_cells_2d(const SensorArgs a);
__global__ void __launch_bounds__(kBlock) sensor_cells_3d(const SensorArgs a);

template <int D>
__device__ __forceinline__ double sensor_value(const SensorArgs &a, double nom, double den,
                                               double vol);
template <int D>
__device__ __forceinline__ void sensor_cell_mapped(const SensorArgs &a, int c);

template <int D>
__device__ __forceinline__ void sensor_cell(const SensorArgs &a)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncells)
    return;
  if (a.dVgeo)
  {
    sensor_cell_mapped<D>(a, c);
    return;
  }
  // affine simplex on the reference element with vertices (-1,..,-1) and -1 + 2 e_k:
  // d x / d xi_k = (X_{k+1} - X_0) / 2
  double X0[D], J[D][D];
  {
    const int v0 = __ldg(a.geo_conn + c);
#pragma unroll
    for (int i = 0; i < D; ++i)
      X0[i] = __ldg(a.X + (size_t)i * a.ngeo_nodes + v0);
#pragma unroll
    for (int k = 0; k < D; ++k)
    {
      const int v = __ldg(a.geo_conn + (size_t)(k + 1) * a.ncells + c);
#pragma unroll
      for (int i = 0; i < D; ++i)
        J[k][i] = 0.5 * (__ldg(a.X + (size_t)i * a.ngeo_nodes + v) - X0[i]);
    }
  }
  double det;
  if constexpr (D == 2)
    det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
  else
    det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) +
          J[0][1] * (J[1][2] * J[2][0] - J[1][0] * J[2][2]) +
          J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);

  double nom = 0.0, den = 0.0, vol = 0.0;
  for (int q = 0; q < a.nq; ++q)
  {
    double s = 0.0, r = 0.0;
    for (int n = 0; n < a.ndof; ++n)
    {
      const double un = __ldg(a.u + __ldg(a.sol_conn + (size_t)n * a.ncells + c));
      s += __ldg(a.Vn + (size_t)q * a.ndof + n) * un;
      r += __ldg(a.R + (size_t)q * a.ndof + n) * un;
    }
    const double wj = det * __ldg(a.w + q);
    vol += wj;
    nom += wj * r * r;
    den += wj * s * s;
  }
  a.out[c] = sensor_value<D>(a, nom, den, vol);
}

// Se = nom / den (0 when den <= 1e-10), se = log10 Se, and the ramp around s0 = 1 / p^4
// (ArtificialViscosity.hpp:468-510); eps0 = factor |K|^(1/D) / p, or 1 for the blending
// coefficient
template <int D>
__device__ __forceinline__ double sensor_value(const SensorArgs &a, double nom, double den,
                                               double vol)
{
  const double Se = (den <= 1.e-10) ? 0.0 : nom / den;
  const double se = log(Se) / log(10.0);
  const double p  = (double)a.order;
  const double s0 = 1.0 / (p * p * p * p);
  const double e0 = a.blend ? 1.0 : a.factor * (pow(vol, 1.0 / D) / p);
  double val;
  if (se < s0 - a.kappa)
    val = 0.0;
  else if (se > s0 + a.kappa)
    val = e0;
  else
    val = 0.5 * e0 * (1.0 + sin(kPi * (se - s0) / (2.0 * a.kappa)));
  return val;
}

// Cells whose Jacobian varies (bilinear quadrilaterals): J = sum_g dVgeo[.][q][g] X_g at every
// point (the geometry metric the reference evaluates at its rule's points).
template <int D>
__device__ __forceinline__ void sensor_cell_mapped(const SensorArgs &a, int c)
{
  double Xg[kStabMaxGeo][D];
#pragma unroll
  for (int g = 0; g < kStabMaxGeo; ++g)
    if (g < a.ngeo)
    {
      const int v = __ldg(a.geo_conn + (size_t)g * a.ncells + c);
#pragma unroll
      for (int i = 0; i < D; ++i)
        Xg[g][i] = __ldg(a.X + (size_t)i * a.ngeo_nodes + v);
    }
  double nom = 0.0, den = 0.0, vol = 0.0;
  for (int q = 0; q < a.nq; ++q)
  {
    double J[D][D];
#pragma unroll
    for (int k = 0; k < D; ++k)
#pragma unroll
      for (int i = 0; i < D; ++i)
        J[k][i] = 0.0;
#pragma unroll
    for (int g = 0; g < kStabMaxGeo; ++g)
      if (g < a.ngeo)
      {
#pragma unroll
        for (int k = 0; k < D; ++k)
        {
          const double d = __ldg(a.dVgeo + ((size_t)k * a.nq + q) * a.ngeo + g);
#pragma unroll
          for (int i = 0; i < D; ++i)
            J[k][i] += d * Xg[g][i];
        }
      }
    double det;
    if constexpr (D == 2)
      det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    else
      det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) +
            J[0][1] * (J[1][2] * J[2][0] - J[1][0] * J[2][2]) +
            J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    double s = 0.0, r = 0.0;
    for (int n = 0; n < a.ndof; ++n)
    {
      const double un = __ldg(a.u + __ldg(a.sol_conn + (size_t)n * a.ncells + c));
      s += __ldg(a.Vn + (size_t)q * a.ndof + n) * un;
      r += __ldg(a.R + (size_t)q * a.ndof + n) * un;
    }
    const double wj = det * __ldg(a.w + q);
    vol += wj;
    nom += wj * r * r;
    den += wj * s * s;
  }
  a.out[c] = sensor_value<D>(a, nom, den, vol);
}

__global__ void __launch_bounds__(kBlock) sensor_cells_2d(const SensorArgs a)
{
  sensor_cell<2>(a);
}
__global__ void __launch_bounds__(kBlock) sensor_cells_3d(const SensorArgs a)
{
  sensor_cell<3>(a);
}

// one block: v /= max(v) unless max(v) < 1e-14 (ArtificialViscosity.hpp:257-279)
__global__ void __launch_bounds__(kGBlock) normalise_max(int n, double *v)
{
  __shared__ double sm[kGBlock / 32];
  double m = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    m = fmax(m, v[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0)
    sm[threadIdx.x >> 5] = m;
  __syncthreads();
  m = 0.0;
  for (int k = 0; k < (int)(blockDim.x >> 5); ++k)
    m = fmax(m, sm[k]);
  if (m < 1.e-14)
    return;
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    v[i] /= m;
}

__global__ void __launch_bounds__(kBlock)
    blend_cells(int kind, int ncells, int ndof, const int32_t *__restrict__ conn,
                const double *__restrict__ u, double param, double *__restrict__ out)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells)
    return;
  double avg = 0.0;
  for (int n = 0; n < ndof; ++n)
    avg += __ldg(u + __ldg(conn + (size_t)n * ncells + c));
  avg /= ndof;
  if (kind == 0)
  {
    double ksi = 0.0;
    for (int n = 0; n < ndof; ++n)
    {
      const double un = __ldg(u + __ldg(conn + (size_t)n * ncells + c));
      ksi             = fmax(ksi, fabs(un - avg) / (fabs(un) + fabs(avg) + 1.e-12));
    }
    out[c] = ksi;
  }
  else
  {
    const double ui2 = param * param;
    double nom = 0.0, den = 1.0 * (ui2 * ui2);
    for (int n = 0; n < ndof; ++n)
    {
      const double un = __ldg(u + __ldg(conn + (size_t)n * ncells + c));
      const double d  = un * un - avg * avg;
      const double t  = d * d;
      nom += t;
      den += t;
    }
    out[c] = nom / den;
  }
}

__global__ void __launch_bounds__(kGBlock)
    node_max(int nnodes, const int32_t *__restrict__ row, const int32_t *__restrict__ ent_ws,
             long long wcells, const double *__restrict__ cellf, double *__restrict__ nodef)
{
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nnodes)
    return;
  double m = 0.0;
  for (int p = row[v]; p < row[v + 1]; ++p)
  {
    const int w = ent_ws[p];
    if (w < wcells)
      m = fmax(m, cellf[w]);
  }
  nodef[v] = m;
}

__global__ void __launch_bounds__(kBlock)
    lf_finish(int ncells, int ndof, const int32_t *__restrict__ conn,
              const double *__restrict__ nodef, double *__restrict__ out)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells)
    return;
  double m = 0.0;
  for (int n = 0; n < ndof; ++n)
    m = fmax(m, nodef[__ldg(conn + (size_t)n * ncells + c)]);
  out[c] = 1.0 - m;
}

// (group, cell, local node) of a cell contribution slot
__device__ __forceinline__ int decode(const StabGroups &g, long long slot, int *c, int *n)
{
  for (int k = 0; k < g.n; ++k)
  {
    const long long off = slot - g.slot_base[k];
    if (off >= 0 && off < (long long)g.ndof[k] * g.ncells[k])
    {
      *n = (int)(off / g.ncells[k]);
      *c = (int)(off % g.ncells[k]);
      return k;
    }
  }
  return -1;
}

// pass 1: vertex nodes take max(0, max over their cells)
__global__ void __launch_bounds__(kGBlock)
    vertex_max(int nnodes, const int32_t *__restrict__ row, const int32_t *__restrict__ ent_slot,
               long long scells, const StabGroups g, const double *__restrict__ cellf,
               double *__restrict__ nodef)
{
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nnodes)
    return;
  double m    = 0.0;
  bool vertex = false;
  for (int p = row[v]; p < row[v + 1]; ++p)
  {
    const long long slot = ent_slot[p];
    if (slot >= scells)
      break; // boundary-facet entries follow the cells
    int c, n;
    const int k = decode(g, slot, &c, &n);
    if (k < 0 || n >= g.nvert[k])
      break; // a node that is not a vertex of its cells
    vertex = true;
    m      = fmax(m, cellf[g.ws_base[k] + c]);
  }
  if (vertex)
    nodef[v] = m;
}

// pass 2: other nodes take the vertex interpolant of the last cell holding them
__global__ void __launch_bounds__(kGBlock)
    interior_interp(int nnodes, const int32_t *__restrict__ row,
                    const int32_t *__restrict__ ent_slot, long long scells, const StabGroups g,
                    double *__restrict__ nodef)
{
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nnodes)
    return;
  int k = -1, c = 0, n = 0;
  for (int p = row[v]; p < row[v + 1]; ++p)
  {
    const long long slot = ent_slot[p];
    if (slot >= scells)
      break;
    int cc, nn;
    const int kk = decode(g, slot, &cc, &nn);
    if (kk < 0 || nn < g.nvert[kk])
      return; // a vertex (pass 1), or not a cell node
    k = kk;
    c = cc;
    n = nn;
  }
  if (k < 0)
    return;
  const int nv     = g.nvert[k];
  const double *P1 = g.P1[k] + (size_t)n * nv;
  double f         = 0.0;
  for (int i = 0; i < nv; ++i)
    f += P1[i] * nodef[g.sol_conn[k][(size_t)i * g.ncells[k] + c]];
  nodef[v] = f;
}


// ---- Bonanni's coefficient

constexpr int kBonBlock = 128;

__device__ __forceinline__ double std_max(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double std_min(double a, double b) { return (b < a) ? b : a; }

// sum / min / max over a block of kBonBlock threads (the result valid in thread 0)
template <int OP>
__device__ __forceinline__ double bon_reduce(double v, double *smem)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
  {
    const double t = __shfl_down_sync(0xffffffffu, v, o);
    v              = OP == 0 ? v + t : OP == 1 ? fmin(v, t) : fmax(v, t);
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0)
    smem[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = smem[0];
  if (threadIdx.x == 0)
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k)
      r = OP == 0 ? r + smem[k] : OP == 1 ? fmin(r, smem[k]) : fmax(r, smem[k]);
  return r;
}

template <int D>
__global__ void __launch_bounds__(kBonBlock) bonanni_cells(const BonanniArgs a)
{
  __shared__ double smem[kBonBlock / 32];
  const int c   = blockIdx.x * blockDim.x + threadIdx.x;
  double vol    = 0.0, vint[D], pmin = 1.7976931348623157e308, pmax = -1.7976931348623157e308;
#pragma unroll
  for (int d = 0; d < D; ++d)
    vint[d] = 0.0;
  if (c < a.ncells)
  {
    const double gm1 = a.gamma - 1.0;
    // nodal pressure and velocity (physics/euler/Euler2DCons.hpp:160-190)
    auto node = [&](int n, double V[D]) -> double {
      const int v        = __ldg(a.sol_conn + (size_t)n * a.ncells + c);
      const double rho   = __ldg(a.u + v);
      const double inv   = 1. / rho;
      double v2          = 0.0;
#pragma unroll
      for (int d = 0; d < D; ++d)
      {
        V[d] = __ldg(a.u + (size_t)(1 + d) * a.nnodes + v) * inv;
        v2   = d == 0 ? V[0] * V[0] : v2 + V[d] * V[d];
      }
      const double rhoE = __ldg(a.u + (size_t)(D + 1) * a.nnodes + v);
      return gm1 * (rhoE - 0.5 * rho * v2);
    };
    for (int n = 0; n < a.ndof; ++n)
    {
      double V[D];
      const double p = node(n, V);
      pmin           = fmin(pmin, p);
      pmax           = fmax(pmax, p);
    }
    double X[4][D];
    for (int g = 0; g < a.ngeo && g < 4; ++g)
    {
      const int v = __ldg(a.geo_conn + (size_t)g * a.ncells + c);
#pragma unroll
      for (int d = 0; d < D; ++d)
        X[g][d] = __ldg(a.X + (size_t)d * a.ngeo_nodes + v);
    }
    double pint[D];
#pragma unroll
    for (int d = 0; d < D; ++d)
      pint[d] = 0.0;
    for (int q = 0; q < a.nq; ++q)
    {
      double J[D][D], iJ[D][D];
#pragma unroll
      for (int xi = 0; xi < D; ++xi)
#pragma unroll
        for (int x = 0; x < D; ++x)
        {
          double sj = 0.0;
          for (int g = 0; g < a.ngeo && g < 4; ++g)
            sj += __ldg(a.dVgeo + ((size_t)xi * a.nq + q) * a.ngeo + g) * X[g][x];
          J[xi][x] = sj;
        }
      const double jw = invert<D>(J, iJ) * __ldg(a.w + q);
      vol += jw;
      double vq[D], gref[D];
#pragma unroll
      for (int d = 0; d < D; ++d)
        vq[d] = gref[d] = 0.0;
      for (int n = 0; n < a.ndof; ++n)
      {
        double V[D];
        const double p  = node(n, V);
        const double bn = __ldg(a.V + (size_t)q * a.ndof + n);
#pragma unroll
        for (int d = 0; d < D; ++d)
        {
          vq[d] += bn * V[d];
          gref[d] += __ldg(a.dV + ((size_t)d * a.nq + q) * a.ndof + n) * p;
        }
      }
#pragma unroll
      for (int x = 0; x < D; ++x)
      {
        double gp = 0.0;
#pragma unroll
        for (int xi = 0; xi < D; ++xi)
          gp += iJ[x][xi] * gref[xi];
        vint[x] += jw * vq[x];
        pint[x] += jw * gp;
      }
    }
    double f = 0.0, vn = 0.0;
#pragma unroll
    for (int d = 0; d < D; ++d)
    {
      const double vm = vint[d] / vol;
      f += vm * (pint[d] / vol);
      vn += vm * vm;
    }
    a.f[c]  = f * sqrt(vn);
    a.lc[c] = pow(vol, 1. / D);
  }
  else
    vol = 0.0;
  // block sums for the mesh-wide quantities
  double *pb = a.part + (size_t)blockIdx.x * (D + 3);
  const double bv = bon_reduce<0>(vol, smem);
  if (threadIdx.x == 0)
    pb[0] = bv;
#pragma unroll
  for (int d = 0; d < D; ++d)
  {
    const double t = bon_reduce<0>(vint[d], smem);
    if (threadIdx.x == 0)
      pb[1 + d] = t;
  }
  const double mn = bon_reduce<1>(pmin, smem);
  if (threadIdx.x == 0)
    pb[D + 1] = mn;
  const double mx = bon_reduce<2>(pmax, smem);
  if (threadIdx.x == 0)
    pb[D + 2] = mx;
}

template <int D>
__global__ void __launch_bounds__(kBonBlock)
    bonanni_reduce(int nblocks, const double *__restrict__ part, double *__restrict__ delta)
{
  __shared__ double smem[kBonBlock / 32];
  double r[D + 3];
#pragma unroll
  for (int k = 0; k < D + 3; ++k)
    r[k] = k == D + 1 ? 1.7976931348623157e308 : k == D + 2 ? -1.7976931348623157e308 : 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
  {
    const double *pb = part + (size_t)b * (D + 3);
#pragma unroll
    for (int k = 0; k <= D; ++k)
      r[k] += pb[k];
    r[D + 1] = fmin(r[D + 1], pb[D + 1]);
    r[D + 2] = fmax(r[D + 2], pb[D + 2]);
  }
  double t[D + 3];
#pragma unroll
  for (int k = 0; k <= D; ++k)
    t[k] = bon_reduce<0>(r[k], smem);
  t[D + 1] = bon_reduce<1>(r[D + 1], smem);
  t[D + 2] = bon_reduce<2>(r[D + 2], smem);
  if (threadIdx.x == 0)
  {
    double n2 = 0.0;
#pragma unroll
    for (int d = 0; d < D; ++d)
    {
      const double vd = t[1 + d] / t[0];
      n2 += vd * vd;
    }
    const double nv = sqrt(n2);
    delta[0]        = (t[D + 2] - t[D + 1]) * nv * nv;
  }
}

__global__ void __launch_bounds__(kGBlock)
    bonanni_finish(int n, const double *__restrict__ delta, double *__restrict__ f,
                   const double *__restrict__ lc)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n)
    return;
  const double sc = std_max(f[c] / delta[0], 0.0);
  f[c]            = std_min(1., sc * sc * lc[c]);
}

} // namespace

cudaError_t launch_viscous(const ViscArgs &a, int dim, int neq, cudaStream_t s, const char **name)
{
  if (a.ncells == 0)
    return cudaSuccess;
  if (dim == 2 && neq == 1)
    return launch_viscous_g<2, 1>(a, s, name);
  if (dim == 2 && neq == 4)
    return launch_viscous_g<2, 4>(a, s, name);
  if (dim == 3 && neq == 5)
    return launch_viscous_g<3, 5>(a, s, name);
  return cudaErrorInvalidValue;
}

cudaError_t launch_sensor(const SensorArgs &a, int dim, cudaStream_t s)
{
  if (a.ncells == 0)
    return cudaSuccess;
  const int grid = (a.ncells + kBlock - 1) / kBlock;
  if (dim == 2)
    sensor_cells_2d<<<grid, kBlock, 0, s>>>(a);
  else
    sensor_cells_3d<<<grid, kBlock, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_normalise_max(int n, double *v, cudaStream_t s)
{
  if (n == 0)
    return cudaSuccess;
  normalise_max<<<1, kGBlock, 0, s>>>(n, v);
  return cudaGetLastError();
}

cudaError_t launch_blend_cells(int kind, int ncells, int ndof, const int32_t *sol_conn,
                               const double *u, double param, double *out, cudaStream_t s)
{
  if (ncells == 0)
    return cudaSuccess;
  blend_cells<<<(ncells + kBlock - 1) / kBlock, kBlock, 0, s>>>(kind, ncells, ndof, sol_conn, u,
                                                                param, out);
  return cudaGetLastError();
}

cudaError_t launch_node_max(int nnodes, const int32_t *row, const int32_t *ent_ws, long long wcells,
                            const double *cellf, double *nodef, cudaStream_t s)
{
  node_max<<<(nnodes + kGBlock - 1) / kGBlock, kGBlock, 0, s>>>(nnodes, row, ent_ws, wcells,
                                                                 cellf, nodef);
  return cudaGetLastError();
}

cudaError_t launch_lf_finish(int ncells, int ndof, const int32_t *sol_conn, const double *nodef,
                             double *out, cudaStream_t s)
{
  if (ncells == 0)
    return cudaSuccess;
  lf_finish<<<(ncells + kBlock - 1) / kBlock, kBlock, 0, s>>>(ncells, ndof, sol_conn, nodef, out);
  return cudaGetLastError();
}

cudaError_t launch_cells_to_nodes(int nnodes, const int32_t *row, const int32_t *ent_slot,
                                  long long scells, const StabGroups &g, const double *cellf,
                                  double *nodef, cudaStream_t s)
{
  const int grid = (nnodes + kGBlock - 1) / kGBlock;
  cudaError_t e  = cudaMemsetAsync(nodef, 0, (size_t)nnodes * sizeof(double), s);
  if (e != cudaSuccess)
    return e;
  vertex_max<<<grid, kGBlock, 0, s>>>(nnodes, row, ent_slot, scells, g, cellf, nodef);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return e;
  interior_interp<<<grid, kGBlock, 0, s>>>(nnodes, row, ent_slot, scells, g, nodef);
  return cudaGetLastError();
}

int bonanni_blocks(int ncells)
{
  return (ncells + kBonBlock - 1) / kBonBlock;
}

cudaError_t launch_bonanni_cells(const BonanniArgs &a, int dim, cudaStream_t s)
{
  if (a.ncells == 0)
    return cudaSuccess;
  if (a.ngeo > 4)
    return cudaErrorInvalidValue;
  const int grid = bonanni_blocks(a.ncells);
  if (dim == 2)
    bonanni_cells<2><<<grid, kBonBlock, 0, s>>>(a);
  else
    bonanni_cells<3><<<grid, kBonBlock, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_bonanni_finish(int dim, int nblocks, const double *part, double *delta, int n,
                                  double *f, const double *lc, cudaStream_t s)
{
  if (dim == 2)
    bonanni_reduce<2><<<1, kBonBlock, 0, s>>>(nblocks, part, delta);
  else
    bonanni_reduce<3><<<1, kBonBlock, 0, s>>>(nblocks, part, delta);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || n == 0)
    return e;
  bonanni_finish<<<(n + kGBlock - 1) / kGBlock, kGBlock, 0, s>>>(n, delta, f, lc);
  return cudaGetLastError();
}

} // namespace rds
