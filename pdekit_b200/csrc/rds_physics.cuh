// Pointwise physics on the device: properties, physical flux, and upwind matrices
// K = R op(Lambda) L for a direction, for Burgers, constant advection and the 2D/3D Euler
// equations in conservative variables.
//
// Reference: physics/scalar/Burgers2D.hpp:154-296, physics/scalar/RotationAdvection2D.hpp:201-336,
// physics/euler/Euler2DCons.hpp:159-536, physics/euler/Euler3DCons.hpp:160-560. The Euler
// eigenvectors are those of the normalised direction, the eigenvalues are scaled by its norm;
// gamma = 1.4 (physics/euler/Euler2DProperties.cpp:13-15).
#pragma once

#include <cuda_runtime.h>

namespace rds
{

template <typename T, int D>
struct EulerProps
{
  T rho, inv_rho, V[D], v2, P, H, a;
};

// Returns true when the pressure is not positive (the reference prints a diagnostic there,
// Euler2DCons.hpp:188-201; here the caller raises a status flag).
template <typename T, int D>
__device__ __forceinline__ bool euler_props(const T *u, T gamma, EulerProps<T, D> &p)
{
  const T gm1 = gamma - T(1);
  p.rho       = u[0];
  p.inv_rho   = T(1) / p.rho;
#pragma unroll
  for (int d = 0; d < D; ++d)
    p.V[d] = u[1 + d] * p.inv_rho;
  T v2 = p.V[0] * p.V[0] + p.V[1] * p.V[1];
  if (D == 3)
    v2 = v2 + p.V[D - 1] * p.V[D - 1];
  p.v2        = v2;
  const T rhoE = u[D + 1];
  p.P         = gm1 * (rhoE - T(0.5) * p.rho * p.v2);
  const T RT  = p.P * p.inv_rho;
  p.H         = rhoE * p.inv_rho + RT;
  p.a         = sqrt(gamma * RT);
  return !(p.P > T(0));
}

// Physical flux F[e][d] at one point.
template <typename T, int D>
__device__ __forceinline__ void euler_flux(const T *u, const EulerProps<T, D> &p, T F[][D])
{
#pragma unroll
  for (int d = 0; d < D; ++d)
  {
    const T m = u[1 + d]; // rho * V_d
    F[0][d]   = m;
#pragma unroll
    for (int k = 0; k < D; ++k)
      F[1 + k][d] = m * p.V[k] + (k == d ? p.P : T(0));
    F[D + 1][d] = m * p.H;
  }
}

// Flux through direction n: F(u) . n (Euler2DCons::flux(p, direction, flux),
// physics/euler/Euler2DCons.hpp:253-266; Euler3DCons.hpp:267-285).
template <typename T, int D>
__device__ __forceinline__ void euler_flux_n(const T *u, const EulerProps<T, D> &p, const T *n,
                                             T *F)
{
  T rhoum = u[1] * n[0] + u[2] * n[1];
  if (D == 3)
    rhoum = u[1] * n[0] + u[2] * n[1] + u[D] * n[D - 1];
  F[0] = rhoum;
#pragma unroll
  for (int d = 0; d < D; ++d)
    F[1 + d] = rhoum * p.V[d] + p.P * n[d];
  F[D + 1] = rhoum * p.H;
}

// Right/left eigenvectors R, L and eigenvalues lam of the flux Jacobian in direction dir.
template <typename T>
__device__ __forceinline__ void euler_eigen(const EulerProps<T, 2> &p, const T *dir, T gamma,
                                            T R[4][4], T L[4][4], T lam[4])
{
  const T norm = sqrt(dir[0] * dir[0] + dir[1] * dir[1]);
  const T nx   = (norm < T(1.e-9)) ? dir[0] : dir[0] / norm;
  const T ny   = (norm < T(1.e-9)) ? dir[1] : dir[1] / norm;
  const T gm1  = gamma - T(1);
  const T inv_a = T(1) / p.a, inv_a2 = inv_a * inv_a;
  const T u = p.V[0], v = p.V[1];
  const T um      = u * nx + v * ny;
  const T ra      = T(0.5) * p.rho * inv_a;
  const T coeffM2 = (T(0.5) * gm1 * p.v2) * inv_a2;
  const T uDivA   = gm1 * u * inv_a;
  const T vDivA   = gm1 * v * inv_a;
  const T gm1_ov_rhoa = gm1 / (p.rho * p.a);
  const T ir = p.inv_rho, a = p.a, H = p.H, rho = p.rho;
  R[0][0] = T(1);
  R[0][1] = T(0);
  R[0][2] = ra;
  R[0][3] = ra;
  R[1][0] = u;
  R[1][1] = rho * ny;
  R[1][2] = ra * (u + a * nx);
  R[1][3] = ra * (u - a * nx);
  R[2][0] = v;
  R[2][1] = -rho * nx;
  R[2][2] = ra * (v + a * ny);
  R[2][3] = ra * (v - a * ny);
  R[3][0] = T(0.5) * p.v2;
  R[3][1] = rho * (u * ny - v * nx);
  R[3][2] = ra * (H + a * um);
  R[3][3] = ra * (H - a * um);
  L[0][0] = T(1) - coeffM2;
  L[0][1] = uDivA * inv_a;
  L[0][2] = vDivA * inv_a;
  L[0][3] = -gm1 * inv_a2;
  L[1][0] = ir * (v * nx - u * ny);
  L[1][1] = ir * ny;
  L[1][2] = -ir * nx;
  L[1][3] = T(0);
  L[2][0] = a * ir * (coeffM2 - um * inv_a);
  L[2][1] = ir * (nx - uDivA);
  L[2][2] = ir * (ny - vDivA);
  L[2][3] = gm1_ov_rhoa;
  L[3][0] = a * ir * (coeffM2 + um * inv_a);
  L[3][1] = -ir * (nx + uDivA);
  L[3][2] = -ir * (ny + vDivA);
  L[3][3] = gm1_ov_rhoa;
  lam[0]  = norm * um;
  lam[1]  = norm * um;
  lam[2]  = norm * (um + a);
  lam[3]  = norm * (um - a);
}

template <typename T>
__device__ __forceinline__ void euler_eigen(const EulerProps<T, 3> &p, const T *dir, T gamma,
                                            T R[5][5], T L[5][5], T lam[5])
{
  const T norm = sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
  const T nx   = (norm == T(0)) ? dir[0] : dir[0] / norm;
  const T ny   = (norm == T(0)) ? dir[1] : dir[1] / norm;
  const T nz   = (norm == T(0)) ? dir[2] : dir[2] / norm;
  const T gm1  = gamma - T(1);
  const T inv_a = T(1) / p.a, inv_a2 = inv_a * inv_a;
  const T u = p.V[0], v = p.V[1], w = p.V[2];
  const T um   = u * nx + v * ny + w * nz;
  const T ra   = T(0.5) * p.rho * inv_a;
  const T gu_a = gm1 * u * inv_a, gv_a = gm1 * v * inv_a, gw_a = gm1 * w * inv_a;
  const T gm1_ov_rhoa = gm1 / (p.rho * p.a);
  const T ke  = T(0.5) * p.v2;
  const T gm2 = (T(0.5) * gm1 * p.v2) * inv_a2;
  const T k2  = T(1) - gm2;
  const T k3  = -gm1 * inv_a2;
  const T rho = p.rho, ir = p.inv_rho, a = p.a, H = p.H;
  R[0][0] = nx;
  R[0][1] = ny;
  R[0][2] = nz;
  R[0][3] = ra;
  R[0][4] = ra;
  R[1][0] = u * nx;
  R[1][1] = u * ny - rho * nz;
  R[1][2] = u * nz + rho * ny;
  R[1][3] = ra * (u + a * nx);
  R[1][4] = ra * (u - a * nx);
  R[2][0] = v * nx + rho * nz;
  R[2][1] = v * ny;
  R[2][2] = v * nz - rho * nx;
  R[2][3] = ra * (v + a * ny);
  R[2][4] = ra * (v - a * ny);
  R[3][0] = w * nx - rho * ny;
  R[3][1] = w * ny + rho * nx;
  R[3][2] = w * nz;
  R[3][3] = ra * (w + a * nz);
  R[3][4] = ra * (w - a * nz);
  R[4][0] = ke * nx + rho * (v * nz - w * ny);
  R[4][1] = ke * ny + rho * (w * nx - u * nz);
  R[4][2] = ke * nz + rho * (u * ny - v * nx);
  R[4][3] = ra * (H + a * um);
  R[4][4] = ra * (H - a * um);
  L[0][0] = nx * k2 - ir * (v * nz - w * ny);
  L[0][1] = gu_a * inv_a * nx;
  L[0][2] = gv_a * inv_a * nx + nz * ir;
  L[0][3] = gw_a * inv_a * nx - ny * ir;
  L[0][4] = k3 * nx;
  L[1][0] = ny * k2 - ir * (w * nx - u * nz);
  L[1][1] = gu_a * inv_a * ny - nz * ir;
  L[1][2] = gv_a * inv_a * ny;
  L[1][3] = gw_a * inv_a * ny + nx * ir;
  L[1][4] = k3 * ny;
  L[2][0] = nz * k2 - ir * (u * ny - v * nx);
  L[2][1] = gu_a * inv_a * nz + ny * ir;
  L[2][2] = gv_a * inv_a * nz - nx * ir;
  L[2][3] = gw_a * inv_a * nz;
  L[2][4] = k3 * nz;
  L[3][0] = a * ir * (gm2 - um / a);
  L[3][1] = ir * (nx - gu_a);
  L[3][2] = ir * (ny - gv_a);
  L[3][3] = ir * (nz - gw_a);
  L[3][4] = gm1_ov_rhoa;
  L[4][0] = a * ir * (gm2 + um / a);
  L[4][1] = ir * (-nx - gu_a);
  L[4][2] = ir * (-ny - gv_a);
  L[4][3] = ir * (-nz - gw_a);
  L[4][4] = gm1_ov_rhoa;
  lam[0]  = norm * um;
  lam[1]  = norm * um;
  lam[2]  = norm * um;
  lam[3]  = norm * (um + a);
  lam[4]  = norm * (um - a);
}

// K = R op(Lambda) L with op = max(0,.) (SIGN > 0) or min(0,.) (SIGN < 0); lam keeps the
// unclipped eigenvalues.
template <int SIGN, typename T, int D>
__device__ __forceinline__ void euler_K(const EulerProps<T, D> &p, const T *dir, T gamma,
                                        T K[D + 2][D + 2], T lam[D + 2])
{
  constexpr int N = D + 2;
  T R[N][N], L[N][N];
  euler_eigen(p, dir, gamma, R, L, lam);
  T lo[N];
#pragma unroll
  for (int k = 0; k < N; ++k)
    lo[k] = SIGN > 0 ? (lam[k] > T(0) ? lam[k] : T(0)) : (lam[k] < T(0) ? lam[k] : T(0));
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j)
    {
      T s = R[i][0] * lo[0] * L[0][j];
#pragma unroll
      for (int k = 1; k < N; ++k)
        s = s + R[i][k] * lo[k] * L[k][j];
      K[i][j] = s;
    }
}

// Direction-independent factors of the acoustic eigenvectors at one state: computed once per
// point and shared by the upwind matrices of all nodes there.
template <typename T, int D>
struct EulerAcoustic
{
  T inv_a;  // 1 / a
  T ra;     // rho / (2 a)
  T kin;    // (gamma - 1) |V|^2 / (2 a^2)
  T gV[D];  // (gamma - 1) V_d / a
  T g_rhoa; // (gamma - 1) / (rho a)
};

template <typename T, int D>
__device__ __forceinline__ void euler_acoustic(const EulerProps<T, D> &p, T gamma,
                                               EulerAcoustic<T, D> &c)
{
  const T gm1 = gamma - T(1);
  c.inv_a     = T(1) / p.a;
  c.ra        = T(0.5) * p.rho * c.inv_a;
  c.kin       = (T(0.5) * gm1 * p.v2) * (c.inv_a * c.inv_a);
#pragma unroll
  for (int d = 0; d < D; ++d)
    c.gV[d] = gm1 * p.V[d] * c.inv_a;
  c.g_rhoa = gm1 * p.inv_rho * c.inv_a;
}

// K = R op(Lambda) L for direction dir (op = max(0, .) for SIGN > 0, min(0, .) for SIGN < 0,
// the identity for SIGN == 0: the flux Jacobian in direction dir), in split form. The convective eigenvalue lam_c = |dir| u.n has multiplicity D and the eigenvector
// pairs satisfy sum_k r_k l_k^T = I, so
//   K = op(lam_c) I + (op(lam_+) - op(lam_c)) r_+ l_+^T + (op(lam_-) - op(lam_c)) r_- l_-^T
// where r_+- = rho/(2a) (1, V +- a n, H +- a u.n) and l_+- are the acoustic eigenvector pairs
// (columns / rows D and D + 1 of R and L in euler_eigen): two rank-one updates instead of the
// product of three N x N matrices. The factors: K = oc I + rp lp^T + rm lm^T.
template <typename T, int D>
struct EulerKFactors
{
  T oc;         // op(lam_c)
  T rp[D + 2];  // (op(lam_+) - op(lam_c)) r_+
  T rm[D + 2];  // (op(lam_-) - op(lam_c)) r_-
  T lp[D + 2];  // l_+
  T lm[D + 2];  // l_-
};

// The factors of K for direction dir; returns max_k max(1e-6, |lam_k|).
template <int SIGN, typename T, int D>
__device__ __forceinline__ T euler_K_factors(const EulerProps<T, D> &p,
                                             const EulerAcoustic<T, D> &c, const T *dir,
                                             EulerKFactors<T, D> &f)
{
  constexpr int N = D + 2;
  T n2            = dir[0] * dir[0] + dir[1] * dir[1];
  if (D == 3)
    n2 = n2 + dir[D - 1] * dir[D - 1];
  // |dir| and 1/|dir| from one reciprocal square root
  const T rn   = n2 > T(0) ? rsqrt(n2) : T(0);
  const T norm = n2 * rn;
  // the reference keeps dir unnormalised below |dir| = 1e-9 (2D) or at |dir| = 0 (3D)
  const bool keep = (D == 2) ? (norm < T(1.e-9)) : (norm == T(0));
  const T inv_n   = keep ? T(1) : rn;
  T n[D];
#pragma unroll
  for (int d = 0; d < D; ++d)
    n[d] = dir[d] * inv_n;
  T um = p.V[0] * n[0] + p.V[1] * n[1];
  if (D == 3)
    um = um + p.V[D - 1] * n[D - 1];
  const T a  = p.a;
  const T lc = norm * um, lp = norm * (um + a), lm = norm * (um - a);
  auto op    = [](T x) -> T {
    return SIGN > 0 ? (x > T(0) ? x : T(0)) : SIGN < 0 ? (x < T(0) ? x : T(0)) : x;
  };
  const T oc = op(lc);
  const T ap = (op(lp) - oc) * c.ra, am = (op(lm) - oc) * c.ra;
  f.oc       = oc;
  f.rp[0]    = ap;
  f.rm[0]    = am;
#pragma unroll
  for (int d = 0; d < D; ++d)
  {
    f.rp[1 + d] = ap * (p.V[d] + a * n[d]);
    f.rm[1 + d] = am * (p.V[d] - a * n[d]);
    f.lp[1 + d] = p.inv_rho * (n[d] - c.gV[d]);
    f.lm[1 + d] = -p.inv_rho * (n[d] + c.gV[d]);
  }
  f.rp[N - 1] = ap * (p.H + a * um);
  f.rm[N - 1] = am * (p.H - a * um);
  f.lp[0]     = a * p.inv_rho * (c.kin - um * c.inv_a);
  f.lm[0]     = a * p.inv_rho * (c.kin + um * c.inv_a);
  f.lp[N - 1] = c.g_rhoa;
  f.lm[N - 1] = c.g_rhoa;
  return fmax(fmax(T(1.e-6), fabs(lc)), fmax(fabs(lp), fabs(lm)));
}

// K itself, from its factors; returns max_k max(1e-6, |lam_k|).
template <int SIGN, typename T, int D>
__device__ __forceinline__ T euler_K_split(const EulerProps<T, D> &p,
                                           const EulerAcoustic<T, D> &c, const T *dir,
                                           T K[D + 2][D + 2])
{
  constexpr int N = D + 2;
  EulerKFactors<T, D> f;
  const T ws = euler_K_factors<SIGN, T, D>(p, c, dir, f);
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j)
    {
      const T s = f.rp[i] * f.lp[j] + f.rm[i] * f.lm[j];
      K[i][j]   = (i == j) ? f.oc + s : s;
    }
  return ws;
}

} // namespace rds
