"""Test oracle (test infrastructure only; the product never imports it): a numpy restatement of
the reference's stabilisation operators that sit either side of the cell residual.

* `sensor_cells`: the Persson-Peraire smoothness sensor per cell
  (src/solver/art_visc/ArtificialViscosity.hpp:300-455, and the same sensor as a blending
  coefficient in src/solver/rdm/blending_coeff/ArtViscIndicatorCoeffImpl.hpp:261-425): the
  first state component is projected in L2 onto the cell's modal basis of order p, the modes
  of total degree p are dropped (at p = 1 all modes), Se = int (u - u_{p-1})^2 / int u^2 (0
  when the denominator is <= 1e-10), se = log10 Se, s0 = 1/p^4, and the value is 0 below s0 - kappa, eps0 above
  s0 + kappa, 0.5 eps0 (1 + sin(pi (se - s0) / (2 kappa))) between; eps0 = factor h / p with
  h = |K|^(1/D) for the viscosity, eps0 = 1 for the blending coefficient.
  Restated with an explicit orthogonal (Dubiner) basis in collapsed coordinates
  (M. Dubiner, J. Sci. Comput. 6, 1991; the basis the reference registers as the modal basis
  of triangles and tetrahedra, mesh/shape_function/ModalBasisFactory.cpp:36-46) and
  collapsed-coordinate Gauss-Legendre quadrature exact to degree 2p (the reference integrates
  with its Gauss rule of order max(2p, geometry order); on affine cells both are exact).
  Bilinear quadrilaterals follow the reference step by step: its tensor Legendre modal basis
  and leading-term flags, its Gauss rule of order 2p, detJ at every point, the cell's mass
  matrix and its solve (at p >= 2 that mass matrix is singular in the reference; the
  projection there uses a rule that keeps it regular, see sensor_cells).
* `nodal_from_cells`: the cell-to-node transfer
  (src/interpolation/mesh_function/MeshFunctionTools.hpp:52-397 without adaptation): every
  vertex takes max(0, max over its cells), every other node the P1 interpolant of the vertex
  values of the last cell (in cell order) that holds it.
* `blend_cells`: LF_Blend (blending_coeff/LFBlendingCoeffImpl.hpp:76-126), WongJansen
  (WongJansenBlendingCoeffImpl.hpp:80-116), ViscosityIndicator (the sensor with eps0 = 1).
* `bonanni`: Bonanni's pressure-based coefficient (BonanniBlendingCoeffImpl.hpp:171-392) of an
  Euler state: per cell, with a Gauss rule of order max(p, 1), the volume, the integrals of the
  velocity and of grad p (p = (gamma - 1)(rhoE - rho |V|^2 / 2) and V from the nodal states,
  physics/euler/Euler2DCons.hpp:160-190), f = (v_m . gp_m)|v_m| (means over the cell) and
  lc = |K|^(1/D); over the mesh p_min, p_max and v_dom = sum int V / sum |K|;
  theta = min(1, max(f / ((p_max - p_min)|v_dom|^2), 0)^2 lc) with std::min / std::max's
  comparisons. Quadrilaterals use the reference's rule (at the orders max(p, 1) <= 3 used here,
  tensor Gauss-Legendre with order // 2 + 1 points per direction,
  mesh/point_set/QdPointSetQuadGauss.cpp); simplices a collapsed rule
  exact to degree 2p (their integrands have degree <= p on affine cells).

Pinned against the reference's own outputs (tests/golden/*_av, *_lf, *_wj, *_visc, *_bonanni,
dumped by oracle/ref_harness.cpp through the reference's classes).
"""

from __future__ import annotations

import numpy as np
from scipy.special import eval_jacobi


# ---- quadrature: collapsed-coordinate Gauss-Legendre (Duffy) rules on the reference simplex
def _simplex_rule(dim: int, n: int):
    x, w = np.polynomial.legendre.leggauss(n)
    if dim == 2:
        a, b = np.meshgrid(x, x, indexing="ij")
        wa, wb = np.meshgrid(w, w, indexing="ij")
        a, b, wt = a.ravel(), b.ravel(), (wa * wb).ravel() * (1 - b.ravel()) / 2
        xi = (1 + a) * (1 - b) / 2 - 1
        return np.stack([xi, b], 1), wt
    a, b, c = np.meshgrid(x, x, x, indexing="ij")
    wa, wb, wc = np.meshgrid(w, w, w, indexing="ij")
    a, b, c = a.ravel(), b.ravel(), c.ravel()
    wt = (wa * wb * wc).ravel() * (1 - b) / 2 * ((1 - c) / 2) ** 2
    zeta = c
    eta = (1 + b) * (1 - c) / 2 - 1
    xi = (1 + a) * (1 - b) / 2 * (1 - c) / 2 - 1
    return np.stack([xi, eta, zeta], 1), wt


# ---- Dubiner basis of total degree <= p at points of the reference simplex
def _dubiner(dim: int, p: int, pts: np.ndarray):
    """[npts, nmodes] values and the degree of each mode."""
    cols, deg = [], []
    if dim == 2:
        xi, eta = pts[:, 0], pts[:, 1]
        den = np.where(np.abs(1 - eta) < 1e-15, 1e-15, 1 - eta)
        a = 2 * (1 + xi) / den - 1
        for i in range(p + 1):
            for j in range(p + 1 - i):
                cols.append(eval_jacobi(i, 0, 0, a) * ((1 - eta) / 2) ** i *
                            eval_jacobi(j, 2 * i + 1, 0, eta))
                deg.append(i + j)
    else:
        xi, eta, zeta = pts[:, 0], pts[:, 1], pts[:, 2]
        d1 = np.where(np.abs(-eta - zeta) < 1e-15, 1e-15, -eta - zeta)
        d2 = np.where(np.abs(1 - zeta) < 1e-15, 1e-15, 1 - zeta)
        a = 2 * (1 + xi) / d1 - 1
        b = 2 * (1 + eta) / d2 - 1
        for i in range(p + 1):
            for j in range(p + 1 - i):
                for k in range(p + 1 - i - j):
                    cols.append(eval_jacobi(i, 0, 0, a) * ((1 - b) / 2) ** i *
                                eval_jacobi(j, 2 * i + 1, 0, b) * ((1 - zeta) / 2) ** (i + j) *
                                eval_jacobi(k, 2 * i + 2 * j + 2, 0, zeta))
                    deg.append(i + j + k)
    return np.stack(cols, 1), np.asarray(deg)


def _monomials(dim: int, p: int, pts: np.ndarray):
    cols = []
    if dim == 2:
        for i in range(p + 1):
            for j in range(p + 1 - i):
                cols.append(pts[:, 0] ** i * pts[:, 1] ** j)
    else:
        for i in range(p + 1):
            for j in range(p + 1 - i):
                for k in range(p + 1 - i - j):
                    cols.append(pts[:, 0] ** i * pts[:, 1] ** j * pts[:, 2] ** k)
    return np.stack(cols, 1)


def lagrange_at(dim: int, p: int, nodes: np.ndarray, pts: np.ndarray):
    """Nodal Lagrange basis through `nodes` (reference coordinates) evaluated at `pts`."""
    return _monomials(dim, p, pts) @ np.linalg.inv(_monomials(dim, p, nodes))


def q1_at(nodes: np.ndarray):
    """[ndof, 4] bilinear values of the square's corners (-1,-1), (1,-1), (1,1), (-1,1) at the
    solution nodes of a quadrilateral."""
    x, y = nodes[:, 0], nodes[:, 1]
    return np.stack([(1 - x) * (1 - y), (1 + x) * (1 - y), (1 + x) * (1 + y),
                     (1 - x) * (1 + y)], 1) / 4


def p1_at(dim: int, nodes: np.ndarray):
    """[ndof, dim+1] P1 (barycentric) values of the vertices at the solution nodes."""
    lam = [-(np.sum(nodes, 1) + (dim - 2)) / 2] + [(1 + nodes[:, d]) / 2 for d in range(dim)]
    return np.stack(lam, 1)


def _ramp(se, s0, kappa, eps0):
    return np.where(se < s0 - kappa, 0.0,
                    np.where(se > s0 + kappa, eps0,
                             0.5 * eps0 * (1 + np.sin(np.pi * (se - s0) / (2 * kappa)))))


def _legendre_quad(p: int, pts: np.ndarray):
    """The reference's modal basis of quadrilaterals (mesh/shape_function/
    ModalExpansionQuad.cpp:60-73): mode (m, n), m-major, P_m(xi) P_n(eta) / sqrt(g_m g_n) with
    g_k = 2 / (2k + 1); and its leading-term flags (ModalExpansionQuad.cpp:240-257), which
    advance the mode index only on modes with m == p or n == p and so set the FIRST 2p + 1 flags
    (the constant mode among them), not those of the modes of degree p."""
    cols = []
    for m in range(p + 1):
        for n in range(p + 1):
            cols.append(eval_jacobi(m, 0, 0, pts[:, 0]) * eval_jacobi(n, 0, 0, pts[:, 1]) /
                        np.sqrt(2.0 / (2 * m + 1) * 2.0 / (2 * n + 1)))
    flags = np.zeros((p + 1) ** 2, dtype=bool)
    flags[:2 * p + 1] = True
    return np.stack(cols, 1), flags


def _gauss_quad(order: int):
    """The reference's Gauss rule of the square for orders 2 - 7
    (mesh/point_set/QdPointSetQuadGauss.cpp): 2 x 2 Gauss-Legendre up to order 3, then the fully
    symmetric rules of degree 5 (8 points) and 7 (12 points) of A. H. Stroud (1971, region C2)
    in closed form: orbits (+-a, 0), (0, +-a) of weight A and (+-b, +-b) of weight B (and
    (+-c, +-c) of weight C), from the moment equations of the square."""
    if order <= 3:
        x, w = np.polynomial.legendre.leggauss(2)
        X, Y = np.meshgrid(x, x, indexing="ij")
        return np.stack([X.ravel(), Y.ravel()], 1), np.outer(w, w).ravel()
    if order <= 5:
        # int x^4 y^0 and int x^2 y^2 fix A a^4 = 8/45 and B b^4 = 1/9
        orbits = [("a0", 40.0 / 49.0, np.sqrt(7.0 / 15.0)), ("aa", 9.0 / 49.0, np.sqrt(7.0 / 9.0))]
    elif order <= 7:
        # int x^4 - int x^2 y^2 and int x^6 - int x^4 y^2 give a^2 = 6/7, A = 98/405; the two
        # diagonal orbits are then the 2-point Gauss rule of the moments m0..m3 left for them
        A, a2 = 98.0 / 405.0, 6.0 / 7.0
        m = [1.0 - A, 1.0 / 3.0 - A * a2 / 2.0, 1.0 / 9.0, 1.0 / 15.0]
        p1, p0 = np.linalg.solve([[m[1], m[0]], [m[2], m[1]]], [-m[2], -m[3]])
        u, v = np.roots([1.0, p1, p0])
        B = (m[1] - v * m[0]) / (u - v)
        orbits = [("a0", A, np.sqrt(a2)), ("aa", B, np.sqrt(u)), ("aa", m[0] - B, np.sqrt(v))]
    else:
        raise ValueError(f"no square rule of order {order} here")
    pts, w = [], []
    for kind, wt, a in orbits:
        orb = ([(a, 0.0), (-a, 0.0), (0.0, a), (0.0, -a)] if kind == "a0" else
               [(a, a), (a, -a), (-a, a), (-a, -a)])
        pts += orb
        w += [wt] * 4
    return np.asarray(pts), np.asarray(w)


def sensor_cells(dim, p, sol_nodes, geo_coords, geo_conn, sol_conn, u0, kappa=5.0, factor=1.0,
                 blend=False):
    """Cellwise artificial viscosity (blend=False) or ViscosityIndicator blending coefficient
    (blend=True) of the first state component u0 [nnodes] on affine simplices, or on bilinear
    quadrilaterals (dim 2 with 4 geometry nodes a cell: the Gauss rule of order 2p, detJ per
    point, the reference's quadrilateral modal basis and flags). On quadrilaterals of order
    p >= 2 the reference's rule has fewer points than the cell has modes and its mass matrix is
    singular (its result follows the rounding of the inversion); there the projection is taken
    with the (p + 1)^2-point tensor Gauss rule, which makes the mass matrix regular, and the
    integrals of Se with the reference's rule."""
    quad = dim == 2 and geo_conn.shape[1] == 4
    proj = None
    if quad:
        qp, qw = _gauss_quad(2 * p)
        Vn, _ = _basis(2, p, sol_nodes, qp, True)
        Vm, flags = _legendre_quad(p, qp)
        Vl = Vm * ~flags
        _, dG = _basis(2, 1, _QUAD_CORNERS, qp, True)                 # [2, nq, 4]
        Jq = np.einsum("aqg,cgx->cqax", dG, geo_coords[geo_conn])    # [nc, nq, xi, x]
        jdet = np.linalg.det(Jq)                                      # [nc, nq]
        if p >= 2:
            x, w1 = np.polynomial.legendre.leggauss(p + 1)
            X, Y = np.meshgrid(x, x, indexing="ij")
            pp, pw = np.stack([X.ravel(), Y.ravel()], 1), np.outer(w1, w1).ravel()
            _, dGp = _basis(2, 1, _QUAD_CORNERS, pp, True)
            proj = (pw, _basis(2, p, sol_nodes, pp, True)[0], _legendre_quad(p, pp)[0],
                    np.linalg.det(np.einsum("aqg,cgx->cqax", dGp, geo_coords[geo_conn])))
    else:
        qp, qw = _simplex_rule(dim, p + 2)
        Vn = lagrange_at(dim, p, sol_nodes, qp)
        Vm, deg = _dubiner(dim, p, qp)
        # the modes of degree p switched off; at p = 1 the reference marks every mode, the
        # constant included, as leading (mesh/shape_function/DubinerExpansionTriag.cpp:460-467,
        # DubinerExpansionTetra.cpp:715-723), so u_{p-1} = 0 there
        Vl = Vm * (deg < p) if p > 1 else 0.0 * Vm
        X = geo_coords[geo_conn[:, :dim + 1]]     # [nc, dim+1, dim] vertex coordinates
        J = np.stack([X[:, k + 1] - X[:, 0] for k in range(dim)], 2) / 2  # dx/dxi
        jdet = np.linalg.det(J)[:, None] * np.ones(len(qw))
    out = np.empty(len(sol_conn))
    s0 = 1.0 / p ** 4
    for c in range(len(sol_conn)):
        wj = jdet[c] * qw
        if proj is None:
            wp, Vnp, Vmp = wj, Vn, Vm
        else:
            wp, Vnp, Vmp = proj[3][c] * proj[0], proj[1], proj[2]
        up = Vnp @ u0[sol_conn[c]]
        M = (Vmp * wp[:, None]).T @ Vmp
        cm = np.linalg.solve(M, (Vmp * (wp * up)[:, None]).sum(0))
        uq = Vm @ cm
        ul = Vl @ cm
        nom = np.sum(wj * (uq - ul) ** 2)
        den = np.sum(wj * uq * uq)
        Se = 0.0 if den <= 1e-10 else nom / den
        with np.errstate(divide="ignore"):
            se = np.log(Se) / np.log(10.0)
        if blend:
            out[c] = _ramp(se, s0, kappa, 1.0)
        else:
            h = np.sum(wj) ** (1.0 / dim)
            out[c] = factor * _ramp(se, s0, kappa, h / p)
    return out


def nodal_from_cells(f_cells, sol_conn, nnodes, P1):
    """Cell values -> nodal values (see the module docstring). P1 [ndof, nvert]."""
    nvert = P1.shape[1]
    f = np.zeros(nnodes)
    vert = sol_conn[:, :nvert]
    np.maximum.at(f, vert.ravel(), np.repeat(f_cells, nvert))
    for c in range(len(sol_conn)):
        fv = f[vert[c]]
        for n in range(nvert, sol_conn.shape[1]):
            f[sol_conn[c, n]] = sum(P1[n, i] * fv[i] for i in range(nvert))
    return f


def blend_cells(kind, sol_conn, u0, param=None):
    """LF_Blend / WongJansen cellwise blending coefficients of the first state component."""
    uc = u0[sol_conn]
    uavg = uc.sum(1) / sol_conn.shape[1]
    if kind == "LF_Blend":
        ksi = np.max(np.abs(uc - uavg[:, None]) / (np.abs(uc) + np.abs(uavg)[:, None] + 1e-12), 1)
        th = np.zeros(int(sol_conn.max()) + 1)
        np.maximum.at(th, sol_conn.ravel(), np.repeat(ksi, sol_conn.shape[1]))
        return 1.0 - th[sol_conn].max(1)
    if kind == "WongJansen":
        u_inf = 1e-14 if param is None else param
        t = (uc * uc - (uavg * uavg)[:, None]) ** 2
        nom = np.zeros(len(uc))
        den = np.full(len(uc), 1.0 * u_inf ** 4)
        for n in range(uc.shape[1]):
            nom += t[:, n]
            den += t[:, n]
        return nom / den
    raise ValueError(kind)


# ---- Bonanni's pressure-based coefficient
_QUAD_CORNERS = np.array([[-1.0, -1.0], [1.0, -1.0], [1.0, 1.0], [-1.0, 1.0]])


def _mono_terms(dim, p, tensor):
    if dim == 2:
        return [(i, j) for i in range(p + 1) for j in range(p + 1) if tensor or i + j <= p]
    return [(i, j, k) for i in range(p + 1) for j in range(p + 1) for k in range(p + 1)
            if i + j + k <= p]


def _mono(terms, pts):
    return np.stack([np.prod([pts[:, d] ** e[d] for d in range(len(e))], 0) for e in terms], 1)


def _mono_d(terms, pts, axis):
    cols = []
    for e in terms:
        if e[axis] == 0:
            cols.append(np.zeros(len(pts)))
            continue
        c = float(e[axis])
        for d in range(len(e)):
            c = c * pts[:, d] ** (e[d] - 1 if d == axis else e[d])
        cols.append(c)
    return np.stack(cols, 1)


def _basis(dim, p, nodes, pts, tensor):
    """Lagrange basis through `nodes` at `pts`: values [npts, n] and derivatives [dim, npts, n]."""
    terms = _mono_terms(dim, p, tensor)
    inv = np.linalg.inv(_mono(terms, nodes))
    return _mono(terms, pts) @ inv, np.stack([_mono_d(terms, pts, a) @ inv for a in range(dim)])


def _bonanni_rule(dim, shape, p):
    if shape == "quad":
        x, w = np.polynomial.legendre.leggauss(max(p, 1) // 2 + 1)
        X, Y = np.meshgrid(x, x, indexing="ij")
        return np.stack([X.ravel(), Y.ravel()], 1), np.outer(w, w).ravel()
    return _simplex_rule(dim, p + 1)


def bonanni(groups, u0, gamma, dim):
    """theta per cell (groups in order). groups: (shape, p, sol_nodes [ndof, dim] reference
    coordinates, geo_coords [n, dim], geo_conn [ncells, ngeo], sol_conn [ncells, ndof])."""
    gm1 = gamma - 1.0
    rho = u0[:, 0]
    V = u0[:, 1:1 + dim] / rho[:, None]
    v2 = np.zeros(len(rho))
    for d in range(dim):
        v2 = V[:, 0] * V[:, 0] if d == 0 else v2 + V[:, d] * V[:, d]
    P = gm1 * (u0[:, dim + 1] - 0.5 * rho * v2)
    f_all, lc_all = [], []
    dom_vol, v_dom = 0.0, np.zeros(dim)
    p_min, p_max = np.inf, -np.inf
    for shape, p, sol_nodes, geo_coords, geo_conn, sol_conn in groups:
        tensor = shape == "quad"
        pts, w = _bonanni_rule(dim, shape, p)
        B, dB = _basis(dim, p, sol_nodes, pts, tensor)
        corners = _QUAD_CORNERS if tensor else np.vstack([-np.ones(dim), -np.ones(dim) +
                                                         2 * np.eye(dim)])
        _, dG = _basis(dim, 1, corners, pts, tensor)
        for c in range(len(sol_conn)):
            dofs = sol_conn[c]
            p_min = min(p_min, P[dofs].min())
            p_max = max(p_max, P[dofs].max())
            Xg = geo_coords[geo_conn[c]]
            vol, vint, pint = 0.0, np.zeros(dim), np.zeros(dim)
            for q in range(len(w)):
                J = dG[:, q, :] @ Xg  # J[xi][x] = dx / dxi
                jw = np.linalg.det(J) * w[q]
                vol += jw
                gp = np.linalg.solve(J, dB[:, q, :] @ P[dofs])
                vint += jw * (B[q] @ V[dofs])
                pint += jw * gp
            dom_vol += vol
            v_dom += vint
            vm, gm = vint / vol, pint / vol
            f_all.append(float(vm @ gm) * np.sqrt(vm @ vm))
            lc_all.append(vol ** (1.0 / dim))
    v_dom = v_dom / dom_vol
    nv = np.sqrt(v_dom @ v_dom)
    delta = (p_max - p_min) * nv * nv
    f = np.asarray(f_all)
    with np.errstate(divide="ignore", invalid="ignore"):
        q = f / delta
    sc = np.where(q < 0.0, 0.0, q)  # std::max(q, 0.0)
    t = sc * sc * np.asarray(lc_all)
    return np.where(t < 1.0, t, 1.0)  # std::min(1., t)
