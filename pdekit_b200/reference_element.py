"""Reference-element tables for the RDS kernels, computed on the host at set-up.

The reference builds the same tables through FEValues (src/interpolation/FEValues.cpp:157-190):
a modal Vandermonde matrix inverted with LAPACK gives the nodal Lagrange basis
(src/mesh/shape_function/ShapeFunction.cpp:22-70), evaluated at Gauss points
(src/mesh/point_set/QdPointSetTriagGauss.*, QdPointSetLineGauss.*). Here:

* equidistant Lagrange bases are evaluated in closed form, Silvester's product formula in
  barycentric coordinates for simplices (P. Silvester, "Higher-order polynomial triangular
  finite elements for potential problems", Int. J. Eng. Sci. 7, 1969) and 1D Lagrange
  products for the line; nodes are numbered as the reference's equidistant reference
  elements (vertices, edge nodes edge by edge, interior);
* triangle rules are Dunavant's symmetric rules (D.A. Dunavant, "High degree efficient
  symmetrical Gaussian quadrature rules for the triangle", IJNME 21, 1985), the same published
  rules the reference tabulates, expanded over their symmetry orbits and mapped to the
  reference triangle (-1,-1),(1,-1),(-1,1) (weights sum to 2);
* line rules are Gauss-Legendre with n = order // 2 + 1 points.

The tables agree with the reference's to rounding (tests/test_reference_element.py compares
them with the golden tables dumped from the reference).
"""

from __future__ import annotations

import numpy as np

from . import meshgen

# ---------------------------------------------------------------------------------------------
# Quadrature
# ---------------------------------------------------------------------------------------------

# Dunavant rules on the unit triangle: orbits (weight on area 1, barycentric parameters).
#   ("s3",  w)            centroid
#   ("s21", w, a)         (a, a, 1-2a) and its 3 permutations
#   ("s111", w, a, b)     (a, b, 1-a-b) and its 6 permutations
_SQ15 = np.sqrt(15.0)
_DUNAVANT = {
    1: [("s3", 1.0)],
    2: [("s21", 1.0 / 3.0, 1.0 / 6.0)],
    4: [("s21", 0.223381589678011, 0.445948490915965),
        ("s21", 0.109951743655322, 0.091576213509771)],
    5: [("s3", 0.225),
        ("s21", (155.0 + _SQ15) / 1200.0, (6.0 + _SQ15) / 21.0),
        ("s21", (155.0 - _SQ15) / 1200.0, (6.0 - _SQ15) / 21.0)],
    8: [("s3", 0.144315607677787),
        ("s21", 0.095091634267285, 0.459292588292723),
        ("s21", 0.103217370534718, 0.170569307751760),
        ("s21", 0.032458497623198, 0.050547228317031),
        ("s111", 0.027230314174435, 0.263112829634638, 0.008394777409958)],
}


def triag_gauss(order: int):
    """Points [n,2] on the reference triangle (-1,-1),(1,-1),(-1,1) and weights [n] (sum 2)."""
    if order not in _DUNAVANT:
        raise ValueError(f"no triangle rule of order {order} (have {sorted(_DUNAVANT)})")
    bary, w = [], []
    for orb in _DUNAVANT[order]:
        if orb[0] == "s3":
            bary.append((1 / 3, 1 / 3, 1 / 3))
            w.append(orb[1])
        elif orb[0] == "s21":
            _, wt, a = orb
            b = 1.0 - 2.0 * a
            for t in ((a, a, b), (a, b, a), (b, a, a)):
                bary.append(t)
                w.append(wt)
        else:
            _, wt, a, b = orb
            c = 1.0 - a - b
            for t in ((a, b, c), (b, c, a), (c, a, b), (a, c, b), (b, a, c), (c, b, a)):
                bary.append(t)
                w.append(wt)
    bary = np.asarray(bary)
    # barycentric (l0, l1, l2) of vertices (-1,-1), (1,-1), (-1,1)
    xi = -1.0 + 2.0 * bary[:, 1]
    eta = -1.0 + 2.0 * bary[:, 2]
    return np.stack([xi, eta], axis=1), 2.0 * np.asarray(w)


def line_gauss(order: int):
    """Gauss-Legendre points [n,1] and weights on [-1,1], n = order // 2 + 1."""
    n = order // 2 + 1
    x, w = np.polynomial.legendre.leggauss(n)
    return x.reshape(-1, 1), w


# ---------------------------------------------------------------------------------------------
# Lagrange bases on equidistant nodes
# ---------------------------------------------------------------------------------------------


def _silvester(i: int, p: int, lam: np.ndarray):
    """R_i(lam) = prod_{m<i} (p lam - m)/(m+1) and its derivative in lam."""
    r = np.ones_like(lam)
    dr = np.zeros_like(lam)
    for m in range(i):
        f = (p * lam - m) / (m + 1)
        df = p / (m + 1)
        dr = dr * f + r * df
        r = r * f
    return r, dr


def line_nodes(p: int) -> np.ndarray:
    """Equidistant line nodes in the reference's order: -1, 1, then interior nodes."""
    inner = [-1.0 + 2.0 * i / p for i in range(1, p)]
    return np.asarray([-1.0, 1.0] + inner).reshape(-1, 1)


def lagrange_line(p: int, pts: np.ndarray):
    """V [npts, p+1] and dV [1, npts, p+1] of the equidistant line basis."""
    x = np.asarray(pts, dtype=np.float64).reshape(-1)
    nodes = line_nodes(p).reshape(-1)
    n = nodes.size
    V = np.ones((x.size, n))
    dV = np.zeros((x.size, n))
    for j in range(n):
        others = [nodes[k] for k in range(n) if k != j]
        for k, xk in enumerate(others):
            den = nodes[j] - xk
            # product rule on prod_k (x - x_k)/(x_j - x_k)
            dV[:, j] = dV[:, j] * (x - xk) / den + V[:, j] / den
            V[:, j] = V[:, j] * (x - xk) / den
    return V, dV[None]


def lagrange_triag(p: int, pts: np.ndarray):
    """V [npts, ndof] and dV [2, npts, ndof] of the equidistant triangle basis of order p."""
    pts = np.asarray(pts, dtype=np.float64)
    nodes = meshgen.equidist_triag_nodes(p)
    l1 = (pts[:, 0] + 1.0) * 0.5
    l2 = (pts[:, 1] + 1.0) * 0.5
    l0 = 1.0 - l1 - l2
    ndof = nodes.shape[0]
    V = np.empty((pts.shape[0], ndof))
    dV = np.empty((2, pts.shape[0], ndof))
    for j, (a, b) in enumerate(nodes):
        i1 = int(round((a + 1.0) * 0.5 * p))
        i2 = int(round((b + 1.0) * 0.5 * p))
        i0 = p - i1 - i2
        r0, d0 = _silvester(i0, p, l0)
        r1, d1 = _silvester(i1, p, l1)
        r2, d2 = _silvester(i2, p, l2)
        V[:, j] = r0 * r1 * r2
        # d/dxi: dl1/dxi = 1/2, dl0/dxi = -1/2 ; d/deta: dl2/deta = 1/2, dl0/deta = -1/2
        dV[0, :, j] = 0.5 * (r0 * d1 * r2 - d0 * r1 * r2)
        dV[1, :, j] = 0.5 * (r0 * r1 * d2 - d0 * r1 * r2)
    return V, dV


def triag_tables(p: int, quad_order: int, geo_order: int = 1) -> dict:
    """Everything the triangle cell and edge-facet kernels need for solution order p."""
    qp, w = triag_gauss(quad_order)
    V, dV = lagrange_triag(p, qp)
    _, dVgeo = lagrange_triag(geo_order, qp)
    _, dVf = lagrange_triag(p + 1, qp)
    Vsf, _ = lagrange_triag(p, meshgen.equidist_triag_nodes(p + 1))
    fqp, fw = line_gauss(quad_order + 1)  # facet rule: cell order + 1 (bc/RDMBCBase.hpp:261-263)
    fV, _ = lagrange_line(p, fqp)
    fVgeo, fdVgeo = lagrange_line(geo_order, fqp)
    return dict(qp=qp, w=w, V=V, dV=dV, dVgeo=dVgeo, dVf=dVf, Vsf=Vsf, fqp=fqp, fw=fw, fV=fV,
                fVgeo=fVgeo, fdVgeo=fdVgeo)
