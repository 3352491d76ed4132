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
* line rules are Gauss-Legendre with n = order // 2 + 1 points; the square's rules are the
  reference's (2 x 2 Gauss-Legendre up to order 3, Stroud's symmetric rules above).

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


# ---------------------------------------------------------------------------------------------
# Quadrilaterals and tetrahedra, more rules
# ---------------------------------------------------------------------------------------------

# Dunavant degree 6, 12 points (area-1 weights).
_DUNAVANT[6] = [("s21", 0.116786275726379, 0.249286745170910),
                ("s21", 0.050844906370207, 0.063089014491502),
                ("s111", 0.082851075618374, 0.053145049844817, 0.310352451033784)]
# Dunavant degree 3, 4 points (centroid weight negative), exact rational weights.
_DUNAVANT[3] = [("s3", -27.0 / 48.0), ("s21", 25.0 / 48.0, 0.2)]


def quad_nodes(p: int) -> np.ndarray:
    """Equidistant nodes of the reference square [-1,1]^2 in the reference's order: the four
    corners counter-clockwise from (-1,-1), the edge nodes of edges (v0 v1), (v1 v2), (v2 v3),
    (v3 v0), then the interior nodes as a square of order p-2 numbered the same way."""
    pts = []

    def layer(lo: float, q: int, h: float):
        hi = -lo
        if q == 0:
            pts.append((lo, lo) if lo == hi else (0.0, 0.0))
            return
        c = [(lo, lo), (hi, lo), (hi, hi), (lo, hi)]
        pts.extend(c)
        for k in range(4):
            a, b = c[k], c[(k + 1) % 4]
            for i in range(1, q):
                t = i / q
                pts.append((a[0] + t * (b[0] - a[0]), a[1] + t * (b[1] - a[1])))
        if q >= 2:
            layer(lo + h, q - 2, h)

    layer(-1.0, p, 2.0 / p)
    return np.asarray(pts, dtype=np.float64)


def lagrange_quad(p: int, pts: np.ndarray):
    """Tensor-product equidistant Lagrange basis on the square: V [npts, ndof], dV [2, npts, ndof]."""
    pts = np.asarray(pts, dtype=np.float64)
    nodes = quad_nodes(p)
    g = np.linspace(-1.0, 1.0, p + 1)

    def basis_1d(i, x):
        v = np.ones_like(x)
        dv = np.zeros_like(x)
        for k in range(p + 1):
            if k == i:
                continue
            den = g[i] - g[k]
            dv = dv * (x - g[k]) / den + v / den
            v = v * (x - g[k]) / den
        return v, dv

    V = np.empty((pts.shape[0], nodes.shape[0]))
    dV = np.empty((2, pts.shape[0], nodes.shape[0]))
    for j, (a, b) in enumerate(nodes):
        i1 = int(round((a + 1.0) / 2.0 * p))
        i2 = int(round((b + 1.0) / 2.0 * p))
        vx, dvx = basis_1d(i1, pts[:, 0])
        vy, dvy = basis_1d(i2, pts[:, 1])
        V[:, j] = vx * vy
        dV[0, :, j] = dvx * vy
        dV[1, :, j] = vx * dvy
    return V, dV


def quad_tensor_gauss(order: int):
    """Tensor Gauss-Legendre rule on [-1,1]^2 with n = order // 2 + 1 points per direction."""
    x, w = line_gauss(order)
    x = x.ravel()
    X, Y = np.meshgrid(x, x, indexing="ij")
    W = np.outer(w, w)
    return np.stack([X.ravel(), Y.ravel()], axis=1), W.ravel()


# The square's rules of orders 4 - 8 the reference uses (src/mesh/point_set/
# QdPointSetQuadGauss.cpp): fully symmetric rules of degree 5 (8 points), 7 (12 points) and
# 9 (20 points, two orbit points outside the square), A. H. Stroud, "Approximate calculation of
# multiple integrals" (1971), region C2. Each is computed here from its orbit structure as the
# solution of the moment equations int x^2i y^2j (2(i + j) < degree) by Newton's method from
# the rough start given; orbits (weight, coordinates):
#   "a0" (a)      (a, 0), (-a, 0), (0, a), (0, -a)
#   "aa" (a)      (a, a), (a, -a), (-a, a), (-a, -a)
#   "ab" (a, b)   (a, b), (a, -b), (-a, b), (-a, -b), (b, a), (b, -a), (-b, a), (-b, -a)
_SQUARE_RULES = {
    5: [("a0", 0.8, (0.7,)), ("aa", 0.2, (0.9,))],
    7: [("a0", 0.24, (0.93,)), ("aa", 0.24, (0.8,)), ("aa", 0.52, (0.38,))],
    9: [("a0", 0.02, (1.1,)), ("a0", 0.39, (0.45,)), ("aa", 0.08, (0.9,)),
        ("ab", 0.25, (0.82, 0.41))],
}
_SQUARE_CACHE = {}


def _square_orbit(kind, c):
    z = 0.0 * c[0]
    if kind == "a0":
        a = c[0]
        return [(a, z), (-a, z), (z, a), (z, -a)]
    if kind == "aa":
        a = c[0]
        return [(a, a), (a, -a), (-a, a), (-a, -a)]
    a, b = c
    return [(a, b), (a, -b), (-a, b), (-a, -b), (b, a), (b, -a), (-b, a), (-b, -a)]


def _square_symmetric(deg: int):
    if deg in _SQUARE_CACHE:
        return _SQUARE_CACHE[deg]
    orbits = _SQUARE_RULES[deg]
    sizes = [len(o[2]) for o in orbits]
    x = np.array([v for o in orbits for v in (o[1],) + tuple(o[2])], dtype=float)
    mons = [(i, s - i) for s in range((deg - 1) // 2 + 1) for i in range(s, -1, -1) if 2 * i >= s]
    exact = np.array([4.0 / ((2 * i + 1) * (2 * j + 1)) for i, j in mons])

    def rule(x):
        pts, w, k = [], [], 0
        for (kind, _, _), n in zip(orbits, sizes):
            for pt in _square_orbit(kind, x[k + 1:k + 1 + n]):
                pts.append(pt)
                w.append(x[k])
            k += 1 + n
        return pts, w

    def moments(x):
        pts, w = rule(x)
        return sum(wt * np.array([px ** (2 * i) * py ** (2 * j) for i, j in mons])
                   for (px, py), wt in zip(pts, w)) - exact

    for _ in range(50):
        f = moments(x)
        if np.abs(f).max() < 4e-15:
            break
        # complex-step derivatives: the moments are polynomials in the unknowns
        h = 1e-30
        J = np.stack([moments(x + 1j * h * e).imag / h for e in np.eye(len(x))], 1)
        x = x - np.linalg.solve(J, f)
    else:
        raise RuntimeError(f"square rule of degree {deg} did not converge")
    pts, w = rule(x)
    out = (np.asarray(pts, dtype=float), np.asarray(w, dtype=float))
    _SQUARE_CACHE[deg] = out
    return out


def quad_gauss(order: int):
    """The reference's rule of the square [-1,1]^2 for `order` (QdPointSetQuadGauss.cpp): the
    centre (order 1), 2 x 2 Gauss-Legendre (orders 2, 3), then the symmetric rules of degree 5
    (orders 4, 5), 7 (orders 6, 7) and 9 (order 8). Weights sum to 4."""
    if order <= 1:
        return np.zeros((1, 2)), np.array([4.0])
    if order <= 3:
        return quad_tensor_gauss(2)
    if order <= 8:
        return _square_symmetric(order + 1 if order % 2 == 0 else order)
    raise ValueError(f"no quadrilateral rule of order {order} (the reference's go up to 8)")


_TET_V = np.array([[-1.0, -1.0, -1.0], [1.0, -1.0, -1.0], [-1.0, 1.0, -1.0], [-1.0, -1.0, 1.0]])
_TET_EDGES = [(0, 1), (1, 2), (2, 0), (3, 0), (3, 2), (3, 1)]
_TET_FACES = [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]


def tet_nodes(p: int) -> np.ndarray:
    """Equidistant nodes of the reference tetrahedron (-1,-1,-1),(1,-1,-1),(-1,1,-1),(-1,-1,1)
    in the reference's order: vertices, edges (v0 v1), (v1 v2), (v2 v0), (v3 v0), (v3 v2),
    (v3 v1), then one centroid node per face (p = 3). Orders up to 3."""
    if p > 3:
        raise ValueError("tetrahedra up to order 3")
    pts = [tuple(v) for v in _TET_V]
    for a, b in _TET_EDGES:
        for i in range(1, p):
            t = i / p
            pts.append(tuple(_TET_V[a] + t * (_TET_V[b] - _TET_V[a])))
    if p == 3:
        for f in _TET_FACES:
            pts.append(tuple(_TET_V[list(f)].mean(axis=0)))
    return np.asarray(pts, dtype=np.float64)


def lagrange_tet(p: int, pts: np.ndarray):
    """Equidistant tetrahedron basis (Silvester's formula in 4 barycentrics):
    V [npts, ndof], dV [3, npts, ndof]."""
    pts = np.asarray(pts, dtype=np.float64)
    nodes = tet_nodes(p)
    lam = [None, (pts[:, 0] + 1) * 0.5, (pts[:, 1] + 1) * 0.5, (pts[:, 2] + 1) * 0.5]
    lam[0] = 1.0 - lam[1] - lam[2] - lam[3]
    V = np.empty((pts.shape[0], nodes.shape[0]))
    dV = np.empty((3, pts.shape[0], nodes.shape[0]))
    for j, node in enumerate(nodes):
        idx = [int(round((node[k] + 1.0) * 0.5 * p)) for k in range(3)]
        idx = [p - sum(idx)] + idx
        r, dr = zip(*[_silvester(idx[k], p, lam[k]) for k in range(4)])
        V[:, j] = r[0] * r[1] * r[2] * r[3]
        for d in range(3):
            # d lam_{d+1} / d xi_d = 1/2, d lam_0 / d xi_d = -1/2
            prod_d = [r[k] for k in range(4)]
            prod_d[d + 1] = dr[d + 1]
            prod_0 = [r[k] for k in range(4)]
            prod_0[0] = dr[0]
            dV[d, :, j] = 0.5 * (np.prod(prod_d, axis=0) - np.prod(prod_0, axis=0))
    return V, dV


# Symmetric tetrahedron rules on the unit tetrahedron (volume-1/6 weights):
#   ("s4", w) centroid; ("s31", w, a): (a,a,a,1-3a) x 4; ("s22", w, a): (a,a,1/2-a,1/2-a) x 6.
_TET_RULES = {
    1: [("s4", 1.0 / 6.0)],
    2: [("s31", 1.0 / 24.0, (5.0 - np.sqrt(5.0)) / 20.0)],
    # 11-point degree-4 rule (P. Keast, "Moderate-degree tetrahedral quadrature formulas",
    # CMAME 55, 1986; negative centroid weight), in closed form
    4: [("s4", -74.0 / 5625.0), ("s31", 343.0 / 45000.0, 1.0 / 14.0),
        ("s22", 56.0 / 2250.0, (1.0 + np.sqrt(5.0 / 14.0)) / 4.0)],
    # 14-point degree-5 rule (Walkington; the rule pdekit tabulates for order 5)
    5: [("s31", 0.01224884051939366, 0.0927352503108912),
        ("s31", 0.01878132095300264, 0.3108859192633006),
        ("s22", 0.007091003462846911, 0.4544962958743504)],
}


def tet_gauss(order: int):
    """Points [n,3] on the reference tetrahedron and weights [n] (sum 4/3)."""
    if order not in _TET_RULES:
        raise ValueError(f"no tetrahedron rule of order {order}")
    bary, w = [], []
    for orb in _TET_RULES[order]:
        if orb[0] == "s4":
            bary.append((0.25, 0.25, 0.25, 0.25))
            w.append(orb[1])
        elif orb[0] == "s31":
            _, wt, a = orb
            b = 1.0 - 3.0 * a
            for k in range(4):
                t = [a] * 4
                t[k] = b
                bary.append(tuple(t))
                w.append(wt)
        else:
            _, wt, a = orb
            b = 0.5 - a
            for i in range(4):
                for j in range(i + 1, 4):
                    t = [b] * 4
                    t[i] = a
                    t[j] = a
                    bary.append(tuple(t))
                    w.append(wt)
    bary = np.asarray(bary)
    pts = -1.0 + 2.0 * bary[:, 1:4]
    return pts, 8.0 * np.asarray(w)


def quad_tables(p: int, quad_order: int, vol_order: int = None, tensor: bool = False) -> dict:
    """Tables for P p quadrilaterals with bilinear (P1) geometry: the cell rule of quad_order is
    the reference's (quad_gauss), or with tensor=True the tensor Gauss-Legendre rule with
    quad_order // 2 + 1 points per direction."""
    qp, w = (quad_tensor_gauss if tensor else quad_gauss)(quad_order)
    V, dV = lagrange_quad(p, qp)
    _, dVgeo = lagrange_quad(1, qp)
    _, dVf = lagrange_quad(p + 1, qp)
    Vsf, _ = lagrange_quad(p, quad_nodes(p + 1))
    vqp, wv = quad_gauss(p if vol_order is None else vol_order)
    _, dVgeo_v = lagrange_quad(1, vqp)
    fqp, fw = line_gauss(quad_order + 1)
    fV, _ = lagrange_line(p, fqp)
    fVgeo, fdVgeo = lagrange_line(1, fqp)
    return dict(qp=qp, w=w, V=V, dV=dV, dVgeo=dVgeo, dVf=dVf, Vsf=Vsf, wv=wv, dVgeo_v=dVgeo_v,
                fqp=fqp, fw=fw, fV=fV, fVgeo=fVgeo, fdVgeo=fdVgeo)


def tet_tables(p: int, quad_order: int) -> dict:
    """Tables for P p tetrahedra with affine geometry; boundary faces are P p triangles with the
    triangle rule of order quad_order + 1."""
    qp, w = tet_gauss(quad_order)
    V, dV = lagrange_tet(p, qp)
    _, dVgeo = lagrange_tet(1, qp)
    _, dVf = lagrange_tet(p + 1, qp)
    Vsf, _ = lagrange_tet(p, tet_nodes(p + 1))
    vqp, wv = tet_gauss(2 if p >= 2 else 1)
    _, dVgeo_v = lagrange_tet(1, vqp)
    fqp, fw = triag_gauss(quad_order + 1)
    fV, _ = lagrange_triag(p, fqp)
    fVgeo, fdVgeo = lagrange_triag(1, fqp)
    return dict(qp=qp, w=w, V=V, dV=dV, dVgeo=dVgeo, dVf=dVf, Vsf=Vsf, wv=wv, dVgeo_v=dVgeo_v,
                fqp=fqp, fw=fw, fV=fV, fVgeo=fVgeo, fdVgeo=fdVgeo)


# ---------------------------------------------------------------------------------------------
# Stabilisation operators
# ---------------------------------------------------------------------------------------------

_STAB_CACHE = {}


def stab_tables(shape: str, p: int, ngeo: int) -> dict:
    """Tables of the stabilisation operators for cells of `shape` and order p.

    * P1 [ndof, nvert]: the vertex interpolant (P1 on simplices, Q1 on quadrilaterals) at the
      cell's nodes, for the cell-to-node transfer
      (src/interpolation/mesh_function/MeshFunctionTools.hpp:328-397);
    * on affine simplices, the smoothness sensor (src/solver/art_visc/ArtificialViscosity.hpp:
      174-300, 388-455): w [nq] and points of a rule exact to degree 2p, Vn [nq, ndof] the nodal
      basis there and R [nq, ndof] the map from nodal values to u - u_{p-1} at the points.
      The reference projects u on its modal basis and switches off the modes of degree p; its
      simplex bases (Dubiner) are orthogonal, so u_{p-1} is the L2 projection of u onto the
      polynomials of degree p - 1, built here with the nodal basis of order p - 1:
      R = Vn - Vl (Vl^T W Vl)^-1 Vl^T W Vn. At p = 1 the reference switches off every mode
      (mesh/shape_function/DubinerExpansionTriag.cpp:460-467), u_{p-1} = 0 and R = Vn.
      On affine cells detJ is constant, so any rule exact to degree 2p gives the reference's
      integrals. Bilinear quadrilaterals (ngeo = 4): the tables of _quad_sensor, with
      dVgeo [2, nq, 4] for detJ at every point. nq = 0 elsewhere (no sensor).
    """
    key = (shape, p, ngeo)
    if key in _STAB_CACHE:
        return _STAB_CACHE[key]
    empty = np.zeros(1)
    if shape == "triag":
        P1, _ = lagrange_triag(1, meshgen.equidist_triag_nodes(p))
        rule = (lambda o: triag_gauss(o)) if 2 * p in _DUNAVANT and ngeo == 3 else None
        basis = lagrange_triag
        order = 2 * p
    elif shape == "tetra":
        P1, _ = lagrange_tet(1, tet_nodes(p))
        order = min([o for o in _TET_RULES if o >= 2 * p], default=None)
        rule = tet_gauss if order is not None and ngeo == 4 else None
        basis = lagrange_tet
    elif shape == "quad":
        P1, _ = lagrange_quad(1, quad_nodes(p))
        rule = None
        if ngeo == 4:
            out = dict(P1=np.ascontiguousarray(P1), **_quad_sensor(p))
            _STAB_CACHE[key] = out
            return out
    else:
        raise ValueError(f"no stabilisation tables for {shape}")
    out = dict(nq=0, w=empty, Vn=empty, R=empty, P1=np.ascontiguousarray(P1))
    if rule is not None:
        qp, w = rule(order)
        Vn, _ = basis(p, qp)
        if p == 1:
            R = Vn.copy()
        else:
            Vl, _ = basis(p - 1, qp)
            G = Vl.T @ (w[:, None] * Vl)
            R = Vn - Vl @ np.linalg.solve(G, Vl.T @ (w[:, None] * Vn))
        out.update(nq=len(w), w=np.ascontiguousarray(w), Vn=np.ascontiguousarray(Vn),
                   R=np.ascontiguousarray(R))
    _STAB_CACHE[key] = out
    return out


def _legendre_square(p: int, pts: np.ndarray):
    """The reference's modal basis of the square (src/mesh/shape_function/
    ModalExpansionQuad.cpp:60-73): mode (m, n), m-major, P_m(xi) P_n(eta) sqrt((2m+1)(2n+1)) / 2;
    and the modes its leading-term flags select (ModalExpansionQuad.cpp:240-257): the flag index
    advances only on modes with m == p or n == p, so the FIRST 2p + 1 modes are flagged."""
    from numpy.polynomial import legendre as L
    E = np.eye(p + 1)
    cols = [L.legval(pts[:, 0], E[m]) * L.legval(pts[:, 1], E[n]) *
            np.sqrt((2 * m + 1) * (2 * n + 1)) / 2.0 for m in range(p + 1) for n in range(p + 1)]
    flags = np.zeros((p + 1) ** 2, dtype=bool)
    flags[:2 * p + 1] = True
    return np.stack(cols, 1), flags


def _quad_sensor(p: int) -> dict:
    """The sensor on bilinear quadrilaterals (ArtificialViscosity.hpp:388-455): the reference's
    rule of order 2p (quad_gauss), Vn the nodal basis there, R = Vm[:, F] T^-1[F, :] the flagged
    modes' part of u (T the modal basis at the nodes, F the flags), and dVgeo [2, nq, 4] for detJ
    at every point. The reference projects u in L2 on its modal basis with the cell's mass matrix;
    when that matrix is regular the projection of the interpolant is the interpolant, whose modal
    coefficients are T^-1 u, independent of the cell's shape. At p = 1 the rule has 4 points for
    4 modes. At p >= 2 it has fewer points than modes (8 for 9, 12 for 16), the reference's mass
    matrix is singular and its coefficients follow the rounding of the inversion; T^-1 u is the
    value every regular projection gives."""
    qp, w = quad_gauss(2 * p)
    Vn, _ = lagrange_quad(p, qp)
    Vm, flags = _legendre_square(p, qp)
    T, _ = _legendre_square(p, quad_nodes(p))
    R = Vm[:, flags] @ np.linalg.inv(T)[flags, :]
    _, dVgeo = lagrange_quad(1, qp)
    return dict(nq=len(w), w=np.ascontiguousarray(w), Vn=np.ascontiguousarray(Vn),
                R=np.ascontiguousarray(R), dVgeo=np.ascontiguousarray(dVgeo))


def bonanni_tables(shape: str, p: int, ngeo: int) -> dict:
    """Tables of Bonanni's pressure-based blending coefficient
    (src/solver/rdm/blending_coeff/BonanniBlendingCoeffImpl.hpp:102-168): the reference
    integrates the velocity and the pressure gradient over a cell with its Gauss rule of order
    max(p, geometry order). Quadrilaterals use that rule (quad_gauss: at the orders <= 3 of
    p <= 3 tensor Gauss-Legendre, order // 2 + 1 points per direction); on affine simplices the integrands are polynomials of degree <= p,
    so a rule exact to degree p gives the same integrals. w [nq], V [nq, ndof],
    dV [D, nq, ndof], dVgeo [D, nq, ngeo]; nq = 0 where not provided (curved cells)."""
    order = max(p, 1)
    if shape == "triag" and ngeo == 3:
        qp, w = triag_gauss(min(o for o in _DUNAVANT if o >= order))
        V, dV = lagrange_triag(p, qp)
        _, dVgeo = lagrange_triag(1, qp)
    elif shape == "quad" and ngeo == 4:
        qp, w = quad_gauss(order)
        V, dV = lagrange_quad(p, qp)
        _, dVgeo = lagrange_quad(1, qp)
    elif shape == "tetra" and ngeo == 4:
        qp, w = tet_gauss(min(o for o in _TET_RULES if o >= order))
        V, dV = lagrange_tet(p, qp)
        _, dVgeo = lagrange_tet(1, qp)
    else:
        z = np.zeros(1)
        return dict(nq=0, w=z, V=z, dV=z, dVgeo=z)
    c = np.ascontiguousarray
    return dict(nq=len(w), w=c(w), V=c(V), dV=c(dV), dVgeo=c(dVgeo))
