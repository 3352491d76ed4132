"""Synthetic unstructured meshes for the RDS path, and their Gmsh 2.2 ASCII form.

The reference reads meshes with its Gmsh reader (src/mesh/io/gmsh/GmshReader.hpp:119) and
raises the solution order with DofMap::clone_continuous (src/mesh/containers/DofMap.hpp:254).
This module produces the same kind of input on the host:

* a P1 geometry (vertex coordinates, cell -> vertex connectivity, named boundary edges),
  seeded interior jitter as in the benchmark configurations;
* a continuous Pk solution numbering (cell -> dof connectivity) whose local dof order follows
  the reference's equidistant reference elements: vertices, then the nodes of edge 0 (v0->v1),
  edge 1 (v1->v2), edge 2 (v2->v0), then interior nodes
  (src/mesh/std_region/EquidistStdRegionTriag.cpp:239-320);
* a writer for Gmsh 2.2 files so the compiled reference can load the identical geometry.

Node numbering of the high-order dofs is our own; the residual does not depend on it.
"""

from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class Mesh2D:
    coords: np.ndarray  # [nverts, 2] float64
    cells: np.ndarray  # [ncells, 3] int32, counter-clockwise
    boundaries: dict  # name -> [nedges, 2] int32 (edge vertices, cell-local orientation)
    shape: str = "triag"


def unit_square_tri(n: int, jitter: float = 0.0, seed: int = 0, lx: float = 1.0,
                    ly: float = 1.0) -> Mesh2D:
    """n x n squares on [0,lx]x[0,ly], each split into two triangles along the (i,j)->(i+1,j+1)
    diagonal; interior vertices moved by U(-jitter*h, +jitter*h) in each direction."""
    nv1 = n + 1
    hx, hy = lx / n, ly / n
    jj, ii = np.meshgrid(np.arange(nv1), np.arange(nv1), indexing="ij")
    x = (ii * hx).astype(np.float64).ravel()
    y = (jj * hy).astype(np.float64).ravel()
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        dx = rng.uniform(-jitter * hx, jitter * hx, size=x.shape)
        dy = rng.uniform(-jitter * hy, jitter * hy, size=y.shape)
        interior = ((ii > 0) & (ii < n) & (jj > 0) & (jj < n)).ravel()
        x = x + np.where(interior, dx, 0.0)
        y = y + np.where(interior, dy, 0.0)
    coords = np.stack([x, y], axis=1)

    def vid(i, j):
        return j * nv1 + i

    cells = []
    for j in range(n):
        for i in range(n):
            a, b, c, d = vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)
            cells.append((a, b, c))
            cells.append((a, c, d))
    cells = np.asarray(cells, dtype=np.int32)

    bnd = {
        "bottom": np.asarray([(vid(i, 0), vid(i + 1, 0)) for i in range(n)], dtype=np.int32),
        "right": np.asarray([(vid(n, j), vid(n, j + 1)) for j in range(n)], dtype=np.int32),
        "top": np.asarray([(vid(i + 1, n), vid(i, n)) for i in range(n)], dtype=np.int32),
        "left": np.asarray([(vid(0, j + 1), vid(0, j)) for j in range(n)], dtype=np.int32),
    }
    return Mesh2D(coords=coords, cells=cells, boundaries=bnd)


def write_gmsh22(path: str, mesh: Mesh2D, domain_name: str = "domain") -> None:
    """Write the P1 geometry as a Gmsh 2.2 ASCII file with one physical group per boundary
    (dimension 1) and one for the cells (dimension 2)."""
    names = list(mesh.boundaries.keys())
    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$PhysicalNames",
             str(len(names) + 1)]
    for k, nm in enumerate(names):
        lines.append(f'1 {k + 1} "{nm}"')
    cell_tag = len(names) + 1
    lines.append(f'2 {cell_tag} "{domain_name}"')
    lines.append("$EndPhysicalNames")
    lines.append("$Nodes")
    lines.append(str(mesh.coords.shape[0]))
    for i, (x, y) in enumerate(mesh.coords):
        lines.append(f"{i + 1} {float(x)!r} {float(y)!r} 0")
    lines.append("$EndNodes")
    lines.append("$Elements")
    nel = sum(len(v) for v in mesh.boundaries.values()) + mesh.cells.shape[0]
    lines.append(str(nel))
    eid = 1
    for k, nm in enumerate(names):
        for a, b in mesh.boundaries[nm]:
            lines.append(f"{eid} 1 2 {k + 1} {k + 1} {a + 1} {b + 1}")
            eid += 1
    for a, b, c in mesh.cells:
        lines.append(f"{eid} 2 2 {cell_tag} {cell_tag} {a + 1} {b + 1} {c + 1}")
        eid += 1
    lines.append("$EndElements")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def tri_dof_layout(p: int) -> int:
    return (p + 1) * (p + 2) // 2


def clone_continuous_tri(mesh: Mesh2D, p: int):
    """Continuous Pk dof numbering on a P1 triangle mesh.

    Returns (sol_conn [ncells, ndof] int32, nsol, sol_coords [nsol, 2]) with vertices keeping
    their geometry ids, then edge dofs, then interior dofs. Local order per cell follows the
    reference's equidistant triangle (vertices, edges 0,1,2 in the v0->v1->v2->v0 sense,
    interior nodes recursively)."""
    nv = mesh.coords.shape[0]
    nc = mesh.cells.shape[0]
    if p == 1:
        return mesh.cells.copy(), nv, mesh.coords.copy()
    ne_int = p - 1
    ndof = tri_dof_layout(p)
    n_int = ndof - 3 - 3 * ne_int
    ref = equidist_triag_nodes(p)  # on (-1,-1),(1,-1),(-1,1)
    cells = mesh.cells.astype(np.int64)
    # directed cell edges v0->v1, v1->v2, v2->v0, cell-major
    a = cells[:, [0, 1, 2]].reshape(-1)
    b = cells[:, [1, 2, 0]].reshape(-1)
    key = np.minimum(a, b) * nv + np.maximum(a, b)
    _, first, inv = np.unique(key, return_index=True, return_inverse=True)
    first_slot = first[inv]  # slot of the edge's first appearance
    is_new = first_slot == np.arange(key.shape[0])
    # ids are handed out while walking the cells in order: new edges of the cell (local edge
    # order), then its interior dofs
    sizes = np.zeros((nc, 4), dtype=np.int64)
    sizes[:, :3] = is_new.reshape(nc, 3) * ne_int
    sizes[:, 3] = n_int
    start = nv + np.concatenate([[0], np.cumsum(sizes.reshape(-1))[:-1]]).reshape(nc, 4)
    conn = np.empty((nc, ndof), dtype=np.int64)
    conn[:, :3] = cells
    slot_start = start[:, :3].reshape(-1)[first_slot]  # [3 nc] first id of each edge's block
    steps = np.arange(ne_int)
    ids = slot_start[:, None] + steps[None, :]
    rev = a > b
    ids[rev] = ids[rev][:, ::-1]
    conn[:, 3:3 + 3 * ne_int] = ids.reshape(nc, 3 * ne_int)
    if n_int > 0:
        conn[:, 3 + 3 * ne_int:] = start[:, 3:4] + np.arange(n_int)[None, :]
    next_id = int(nv + sizes.sum())
    conn = conn.astype(np.int32)
    nsol = next_id
    # physical coordinates of every dof (P1 map)
    xi = (ref[:, 0] + 1.0) * 0.5
    eta = (ref[:, 1] + 1.0) * 0.5
    lam = np.stack([1.0 - xi - eta, xi, eta], axis=1)  # [ndof, 3]
    X = mesh.coords[mesh.cells]  # [nc, 3, 2]
    dof_xy = np.einsum("nk,ckd->cnd", lam, X)
    sol_coords = np.zeros((nsol, 2))
    sol_coords[conn.ravel()] = dof_xy.reshape(-1, 2)
    return conn, nsol, sol_coords


def equidist_triag_nodes(p: int) -> np.ndarray:
    """Equidistant reference-triangle nodes in the reference's order
    (src/mesh/std_region/EquidistStdRegionTriag.cpp:239-320): vertices (-1,-1),(1,-1),(-1,1);
    edge nodes of edges 0,1,2; then the same pattern recursively on the interior triangle."""
    pts = []

    def layer(offset: int, q: int):
        # sub-triangle whose vertices sit 'offset' steps inside, of polynomial order q
        d = 2.0 / p
        v0 = (-1.0 + offset * d, -1.0 + offset * d)
        v1 = (1.0 - 2 * offset * d, -1.0 + offset * d)
        v2 = (-1.0 + offset * d, 1.0 - 2 * offset * d)
        if q == 0:
            pts.append(v0)
            return
        pts.extend([v0, v1, v2])
        for i in range(1, q):
            pts.append((v0[0] + i * d, v0[1]))
        for i in range(1, q):
            pts.append((v1[0] - i * d, v1[1] + i * d))
        for i in range(1, q):
            pts.append((v2[0], v2[1] - i * d))
        if q >= 3:
            layer(offset + 1, q - 3)

    layer(0, p)
    return np.asarray(pts, dtype=np.float64)


def boundary_facets_tri(mesh: Mesh2D, sol_conn: np.ndarray, p: int, name: str):
    """Facet (edge) connectivity of a named boundary: geometry vertices [nf, 2] and solution
    dofs [nf, p+1] in the line element's order (two end vertices, then interior edge nodes
    from the first vertex to the second), oriented like the parent cell's edge."""
    edges = np.asarray(mesh.boundaries[name], dtype=np.int64).reshape(-1, 2)
    nv = mesh.coords.shape[0]
    cells = mesh.cells.astype(np.int64)
    a = cells[:, [0, 1, 2]].reshape(-1)
    b = cells[:, [1, 2, 0]].reshape(-1)
    key = np.minimum(a, b) * nv + np.maximum(a, b)
    order = np.argsort(key, kind="stable")
    bkey = np.minimum(edges[:, 0], edges[:, 1]) * nv + np.maximum(edges[:, 0], edges[:, 1])
    pos = np.searchsorted(key[order], bkey)
    if np.any(pos >= key.shape[0]) or np.any(key[order][np.minimum(pos, key.shape[0] - 1)] != bkey):
        raise ValueError(f"boundary {name}: an edge belongs to no cell")
    # a boundary edge has one cell; with several matches the last one in cell order wins
    last = np.searchsorted(key[order], bkey, side="right") - 1
    slot = order[last]
    c, le = slot // 3, slot % 3
    geo = np.stack([a[slot], b[slot]], axis=1).astype(np.int32)
    sol = np.empty((edges.shape[0], p + 1), dtype=np.int32)
    sol[:, :2] = geo
    if p > 1:
        start = 3 + le * (p - 1)
        sol[:, 2:] = sol_conn[c[:, None], start[:, None] + np.arange(p - 1)[None, :]]
    return geo, sol


# ---------------------------------------------------------------------------------------------
# General meshes (triangles, quadrilaterals, tetrahedra) for the Euler configurations
# ---------------------------------------------------------------------------------------------

GMSH_TYPE = {"line": 1, "triag": 2, "quad": 3, "tetra": 4}
GMSH_FACET = {"triag": "line", "quad": "line", "tetra": "triag"}


@dataclasses.dataclass
class Mesh:
    """P1 geometry: coords [nv, dim]; cell groups {shape: [nc, nvert]} (reference vertex
    order, positive orientation); named boundaries {name: (facet shape, [nf, nvert])}."""
    coords: np.ndarray
    cells: dict
    boundaries: dict

    @property
    def dim(self):
        return self.coords.shape[1]


def bump_profile(x, h=0.1, k=25.0):
    return h * np.exp(-k * x * x)


def channel_2d(nx_tri: int, nx_quad: int, ny: int, x0=-1.5, xm=0.0, x1=1.5, bump_h=0.1,
               jitter=0.0, seed=0) -> Mesh:
    """Bump channel [x0,x1] x [0,1] with bottom wall y = bump_h exp(-25 x^2): triangles on
    [x0,xm] (nx_tri columns of squares split along the (i,j)->(i+1,j+1) diagonal) and
    quadrilaterals on [xm,x1] (nx_quad columns); ny rows; the two halves share the vertical
    line x = xm. y is mapped as y' = yb(x) + y (1 - yb(x)). Interior vertices jittered by
    U(+-jitter h). Boundaries: bottom_wall, top_wall, inlet (x = x0), outlet (x = x1)."""
    xs = np.concatenate([np.linspace(x0, xm, nx_tri + 1) if nx_tri > 0 else np.array([x0]),
                         np.linspace(xm, x1, nx_quad + 1)[1:] if nx_quad > 0 else np.array([])])
    if nx_tri == 0:
        xs = np.linspace(xm, x1, nx_quad + 1) if x0 == xm else np.linspace(x0, x1, nx_quad + 1)
    nxv = xs.size
    ys = np.linspace(0.0, 1.0, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="xy")  # [ny+1, nxv]
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        hx = np.diff(xs).min()
        hy = 1.0 / ny
        interior = np.zeros_like(X, dtype=bool)
        interior[1:-1, 1:-1] = True
        X = X + np.where(interior, rng.uniform(-jitter * hx, jitter * hx, X.shape), 0.0)
        Y = Y + np.where(interior, rng.uniform(-jitter * hy, jitter * hy, Y.shape), 0.0)
    yb = bump_profile(X, bump_h)
    Y = yb + Y * (1.0 - yb)
    coords = np.stack([X.ravel(), Y.ravel()], axis=1)

    def vid(i, j):
        return j * nxv + i

    tris, quads = [], []
    ntri_cols = nx_tri if nx_tri > 0 else 0
    for j in range(ny):
        for i in range(nxv - 1):
            a, b, c, d = vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)
            if i < ntri_cols:
                tris.append((a, b, c))
                tris.append((a, c, d))
            else:
                quads.append((a, b, c, d))
    cells = {}
    if tris:
        cells["triag"] = np.asarray(tris, dtype=np.int32)
    if quads:
        cells["quad"] = np.asarray(quads, dtype=np.int32)
    bnd = {
        "bottom_wall": ("line", np.asarray([(vid(i, 0), vid(i + 1, 0)) for i in range(nxv - 1)],
                                           dtype=np.int32)),
        "outlet": ("line", np.asarray([(vid(nxv - 1, j), vid(nxv - 1, j + 1)) for j in range(ny)],
                                      dtype=np.int32)),
        "top_wall": ("line", np.asarray([(vid(i + 1, ny), vid(i, ny)) for i in range(nxv - 1)],
                                        dtype=np.int32)),
        "inlet": ("line", np.asarray([(vid(0, j + 1), vid(0, j)) for j in range(ny)],
                                     dtype=np.int32)),
    }
    return Mesh(coords=coords, cells=cells, boundaries=bnd)


# Kuhn split of the unit cube into 6 tetrahedra along the (0,0,0)-(1,1,1) diagonal; hex vertex
# k = i + 2 j + 4 l at (i, j, l). Every tetrahedron is (v0, v0+e_a, v0+e_a+e_b, v7).
_KUHN = [(0, 1, 3, 7), (0, 1, 5, 7), (0, 2, 3, 7), (0, 2, 6, 7), (0, 4, 5, 7), (0, 4, 6, 7)]


def box_tet(nx: int, ny: int, nz: int, x0=-2.0, x1=2.0, bump_h=0.05, bump_k=16.0, jitter=0.0,
            seed=0) -> Mesh:
    """[x0,x1] x [0,1] x [0,1] hexahedra split into 6 tetrahedra each (Kuhn split, conforming),
    bottom y = bump_h exp(-bump_k (x^2 + z^2)), y' = yb + y (1 - yb). Boundaries: bottom_wall
    (y=0), top_wall (y=1), side_walls (z=0, z=1), inlet (x=x0), outlet (x=x1)."""
    xs = np.linspace(x0, x1, nx + 1)
    ys = np.linspace(0.0, 1.0, ny + 1)
    zs = np.linspace(0.0, 1.0, nz + 1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")  # [nz+1, ny+1, nx+1]
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        interior = np.zeros_like(X, dtype=bool)
        interior[1:-1, 1:-1, 1:-1] = True
        h = (np.diff(xs).min(), 1.0 / ny, 1.0 / nz)
        X = X + np.where(interior, rng.uniform(-jitter * h[0], jitter * h[0], X.shape), 0.0)
        Y = Y + np.where(interior, rng.uniform(-jitter * h[1], jitter * h[1], Y.shape), 0.0)
        Z = Z + np.where(interior, rng.uniform(-jitter * h[2], jitter * h[2], Z.shape), 0.0)
    yb = bump_h * np.exp(-bump_k * (X * X + Z * Z))
    Y = yb + Y * (1.0 - yb)
    coords = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    nxv, nyv = nx + 1, ny + 1

    def vid(i, j, l):
        return (l * nyv + j) * nxv + i

    tets = []
    for l in range(nz):
        for j in range(ny):
            for i in range(nx):
                hexv = [vid(i + (k & 1), j + ((k >> 1) & 1), l + ((k >> 2) & 1)) for k in range(8)]
                for t in _KUHN:
                    tets.append([hexv[k] for k in t])
    tets = np.asarray(tets, dtype=np.int32)
    # positive orientation
    P = coords[tets]
    vol6 = np.einsum("ij,ij->i", np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0]), P[:, 3] - P[:, 0])
    neg = vol6 < 0
    tets[neg] = tets[neg][:, [0, 2, 1, 3]]
    # boundary faces: faces of tets that lie on the box sides
    faces = {}
    for t in tets:
        for f in ((t[1], t[2], t[3]), (t[0], t[3], t[2]), (t[0], t[1], t[3]), (t[0], t[2], t[1])):
            key = tuple(sorted(f))
            faces[key] = None if key in faces else f
    bnd = {k: [] for k in ("bottom_wall", "top_wall", "side_walls", "inlet", "outlet")}
    Xr, Yr, Zr = (np.meshgrid(zs, ys, xs, indexing="ij")[2].ravel(),
                  np.meshgrid(zs, ys, xs, indexing="ij")[1].ravel(),
                  np.meshgrid(zs, ys, xs, indexing="ij")[0].ravel())
    for key, f in faces.items():
        if f is None:
            continue
        f = np.asarray(f)
        if np.all(Yr[f] == 0.0):
            bnd["bottom_wall"].append(f)
        elif np.all(Yr[f] == 1.0):
            bnd["top_wall"].append(f)
        elif np.all(Xr[f] == x0):
            bnd["inlet"].append(f)
        elif np.all(Xr[f] == x1):
            bnd["outlet"].append(f)
        else:
            bnd["side_walls"].append(f)
    boundaries = {k: ("triag", np.asarray(sorted(v, key=lambda a: tuple(sorted(a))),
                                          dtype=np.int32)) for k, v in bnd.items()}
    return Mesh(coords=coords, cells={"tetra": tets}, boundaries=boundaries)


def write_gmsh22_mesh(path: str, mesh: Mesh, domain_name: str = "domain") -> None:
    """Gmsh 2.2 ASCII of a general P1 Mesh (one physical group per boundary and one for the
    cells)."""
    names = list(mesh.boundaries.keys())
    tdim = mesh.dim
    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$PhysicalNames", str(len(names) + 1)]
    for k, nm in enumerate(names):
        lines.append(f'{tdim - 1} {k + 1} "{nm}"')
    cell_tag = len(names) + 1
    lines.append(f'{tdim} {cell_tag} "{domain_name}"')
    lines += ["$EndPhysicalNames", "$Nodes", str(mesh.coords.shape[0])]
    for i, xyz in enumerate(mesh.coords):
        c = [float(v) for v in xyz] + [0.0] * (3 - len(xyz))
        lines.append(f"{i + 1} {c[0]!r} {c[1]!r} {c[2]!r}")
    lines.append("$EndNodes")
    nel = sum(len(v[1]) for v in mesh.boundaries.values()) + sum(len(c) for c in mesh.cells.values())
    lines += ["$Elements", str(nel)]
    eid = 1
    for k, nm in enumerate(names):
        shape, facets = mesh.boundaries[nm]
        for f in facets:
            lines.append(f"{eid} {GMSH_TYPE[shape]} 2 {k + 1} {k + 1} " +
                         " ".join(str(v + 1) for v in f))
            eid += 1
    for shape, cells in mesh.cells.items():
        for c in cells:
            lines.append(f"{eid} {GMSH_TYPE[shape]} 2 {cell_tag} {cell_tag} " +
                         " ".join(str(v + 1) for v in c))
            eid += 1
    lines.append("$EndElements")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


# ---------------------------------------------------------------------------------------------
# Continuous P_p numbering of a general mesh (vectorised)
# ---------------------------------------------------------------------------------------------

CELL_EDGES = {"triag": [(0, 1), (1, 2), (2, 0)],
              "quad": [(0, 1), (1, 2), (2, 3), (3, 0)],
              "tetra": [(0, 1), (1, 2), (2, 0), (3, 0), (3, 2), (3, 1)]}
TET_FACES = [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]


def _ref_nodes(shape, p):
    from . import reference_element as R
    return {"triag": lambda: equidist_triag_nodes(p), "quad": lambda: R.quad_nodes(p),
            "tetra": lambda: R.tet_nodes(p)}[shape]()


def _p1_map(shape, ref):
    """Weights [nref, nvert] of the P1 geometry map at reference points."""
    if shape == "quad":
        from . import reference_element as R
        V, _ = R.lagrange_quad(1, ref)
        return V
    lam = (ref + 1.0) * 0.5
    return np.concatenate([1.0 - lam.sum(axis=1, keepdims=True), lam], axis=1)


@dataclasses.dataclass
class Clone:
    p: int
    conn: dict  # shape -> [nc, ndof] int32
    nsol: int
    coords: np.ndarray  # [nsol, dim]
    edge_index: dict  # (min, max) vertex pair -> edge id (only via lookup arrays below)
    edge_keys: np.ndarray  # [nedges, 2] sorted vertex pairs
    edge_base: int  # first edge-dof id
    face_keys: np.ndarray = None  # [nfaces, 3] sorted (tets, p = 3)
    face_base: int = 0


def clone_continuous(mesh: Mesh, p: int) -> Clone:
    """Continuous P_p dofs over all cell groups of `mesh` (vertices keep their ids; then one
    block of p-1 nodes per edge, ordered from the lower to the higher vertex id; then one node
    per tetrahedron face for p = 3; then cell-interior nodes group by group). The local order in
    every cell follows the reference elements: vertices, edges in local order and direction,
    faces, interior."""
    nv = mesh.coords.shape[0]
    ne_int = p - 1
    all_edges = []
    for shape, cells in mesh.cells.items():
        for a, b in CELL_EDGES[shape]:
            all_edges.append(np.sort(cells[:, [a, b]], axis=1))
    all_edges = np.concatenate(all_edges) if all_edges else np.zeros((0, 2), np.int32)
    edge_keys, _ = np.unique(all_edges, axis=0, return_inverse=True)
    edge_base = nv
    next_id = nv + edge_keys.shape[0] * ne_int
    ekey = edge_keys[:, 0].astype(np.int64) * (nv + 1) + edge_keys[:, 1]

    def edge_ids(u, v):
        lo, hi = np.minimum(u, v), np.maximum(u, v)
        idx = np.searchsorted(ekey, lo.astype(np.int64) * (nv + 1) + hi)
        return idx, u > v

    face_keys, face_base = None, 0
    if p == 3 and "tetra" in mesh.cells:
        t = mesh.cells["tetra"]
        allf = np.concatenate([np.sort(t[:, list(f)], axis=1) for f in TET_FACES])
        face_keys = np.unique(allf, axis=0)
        face_base = next_id
        next_id += face_keys.shape[0]
    if p > 3 and "tetra" in mesh.cells:
        raise ValueError("tetrahedra up to P3")

    conn, coords_parts = {}, []
    for shape, cells in mesh.cells.items():
        nc = cells.shape[0]
        ref = _ref_nodes(shape, p)
        ndof = ref.shape[0]
        c = np.empty((nc, ndof), dtype=np.int64)
        nvert = cells.shape[1]
        c[:, :nvert] = cells
        k = nvert
        for a, b in CELL_EDGES[shape]:
            idx, rev = edge_ids(cells[:, a], cells[:, b])
            for i in range(ne_int):
                j = np.where(rev, ne_int - 1 - i, i)
                c[:, k + i] = edge_base + idx * ne_int + j
            k += ne_int
        if shape == "tetra" and p == 3:
            fkey = face_keys[:, 0].astype(np.int64) * (nv + 1) ** 2 + \
                face_keys[:, 1].astype(np.int64) * (nv + 1) + face_keys[:, 2]
            for f in TET_FACES:
                s = np.sort(cells[:, list(f)], axis=1).astype(np.int64)
                key = s[:, 0] * (nv + 1) ** 2 + s[:, 1] * (nv + 1) + s[:, 2]
                c[:, k] = face_base + np.searchsorted(fkey, key)
                k += 1
        n_int = ndof - k
        if n_int > 0:
            c[:, k:] = next_id + np.arange(nc * n_int).reshape(nc, n_int)
            next_id += nc * n_int
        conn[shape] = c.astype(np.int32)
        W = _p1_map(shape, ref)  # [ndof, nvert]
        coords_parts.append((c, np.einsum("nk,ckd->cnd", W, mesh.coords[cells])))
    coords = np.zeros((next_id, mesh.dim))
    for c, xy in coords_parts:
        coords[c.ravel()] = xy.reshape(-1, mesh.dim)
    return Clone(p=p, conn=conn, nsol=int(next_id), coords=coords, edge_index=None,
                 edge_keys=edge_keys, edge_base=edge_base, face_keys=face_keys,
                 face_base=face_base)


def boundary_facets(mesh: Mesh, clone: Clone, name: str):
    """(geometry vertices [nf, nfv], solution dofs [nf, nfdof]) of a named boundary, facets in
    the orientation stored in the mesh (outward normals): lines [u, v, edge nodes u->v];
    triangles [a, b, c, edges (a b), (b c), (c a)]."""
    shape, fac = mesh.boundaries[name]
    p = clone.p
    nv = mesh.coords.shape[0]
    ekey = clone.edge_keys[:, 0].astype(np.int64) * (nv + 1) + clone.edge_keys[:, 1]
    ne_int = p - 1

    def edge_nodes(u, v):
        lo, hi = np.minimum(u, v), np.maximum(u, v)
        idx = np.searchsorted(ekey, lo.astype(np.int64) * (nv + 1) + hi)
        rev = u > v
        return np.stack([clone.edge_base + idx * ne_int + np.where(rev, ne_int - 1 - i, i)
                         for i in range(ne_int)], axis=1) if ne_int else np.zeros((len(u), 0), int)

    if shape == "line":
        sol = np.concatenate([fac, edge_nodes(fac[:, 0], fac[:, 1])], axis=1)
    else:
        parts = [fac]
        for a, b in ((0, 1), (1, 2), (2, 0)):
            parts.append(edge_nodes(fac[:, a], fac[:, b]))
        if p == 3:
            raise ValueError("P3 tetrahedron faces need the face node")
        sol = np.concatenate(parts, axis=1)
    return fac.astype(np.int32), sol.astype(np.int32)
