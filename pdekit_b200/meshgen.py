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
    edge_ids = {}
    next_id = nv
    ndof = tri_dof_layout(p)
    n_int = ndof - 3 - 3 * ne_int
    conn = np.empty((nc, ndof), dtype=np.int32)
    ref = equidist_triag_nodes(p)  # on (-1,-1),(1,-1),(-1,1)
    coords_out = {}
    for c in range(nc):
        v = mesh.cells[c]
        conn[c, :3] = v
        k = 3
        for (a, b) in ((v[0], v[1]), (v[1], v[2]), (v[2], v[0])):
            key = (min(a, b), max(a, b))
            if key not in edge_ids:
                edge_ids[key] = np.arange(next_id, next_id + ne_int, dtype=np.int32)
                next_id += ne_int
            ids = edge_ids[key]
            if a > b:
                ids = ids[::-1]
            conn[c, k:k + ne_int] = ids
            k += ne_int
        if n_int > 0:
            conn[c, k:] = np.arange(next_id, next_id + n_int, dtype=np.int32)
            next_id += n_int
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
    edges = mesh.boundaries[name]
    # map each directed cell edge to (cell, local edge)
    lookup = {}
    for c, (a, b, cc) in enumerate(mesh.cells):
        for le, (u, v) in enumerate(((a, b), (b, cc), (cc, a))):
            lookup[(min(u, v), max(u, v))] = (c, le, u, v)
    geo = np.empty((len(edges), 2), dtype=np.int32)
    sol = np.empty((len(edges), p + 1), dtype=np.int32)
    for k, (a, b) in enumerate(edges):
        c, le, u, v = lookup[(min(a, b), max(a, b))]
        geo[k] = (u, v)
        dofs = [u, v]
        if p > 1:
            start = 3 + le * (p - 1)
            dofs += list(sol_conn[c, start:start + p - 1])
        sol[k] = dofs
    return geo, sol
