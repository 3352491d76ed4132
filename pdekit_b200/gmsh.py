"""Gmsh 2.2 ASCII input and nodal-field checkpoints: the on-disk formats the reference reads and
writes around the solver.

* `read_gmsh22(path)` reads a mesh file into a P1 `meshgen.Mesh` (cells grouped by shape,
  boundary facets grouped by physical name), as the reference's GmshReader does
  (src/mesh/io/gmsh/GmshReader.hpp:119-476): nodes, elements of the mesh's top dimension as
  cells, elements of one dimension lower as boundary facets of the physical group they carry.
  Cells with negative orientation are turned (two vertices swapped) and every boundary facet is
  ordered so that its normal points out of its cell, which is the orientation the facet kernels
  and `meshgen.boundary_facets` expect.
* `write_node_data` / `read_node_data` write and read `$NodeData` blocks in the reference's form
  (src/mesh/io/gmsh/GmshWriter.hpp:205-280, GmshReader.hpp:481-545): one block per component
  named "<field>_<component>" (a one-column field: "<field>"), one real tag (time), three integer
  tags (time step, 1 component, number of entries), then "index value" lines, 1-based, written
  with enough digits to read back the same doubles. A solver state saved this way is a
  checkpoint that the reference's reader also accepts.
"""

from __future__ import annotations

import numpy as np

from .meshgen import Mesh

# Gmsh element type -> (shape, number of nodes, dimension)
_ELEM = {1: ("line", 2, 1), 2: ("triag", 3, 2), 3: ("quad", 4, 2), 4: ("tetra", 4, 3),
         15: ("point", 1, 0)}


def _sections(path):
    """{section name: list of lines between $Name and $EndName}; $NodeData may repeat."""
    out = {}
    cur, buf = None, []
    with open(path) as f:
        for raw in f:
            line = raw.strip()
            if cur is None:
                if line.startswith("$") and not line.startswith("$End"):
                    cur, buf = line[1:], []
            elif line == "$End" + cur:
                out.setdefault(cur, []).append(buf)
                cur = None
            else:
                buf.append(line)
    return out


def read_gmsh22(path: str) -> Mesh:
    """P1 mesh of a Gmsh 2.2 ASCII file (see the module docstring)."""
    sec = _sections(path)
    fmt = sec.get("MeshFormat", [[""]])[0][0].split()
    if not fmt or not fmt[0].startswith("2"):
        raise ValueError(f"{path}: not a Gmsh 2.x ASCII file")
    if len(fmt) > 1 and fmt[1] != "0":
        raise ValueError(f"{path}: binary Gmsh files are not supported")
    names = {}
    for line in sec.get("PhysicalNames", [[]])[0][1:]:
        d, tag, nm = line.split(maxsplit=2)
        names[(int(d), int(tag))] = nm.strip('"')
    nodes = sec["Nodes"][0]
    nn = int(nodes[0])
    ids = np.empty(nn, dtype=np.int64)
    xyz = np.empty((nn, 3))
    for i, line in enumerate(nodes[1:nn + 1]):
        t = line.split()
        ids[i] = int(t[0])
        xyz[i] = [float(v) for v in t[1:4]]
    index = {int(k): i for i, k in enumerate(ids)}
    elems = sec["Elements"][0]
    ne = int(elems[0])
    by_dim = {}
    for line in elems[1:ne + 1]:
        t = [int(v) for v in line.split()]
        etype, ntags = t[1], t[2]
        if etype not in _ELEM:
            raise ValueError(f"{path}: Gmsh element type {etype} is not supported")
        shape, nv, d = _ELEM[etype]
        phys = t[3] if ntags > 0 else 0
        verts = [index[v] for v in t[3 + ntags:3 + ntags + nv]]
        by_dim.setdefault(d, []).append((shape, phys, verts))
    tdim = max(by_dim)
    if tdim < 2:
        raise ValueError(f"{path}: no 2D or 3D cells")
    coords = np.ascontiguousarray(xyz[:, :tdim])

    cells = {}
    for shape, _, verts in by_dim[tdim]:
        cells.setdefault(shape, []).append(verts)
    cells = {s: np.array(v, dtype=np.int32) for s, v in cells.items()}
    for s, c in cells.items():
        _orient_cells(s, c, coords)

    # every face of every cell, keyed by its sorted vertices -> (a vertex of the cell off it)
    faces = {}
    for s, c in cells.items():
        for lf in _FACES[s]:
            other = [k for k in range(c.shape[1]) if k not in lf][0]
            for row in c:
                faces[tuple(sorted(row[list(lf)]))] = row[other]
    bnd = {}
    for shape, phys, verts in by_dim.get(tdim - 1, []):
        nm = names.get((tdim - 1, phys), f"physical_{phys}")
        key = tuple(sorted(verts))
        if key not in faces:
            raise ValueError(f"{path}: boundary element {verts} of '{nm}' is no cell face")
        bnd.setdefault(nm, (shape, []))[1].append(_orient_facet(verts, faces[key], coords))
    boundaries = {nm: (s, np.array(f, dtype=np.int32)) for nm, (s, f) in bnd.items()}
    return Mesh(coords=coords, cells=cells, boundaries=boundaries)


_FACES = {"triag": [(0, 1), (1, 2), (2, 0)], "quad": [(0, 1), (1, 2), (2, 3), (3, 0)],
          "tetra": [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]}


def _orient_cells(shape, c, X):
    """Positive orientation (counter-clockwise in 2D, positive volume in 3D), in place."""
    if shape == "tetra":
        a, b, cc, d = (X[c[:, k]] for k in range(4))
        neg = np.einsum("ij,ij->i", np.cross(b - a, cc - a), d - a) < 0
        c[neg] = c[neg][:, [0, 2, 1, 3]]
    else:
        p = X[c]
        area = 0.5 * np.sum(p[:, :, 0] * np.roll(p[:, :, 1], -1, axis=1)
                            - np.roll(p[:, :, 0], -1, axis=1) * p[:, :, 1], axis=1)
        neg = area < 0
        c[neg] = c[neg][:, ::-1] if shape == "triag" else c[neg][:, [0, 3, 2, 1]]


def _orient_facet(verts, off, X):
    """The facet's vertices ordered so that its normal points away from the cell vertex `off`
    (2D: normal (dy, -dx) of the edge v0 -> v1; 3D: (v1 - v0) x (v2 - v0))."""
    p = X[verts]
    if len(verts) == 2:
        t = p[1] - p[0]
        n = np.array([t[1], -t[0]])
    else:
        n = np.cross(p[1] - p[0], p[2] - p[0])
    if np.dot(n, X[off] - p[0]) > 0:
        verts = [verts[1], verts[0]] if len(verts) == 2 else [verts[0], verts[2], verts[1]]
    return verts


def write_node_data(path: str, name: str, values, time: float = 0.0, step: int = 0) -> None:
    """Append `values` ([n] or [n, k]) to a Gmsh file as $NodeData blocks (one per column,
    named "<name>_<column>" when k > 1)."""
    v = np.asarray(values, dtype=np.float64)
    cols = [(name, v)] if v.ndim == 1 else [(f"{name}_{c}", v[:, c]) for c in range(v.shape[1])]
    with open(path, "a") as f:
        for nm, col in cols:
            f.write(f'$NodeData\n1\n"{nm}"\n1\n{time!r}\n3\n{step}\n1\n{len(col)}\n')
            f.write("".join(f"{i + 1} {x!r}\n" for i, x in enumerate(col.tolist())))
            f.write("$EndNodeData\n")


def read_node_data(path: str, names) -> np.ndarray:
    """[n, len(names)] from the $NodeData blocks of those names (the last block of a name wins,
    as in the reference's reader, which reads every block of a requested name in turn)."""
    blocks = {}
    for b in _sections(path).get("NodeData", []):
        nstr = int(b[0])
        nm = b[1].strip('"')
        k = 1 + nstr
        nreal = int(b[k])
        k += 1 + nreal
        nint = int(b[k])
        ints = [int(x) for x in b[k + 1:k + 1 + nint]]
        k += 1 + nint
        n = ints[-1]
        idx = np.empty(n, dtype=np.int64)
        val = np.empty(n)
        for i, line in enumerate(b[k:k + n]):
            a, x = line.split()
            idx[i], val[i] = int(a) - 1, float(x)
        col = np.zeros(int(idx.max()) + 1 if n else 0)
        col[idx] = val
        blocks[nm] = col
    missing = [nm for nm in names if nm not in blocks]
    if missing:
        raise KeyError(f"{path}: no $NodeData named {missing}")
    n = max(len(blocks[nm]) for nm in names)
    out = np.zeros((n, len(names)))
    for c, nm in enumerate(names):
        out[:len(blocks[nm]), c] = blocks[nm]
    return out
