"""Gmsh 2.2 input and nodal-field checkpoints (pdekit_b200/gmsh.py).

The golden cases' mesh files (written for the compiled reference, which read them) are read
back, turned into problems with the library's own continuous numbering, and assembled with the
oracle: the residual, wave speed, time step and dual volume equal the reference's (matched node
by node through the dof coordinates) to 1e-12."""

import json
import os

import numpy as np
import pytest
from scipy.spatial import cKDTree

from conftest import GOLDEN
from helpers import rel_err
from oracle.rds_oracle import Oracle
from pdekit_b200 import gmsh, meshgen
from golden_io import load_golden
from pdekit_b200.workloads import mesh_problem

CASES = ["adv_p1_lda", "adv_p2_b", "adv_p3_lda", "burgers_p2_b", "burgers_p3_b",
         "euler2d_tri_p3_b", "euler2d_quad_p3_b", "euler2d_tri_p1_lda", "euler3d_tet_p2_lda",
         "euler2d_tri_p2_farfield", "euler3d_tet_p2_farfield", "adv_p1_strong"]


def _tables(a, dim):
    st = lambda k, n: np.stack([a[f"{k}{d}"] for d in range(n)])
    t = dict(w=a["w"], V=a["V"], dV=st("dV", dim), dVgeo=st("dVgeo", dim), dVf=st("dVf", dim),
             Vsf=a["Vsf"], fw=a["fw"], fV=a["fV"], fVgeo=a["fVgeo"], fdVgeo=st("fdVgeo", dim - 1))
    if "vw" in a:
        t["wv"], t["dVgeo_v"] = a["vw"], st("vdVgeo", dim)
    return t


def _bc_specs(meta):
    out = []
    for bc in meta["bcs"]:
        kind, name, bnd, expr = bc["type"], bc["name"], bc["boundary"], bc["expr"]
        if kind in ("WeakDirichlet", "StrongDirichlet"):
            out.append((kind, name, bnd, expr))
        elif kind == "WeakFarfield":
            out.append((kind, name, bnd, tuple(float(v) for v in expr[6:].split("|"))))
        elif kind == "WeakSubInlet":
            kv = dict(i.split("=") for i in expr.split(";"))
            out.append((kind, name, bnd, (float(kv["total_temperature"]),
                                          float(kv["total_pressure"]), 0.0, 0.0)))
        elif kind == "WeakSubOutlet":
            kv = dict(i.split("=") for i in expr.split(";"))
            out.append((kind, name, bnd, (float(kv["total_pressure"]), 0.0, 0.0, 0.0)))
        else:
            out.append((kind, name, bnd))
    return out


@pytest.mark.parametrize("case", CASES)
def test_mesh_file_gives_the_reference_residual(case):
    path = os.path.join(GOLDEN, case)
    gprob, a, meta = load_golden(path)
    mesh = gmsh.read_gmsh22(os.path.join(path, "mesh.msh"))
    shape = next(iter(mesh.cells))
    prob = mesh_problem(mesh, meta["physics"], meta["scheme"], meta["p"],
                        {shape: _tables(a, meta["dim"])}, _bc_specs(meta))
    assert prob.nnodes == gprob.nnodes
    dist, perm = cKDTree(a["sol_coords"]).query(prob.sol_coords)
    assert dist.max() < 1e-12 and len(np.unique(perm)) == prob.nnodes
    o = Oracle(prob)
    assert rel_err(o.vol, a["dual_volume"][perm]) < 1e-12
    res, ws, dt, bad = o.assemble(np.asarray(a["u0"])[perm], meta["cfl"])
    assert bad == 0
    assert rel_err(res, np.asarray(a["res1"])[perm]) < 1e-12
    assert rel_err(ws, np.asarray(a["ws1"])[perm]) < 1e-12
    assert rel_err(dt, np.asarray(a["dt1"])[perm]) < 1e-12


def test_read_equals_generated_meshes(tmp_path):
    m2 = meshgen.channel_2d(3, 2, 2, jitter=0.1, seed=5)
    m3 = meshgen.box_tet(2, 2, 1, jitter=0.1, seed=6)
    for m in (m2, m3):
        f = str(tmp_path / "m.msh")
        meshgen.write_gmsh22_mesh(f, m)
        r = gmsh.read_gmsh22(f)
        assert np.array_equal(r.coords, m.coords)
        assert set(r.cells) == set(m.cells)
        for s in m.cells:
            assert np.array_equal(r.cells[s], m.cells[s])
        assert set(r.boundaries) == set(m.boundaries)
        for nm, (s, fac) in m.boundaries.items():
            assert r.boundaries[nm][0] == s
            # same facets with the same (outward) orientation, up to a rotation of the vertices
            canon = lambda f: tuple(np.roll(f, -int(np.argmin(f))))
            assert sorted(map(canon, r.boundaries[nm][1])) == sorted(map(canon, fac))


def test_cells_and_facets_oriented_on_read(tmp_path):
    """A file with clockwise cells and inward facets reads as counter-clockwise cells with
    outward facets."""
    f = str(tmp_path / "cw.msh")
    with open(f, "w") as fh:
        fh.write('$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$PhysicalNames\n2\n1 1 "bottom"\n'
                 '2 2 "domain"\n$EndPhysicalNames\n$Nodes\n4\n1 0 0 0\n2 1 0 0\n3 1 1 0\n'
                 '4 0 1 0\n$EndNodes\n$Elements\n3\n1 1 2 1 1 2 1\n2 2 2 2 2 1 3 2\n'
                 '3 2 2 2 2 1 4 3\n$EndElements\n')
    m = gmsh.read_gmsh22(f)
    X = m.coords
    for c in m.cells["triag"]:
        e1, e2 = X[c[1]] - X[c[0]], X[c[2]] - X[c[0]]
        assert e1[0] * e2[1] - e1[1] * e2[0] > 0
    (u, v), = m.boundaries["bottom"][1]
    t = X[v] - X[u]
    assert np.array_equal([u, v], [0, 1]) and t[0] > 0  # outward normal (0, -1)


def test_node_data_round_trip(tmp_path):
    f = str(tmp_path / "field.msh")
    rng = np.random.default_rng(3)
    u = rng.standard_normal((57, 4)) * 1e5
    dt = rng.random(57)
    gmsh.write_node_data(f, "solution", u, time=0.25, step=7)
    gmsh.write_node_data(f, "time_step", dt)
    got = gmsh.read_node_data(f, [f"solution_{c}" for c in range(4)])
    assert np.array_equal(got, u)
    assert np.array_equal(gmsh.read_node_data(f, ["time_step"])[:, 0], dt)
    text = open(f).read()
    assert text.startswith('$NodeData\n1\n"solution_0"\n1\n0.25\n3\n7\n1\n57\n1 ')
    with pytest.raises(KeyError):
        gmsh.read_node_data(f, ["missing"])
