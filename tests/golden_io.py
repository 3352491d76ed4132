"""Reader of the golden cases that oracle/ref_harness.cpp dumps from the reference's own solver
(meta.json + raw little-endian arrays). Test infrastructure: the tests, smoke() and the golden
script use it; the library does not.

A case holds the reference's connectivity (reference dof order), its reference-element tables
built through FEValues, its boundary facets in the order its weak conditions traverse them, the
initial state and the reference's outputs. A mixed mesh (e.g. triangles + quadrilaterals) has one
table set and connectivity per element type, listed under "groups" in meta.json with the array
suffix of each type."""

from __future__ import annotations

import json
import os

import numpy as np

from pdekit_b200 import bcexpr
from pdekit_b200.problem import ADV_CONST_DIR, BCGroup, CellGroup, Problem


def read_arrays(path: str, meta: dict) -> dict:
    arrs = {}
    for k, shp in meta["arrays"].items():
        f64 = os.path.join(path, k + ".f64")
        if os.path.exists(f64):
            arrs[k] = np.fromfile(f64, dtype=np.float64).reshape(shp)
        else:
            arrs[k] = np.fromfile(os.path.join(path, k + ".i32"), dtype=np.int32).reshape(shp)
    return arrs


def _group(arrs: dict, D: int, sfx: str, shape: str, order: int) -> CellGroup:
    g = CellGroup(sol_conn=arrs["sol_conn" + sfx], geo_conn=arrs["geo_conn" + sfx],
                  w=arrs["w" + sfx], V=arrs["V" + sfx],
                  dV=np.stack([arrs[f"dV{d}{sfx}"] for d in range(D)]),
                  dVgeo=np.stack([arrs[f"dVgeo{d}{sfx}"] for d in range(D)]),
                  dVf=np.stack([arrs[f"dVf{d}{sfx}"] for d in range(D)]), Vsf=arrs["Vsf" + sfx],
                  shape=shape, order=order)
    if "vw" + sfx in arrs:
        g.wv = arrs["vw" + sfx]
        g.dVgeo_v = np.stack([arrs[f"vdVgeo{d}{sfx}"] for d in range(D)])
    return g


def load_golden(path: str):
    """Load a golden case written by oracle/ref_harness.cpp.

    Returns (problem, arrays dict, meta dict). The problem uses the reference's own tables and
    connectivity; boundary states are evaluated at the facet quadrature points with the
    named expressions of the case."""
    meta = json.load(open(os.path.join(path, "meta.json")))
    arrs = read_arrays(path, meta)
    D = meta["dim"]
    groups = meta.get("groups") or [{"shape": meta["shape"], "suffix": ""}]
    prob = Problem(physics=meta["physics"], scheme=meta["scheme"], dim=D, neq=meta["neq"],
                   nnodes=meta["nsol"], geo_coords=arrs["geo_coords"],
                   groups=[_group(arrs, D, gm["suffix"], gm["shape"], meta["p"])
                           for gm in groups],
                   bcs=[], adv=ADV_CONST_DIR if meta["physics"] == "advconst" else (0.0, 0.0, 0.0))
    for ib, bc in enumerate(meta["bcs"]):
        b = BCGroup(kind=bc["type"], name=bc["name"], sol_conn=arrs[f"bc{ib}_sol"],
                    geo_conn=arrs[f"bc{ib}_geo"], fw=arrs["fw"], fV=arrs["fV"],
                    fVgeo=arrs["fVgeo"],
                    fdVgeo=np.stack([arrs[f"fdVgeo{d}"] for d in range(D - 1)]),
                    gq=np.zeros((arrs[f"bc{ib}_sol"].shape[0], arrs["fw"].shape[0], meta["neq"])))
        b.order = meta["p"]
        expr = bc["expr"]
        if bc["type"] == "WeakFarfield":  # "state=v0|v1|...", set_reference_state
            b.gq = np.array([float(v) for v in expr.split("=", 1)[1].split("|")])
        elif "=" in expr:  # parameters of WeakSubInlet / WeakSubOutlet
            kv = dict(item.split("=") for item in expr.split(";"))
            if bc["type"] == "WeakSubInlet":
                b.params = (float(kv["total_temperature"]), float(kv["total_pressure"]), 0.0, 0.0)
            else:
                b.params = (float(kv["total_pressure"]), 0.0, 0.0, 0.0)
        elif bc["type"] == "StrongDirichlet":
            # the values the reference's StrongDirichletBC applied (state after its first
            # assemble at the facet dofs): for P2 / P3 facets the reference evaluates its
            # expression at the facet's geometry-node coordinates, also for the dofs past the
            # geometry nodes, so these are not the expression at the dof coordinates there
            b.gq = np.ascontiguousarray(arrs["ua1"][b.sol_conn])
        elif bc["type"] == "WeakDirichlet":
            xq = b.quadrature_coords(prob.geo_coords)
            b.gq = bcexpr.evaluate(expr, xq, meta["neq"])
        prob.bcs.append(b)
    # boundary conditions are applied in the order of their names (std::map in
    # src/solver/rdm/bc/RDMBCManager.hpp:146)
    prob.bcs.sort(key=lambda b: b.name)
    return prob, arrs, meta
