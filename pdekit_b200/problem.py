"""Problem description shared by the GPU solver and its checkers.

A problem is what the reference's RDMethod is configured with before the pseudo-time loop
(src/solver/rdm/RDMethod.hpp:159-243): the physics and scheme (template arguments of
PGRDMethodExplicit), geometry node coordinates, one group of cells per element type with its
reference-element tables (FEValues: V, dV, quadrature weights; FluxSpaceMetric: dVf, Vsf), and
one group of boundary facets per weak boundary condition with its facet tables and the
boundary state at the facet quadrature points.

All arrays are host numpy arrays; layouts are row-major, derivative tables are stacked
[dim][rows][cols], connectivities are int32 [entities][local nodes].
"""

from __future__ import annotations

import dataclasses
import json
import os

import numpy as np


@dataclasses.dataclass
class CellGroup:
    sol_conn: np.ndarray  # [ncells, ndof] int32
    geo_conn: np.ndarray  # [ncells, ngeo] int32
    w: np.ndarray  # [nq]
    V: np.ndarray  # [nq, ndof]
    dV: np.ndarray  # [dim, nq, ndof]
    dVgeo: np.ndarray  # [dim, nq, ngeo]
    dVf: np.ndarray  # [dim, nq, nfl]
    Vsf: np.ndarray  # [nfl, ndof]
    shape: str = "triag"
    order: int = 1
    wv: np.ndarray = None  # [nqv] dual-volume rule (Gauss rule of the cell order), optional
    dVgeo_v: np.ndarray = None  # [dim, nqv, ngeo]

    @property
    def ncells(self):
        return self.sol_conn.shape[0]

    @property
    def ndof(self):
        return self.sol_conn.shape[1]

    @property
    def ngeo(self):
        return self.geo_conn.shape[1]

    @property
    def nq(self):
        return self.w.shape[0]

    @property
    def nfl(self):
        return self.Vsf.shape[0]


@dataclasses.dataclass
class BCGroup:
    kind: str  # WeakDirichlet | WeakWall | WeakSubInlet | WeakSubOutlet | WeakFarfield |
    # StrongDirichlet
    name: str
    sol_conn: np.ndarray  # [nfacets, nfdof] int32
    geo_conn: np.ndarray  # [nfacets, nfgeo] int32
    fw: np.ndarray  # [nfq]
    fV: np.ndarray  # [nfq, nfdof]
    fVgeo: np.ndarray  # [nfq, nfgeo]
    fdVgeo: np.ndarray  # [dim-1, nfq, nfgeo]
    # WeakDirichlet: [nfacets, nfq, neq] boundary state at the facet quadrature points;
    # WeakFarfield: [neq] reference state (conservative); StrongDirichlet: [nfacets, nfdof, neq]
    # values the facet dofs take (facet by facet, a shared dof keeps the later value)
    gq: np.ndarray
    order: int = 1  # polynomial order of the facet's solution basis
    params: tuple = (0.0, 0.0, 0.0, 0.0)  # WeakSubInlet: (T_tot, p_tot); WeakSubOutlet: (p,)

    @property
    def nfacets(self):
        return self.sol_conn.shape[0]

    @property
    def nfdof(self):
        return self.sol_conn.shape[1]

    @property
    def nfgeo(self):
        return self.geo_conn.shape[1]

    @property
    def nfq(self):
        return self.fw.shape[0]

    def quadrature_coords(self, geo_coords):
        """Physical coordinates of the facet quadrature points [nfacets, nfq, dim]."""
        X = geo_coords[self.geo_conn]  # [nf, nfgeo, dim]
        return np.einsum("qg,fgd->fqd", self.fVgeo, X)


@dataclasses.dataclass
class Problem:
    physics: str  # advconst | burgers | euler2d | euler3d
    scheme: str  # lda | n | b
    dim: int
    neq: int
    nnodes: int
    geo_coords: np.ndarray  # [ngeo_nodes, dim]
    groups: list
    bcs: list
    adv: tuple = (0.0, 0.0, 0.0)
    gamma: float = 1.4

    @property
    def ncells(self):
        return sum(g.ncells for g in self.groups)


ADV_CONST_DIR = (0.5 / np.sqrt(1.25), 1.0 / np.sqrt(1.25), 0.0)


def load_golden(path: str):
    """Load a golden case written by oracle/ref_harness.cpp (meta.json + raw arrays).

    Returns (problem, arrays dict, meta dict). The problem uses the reference's own tables and
    connectivity; boundary states are evaluated at the facet quadrature points with the
    named expressions of the case."""
    meta = json.load(open(os.path.join(path, "meta.json")))
    arrs = {}
    for k, shp in meta["arrays"].items():
        f64 = os.path.join(path, k + ".f64")
        if os.path.exists(f64):
            arrs[k] = np.fromfile(f64, dtype=np.float64).reshape(shp)
        else:
            arrs[k] = np.fromfile(os.path.join(path, k + ".i32"), dtype=np.int32).reshape(shp)
    D = meta["dim"]
    g = CellGroup(sol_conn=arrs["sol_conn"], geo_conn=arrs["geo_conn"], w=arrs["w"],
                  V=arrs["V"], dV=np.stack([arrs[f"dV{d}"] for d in range(D)]),
                  dVgeo=np.stack([arrs[f"dVgeo{d}"] for d in range(D)]),
                  dVf=np.stack([arrs[f"dVf{d}"] for d in range(D)]), Vsf=arrs["Vsf"],
                  shape=meta["shape"], order=meta["p"])
    if "vw" in arrs:
        g.wv = arrs["vw"]
        g.dVgeo_v = np.stack([arrs[f"vdVgeo{d}"] for d in range(D)])
    prob = Problem(physics=meta["physics"], scheme=meta["scheme"], dim=D, neq=meta["neq"],
                   nnodes=meta["nsol"], geo_coords=arrs["geo_coords"], groups=[g], bcs=[],
                   adv=ADV_CONST_DIR if meta["physics"] == "advconst" else (0.0, 0.0, 0.0))
    from . import bcexpr
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
