"""Synthetic workloads of the benchmark configurations, as Problem descriptions.

Configuration 1: linear advection, a = (0.5,1)/|(0.5,1)|, unit square, 64x64 squares split into
P1 triangles, interior jitter +-0.2h, inflow u = sin(2 pi x) at y = 0 and u = 0 at x = 0, LDA,
P4 quadrature rule (6 points), local CFL 0.9, initial u = 0.
Configuration 2: Burgers u_t + (u^2/2)_x + u_y = 0, [0,1]^2, 512x512 squares split into P2
triangles (equispaced nodes, straight edges), interior jitter +-0.15h, inflow u = 1.5 - 2x at
y = 0 (with u = 1.5 / -0.5 on the left / right edges, which are inflow for this flux), blended
B scheme, 7-point rule.
Configuration 5 (batched): many independent advection / Burgers problems on P1-P3 triangles.
"""

from __future__ import annotations

import numpy as np

from . import bcexpr, meshgen
from .problem import ADV_CONST_DIR, BCGroup, CellGroup, Problem

ADV_BCS = [("WeakDirichlet", "inlet_bottom", "bottom", "sin2pix"),
           ("WeakDirichlet", "inlet_left", "left", "zero")]
BURGERS_BCS = [("WeakDirichlet", "inlet", "bottom", "burgers_inlet"),
               ("WeakDirichlet", "left", "left", "c1.5"),
               ("WeakDirichlet", "right", "right", "c-0.5")]


def tri_problem(physics: str, scheme: str, p: int, n: int, jitter: float, seed: int, bcs,
                tables: dict) -> Problem:
    """Unit-square triangle problem of order p with the reference-element tables `tables`
    (keys w, V, dV, dVgeo, dVf, Vsf for cells; fw, fV, fVgeo, fdVgeo for facets)."""
    mesh = meshgen.unit_square_tri(n, jitter, seed=seed)
    conn, nsol, _ = meshgen.clone_continuous_tri(mesh, p)
    g = CellGroup(sol_conn=conn, geo_conn=mesh.cells, w=tables["w"], V=tables["V"],
                  dV=tables["dV"], dVgeo=tables["dVgeo"], dVf=tables["dVf"], Vsf=tables["Vsf"],
                  shape="triag", order=p)
    neq = 1
    prob = Problem(physics=physics, scheme=scheme, dim=2, neq=neq, nnodes=nsol,
                   geo_coords=mesh.coords, groups=[g], bcs=[],
                   adv=ADV_CONST_DIR if physics == "advconst" else (0.0, 0.0, 0.0))
    for kind, name, boundary, expr in bcs:
        geo, sol = meshgen.boundary_facets_tri(mesh, conn, p, boundary)
        b = BCGroup(kind=kind, name=name, sol_conn=sol, geo_conn=geo, fw=tables["fw"],
                    fV=tables["fV"], fVgeo=tables["fVgeo"], fdVgeo=tables["fdVgeo"],
                    gq=np.zeros((geo.shape[0], tables["fw"].shape[0], neq)))
        b.gq = bcexpr.evaluate(expr, b.quadrature_coords(mesh.coords), neq)
        prob.bcs.append(b)
    prob.bcs.sort(key=lambda b: b.name)  # the reference applies BCs in name order
    return prob


def initial_state(prob: Problem, name: str, sol_coords: np.ndarray) -> np.ndarray:
    """Initial states as functions of the node coordinates (same definitions as the golden
    fixtures' harness)."""
    x, y = sol_coords[:, 0], sol_coords[:, 1]
    if name == "zero":
        u = np.zeros_like(x)
    elif name == "smooth":
        u = 0.3 * np.sin(3.1 * x + 1.7 * y) + 0.2 * np.cos(5.3 * x * y) + 0.1 * x - 0.05
    elif name == "burgers":
        u = 1.5 - 2.0 * x + 0.1 * np.sin(7.0 * x + 3.0 * y) * y
    else:
        raise ValueError(name)
    return u.reshape(-1, 1)


def sol_coords_tri(n: int, jitter: float, seed: int, p: int) -> np.ndarray:
    mesh = meshgen.unit_square_tri(n, jitter, seed=seed)
    _, _, xy = meshgen.clone_continuous_tri(mesh, p)
    return xy
