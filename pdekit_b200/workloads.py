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
    conn, nsol, xy = meshgen.clone_continuous_tri(mesh, p)
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
    prob.sol_coords = xy
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


def config1(n=64, seed=1, scheme="lda"):
    """Configuration 1: constant advection, P1 triangles on an n x n grid (jitter 0.2h), 6-point
    rule, inflow sin(2 pi x) / 0, initial u = 0 (run at CFL 0.9)."""
    from . import reference_element as R

    prob = tri_problem("advconst", scheme, 1, n, 0.2, seed, ADV_BCS, R.triag_tables(1, 4))
    return prob, initial_state(prob, "zero", prob.sol_coords)


def config2(n=512, seed=7, scheme="b"):
    """Configuration 2: Burgers, P2 triangles on an n x n grid (jitter 0.15h), 7-point rule,
    inflow 1.5 - 2x, initial 1.5 - 2x + 0.1 sin(7x + 3y) y (run at CFL 0.5)."""
    from . import reference_element as R

    prob = tri_problem("burgers", scheme, 2, n, 0.15, seed, BURGERS_BCS, R.triag_tables(2, 5))
    return prob, initial_state(prob, "burgers", prob.sol_coords)


# ---------------------------------------------------------------------------------------------
# Configurations 3 and 4 (Euler) on general meshes
# ---------------------------------------------------------------------------------------------

T_TOT, P_TOT, P_OUT = 307.6488978, 120195.4453, 101325.0


def euler_bcs(dim: int):
    """Weak walls, subsonic total-condition inlet and static-pressure outlet of the reference's
    bump case (examples/testcases-rdm/Bump-RDS-2D-Explicit.cpp:137-150)."""
    walls = [("WeakWall", "bottom_wall_bc", "bottom_wall"), ("WeakWall", "top_wall_bc", "top_wall")]
    if dim == 3:
        walls.append(("WeakWall", "side_walls_bc", "side_walls"))
    return walls + [("WeakSubInlet", "inlet_bc", "inlet", (T_TOT, P_TOT, 0.0, 0.0)),
                    ("WeakSubOutlet", "outlet_bc", "outlet", (P_OUT, 0.0, 0.0, 0.0))]


def mesh_problem(mesh, physics: str, scheme: str, p: int, tables: dict, bcs) -> Problem:
    """Problem on a general mesh: one cell group per element shape (tables[shape]), one boundary
    condition per (kind, name, boundary[, data]) in `bcs`; data: the expression name
    (WeakDirichlet, at the facet quadrature points; StrongDirichlet, at the facet dofs), the
    parameters (WeakSubInlet / WeakSubOutlet) or the reference state (WeakFarfield)."""
    clone = meshgen.clone_continuous(mesh, p)
    dim = mesh.dim
    neq = {"advconst": 1, "burgers": 1, "euler2d": 4, "euler3d": 5}[physics]
    groups = []
    for shape, conn in clone.conn.items():
        t = tables[shape]
        groups.append(CellGroup(sol_conn=conn, geo_conn=mesh.cells[shape], w=t["w"], V=t["V"],
                                dV=t["dV"], dVgeo=t["dVgeo"], dVf=t["dVf"], Vsf=t["Vsf"],
                                shape=shape, order=p, wv=t.get("wv"), dVgeo_v=t.get("dVgeo_v")))
    prob = Problem(physics=physics, scheme=scheme, dim=dim, neq=neq, nnodes=clone.nsol,
                   geo_coords=mesh.coords, groups=groups, bcs=[],
                   adv=ADV_CONST_DIR if physics == "advconst" else (0.0, 0.0, 0.0))
    facet_tables = tables[next(iter(clone.conn))]
    for spec in bcs:
        kind, name, boundary = spec[:3]
        params = spec[3] if len(spec) > 3 and not isinstance(spec[3], str) else (0.0,) * 4
        geo, sol = meshgen.boundary_facets(mesh, clone, boundary)
        t = facet_tables
        b = BCGroup(kind=kind, name=name, sol_conn=sol, geo_conn=geo, fw=t["fw"], fV=t["fV"],
                    fVgeo=t["fVgeo"], fdVgeo=t["fdVgeo"],
                    gq=np.zeros((geo.shape[0], t["fw"].shape[0], neq)), order=p,
                    params=tuple(params))
        if kind == "WeakDirichlet":
            b.gq = bcexpr.evaluate(spec[3], b.quadrature_coords(mesh.coords), neq)
        elif kind == "StrongDirichlet":
            b.gq = bcexpr.evaluate(spec[3], clone.coords[sol], neq)
        elif kind == "WeakFarfield":
            b.gq = np.asarray(spec[3], dtype=np.float64)
            b.params = (0.0,) * 4
        prob.bcs.append(b)
    prob.bcs.sort(key=lambda b: b.name)
    prob.sol_coords = clone.coords
    return prob


def bump_state(xyz: np.ndarray, dim: int, mach: float) -> np.ndarray:
    """Freestream of the bump cases (total 307.6488978 K / 120195.4453 Pa, R = 287.046) with a
    +-1% perturbation of density and pressure that is a fixed pseudo-random function of the
    coordinates (the same definition as the golden fixtures' harness)."""
    gamma, R = 1.4, 287.046
    f = 1.0 + 0.5 * (gamma - 1.0) * mach * mach
    T = T_TOT / f
    p0 = P_TOT / f ** (gamma / (gamma - 1.0))
    x, y = xyz[:, 0], xyz[:, 1]
    z = xyz[:, 2] if dim == 3 else np.zeros_like(x)

    def h(a, b, c):
        s = np.sin(12.9898 * a + 78.233 * b + 37.719 * c) * 43758.5453
        return 2.0 * (s - np.floor(s)) - 1.0

    rho = p0 / (R * T) * (1.0 + 0.01 * h(x, y, z))
    p = p0 * (1.0 + 0.01 * h(y, z, x))
    ux = mach * np.sqrt(gamma * R * T)
    u = np.zeros((xyz.shape[0], dim + 2))
    u[:, 0] = rho
    u[:, 1] = rho * ux
    u[:, dim + 1] = p / (gamma - 1.0) + 0.5 * rho * ux * ux
    return u


def config3(nx_tri=500, nx_quad=1000, ny=500, seed=3):
    """Configuration 3: Euler 2D bump channel, P3 triangles (16-point rule) on x < 0 and P3
    quadrilaterals (25-point rule) on x > 0, blended B scheme, Mach 0.5."""
    from . import reference_element as R

    mesh = meshgen.channel_2d(nx_tri, nx_quad, ny, jitter=0.0, seed=seed)
    tables = {"triag": dict(R.triag_tables(3, 8), wv=R.triag_gauss(3)[1],
                            dVgeo_v=R.lagrange_triag(1, R.triag_gauss(3)[0])[1]),
              "quad": R.quad_tables(3, 8, tensor=True)}
    prob = mesh_problem(mesh, "euler2d", "b", 3, tables, euler_bcs(2))
    return prob, bump_state(prob.sol_coords, 2, 0.5)


def config4(nx=128, ny=32, nz=32, seed=4):
    """Configuration 4: Euler 3D bump box, 128 x 32 x 32 hexahedra split into 6 P2 tetrahedra
    (786,432 cells), 14-point rule, LDA, Mach 0.6, vertices jittered by +-0.1h."""
    from . import reference_element as R

    mesh = meshgen.box_tet(nx, ny, nz, jitter=0.1, seed=seed)
    prob = mesh_problem(mesh, "euler3d", "lda", 2, {"tetra": R.tet_tables(2, 5)}, euler_bcs(3))
    return prob, bump_state(prob.sol_coords, 3, 0.6)


def config5(nprob=256, seed=5, min_cells=1000, max_cells=200000):
    """Configuration 5: `nprob` independent unit-square problems drawn from `seed`: advection
    (LDA, CFL U[0.5, 0.9], initial 0) or Burgers (N scheme, CFL U[0.3, 0.6], initial
    1.5 - 2x + 0.1 sin(7x + 3y) y), order P1 / P2 / P3 (6 / 7 / 16-point rules), cell count
    log-uniform in [min_cells, max_cells] (n x n squares, n = round(sqrt(cells / 2))), jitter
    0.2h. Returns (problems, initial states, CFLs, descriptions)."""
    from . import reference_element as R

    rng = np.random.default_rng(seed)
    rules = {1: 4, 2: 5, 3: 8}
    tables = {p: R.triag_tables(p, rules[p]) for p in (1, 2, 3)}
    probs, states, cfls, info = [], [], [], []
    for i in range(nprob):
        kind = "advconst" if rng.random() < 0.5 else "burgers"
        p = int(rng.integers(1, 4))
        cells = float(np.exp(rng.uniform(np.log(min_cells), np.log(max_cells))))
        n = max(2, int(round(np.sqrt(cells / 2.0))))
        pseed = int(rng.integers(0, 2**31 - 1))
        if kind == "advconst":
            prob = tri_problem(kind, "lda", p, n, 0.2, pseed, ADV_BCS, tables[p])
            u0 = initial_state(prob, "zero", prob.sol_coords)
            cfl = float(rng.uniform(0.5, 0.9))
        else:
            prob = tri_problem(kind, "n", p, n, 0.2, pseed, BURGERS_BCS, tables[p])
            u0 = initial_state(prob, "burgers", prob.sol_coords)
            cfl = float(rng.uniform(0.3, 0.6))
        probs.append(prob)
        states.append(u0)
        cfls.append(cfl)
        info.append({"physics": kind, "order": p, "n": n, "cells": prob.ncells, "cfl": cfl})
    return probs, states, np.array(cfls), info
