"""Stabilisation operators on the CPU: the oracle restatement against the reference's own
outputs (tests/golden/*: the sensor, the normalised indicator, the blending coefficients and
their nodal fields, dumped through ArtificialViscosity / RDBlendingCoeff), and the host tables
the GPU sensor uses (reference_element.stab_tables) evaluated in numpy with the kernel's
formula against the same outputs."""

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, stab_cases
from oracle import stab_oracle as so
from golden_io import load_golden
from pdekit_b200.reference_element import stab_tables

# FP64 restatement: rounding only; the reference's tetrahedron rules of orders 2 and 4 are
# tabulated to about 10 digits (its results differ from exact integration by ~1e-10 - 1e-9
# relative)
TOL = {2: 1e-12, 3: 1e-8}


def _case(c):
    prob, a, meta = load_golden(os.path.join(GOLDEN, c))
    kind, *par = meta["stab"].split(":")
    return prob, a, meta, kind, par


def _rel(got, ref):
    scale = max(np.abs(ref).max(), 1e-300)
    return np.abs(got - ref).max() / scale


@pytest.mark.parametrize("case", stab_cases())
def test_oracle_matches_reference(case):
    prob, a, meta, kind, par = _case(case)
    dim, p = meta["dim"], meta["p"]
    u0 = a["u0"][:, 0]
    quad = prob.groups[0].shape == "quad"
    P1 = so.q1_at(a["sol_nodes"]) if quad else so.p1_at(dim, a["sol_nodes"])
    tol = TOL[dim]
    if kind.startswith("av"):
        kappa, factor = float(par[0]), float(par[1])
        av = so.sensor_cells(dim, p, a["sol_nodes"], a["geo_coords"], a["geo_conn"],
                             a["sol_conn"], u0, kappa, factor)
        assert _rel(av, a["av_cell"]) < tol
        ind = so.sensor_cells(dim, p, a["sol_nodes"], a["geo_coords"], a["geo_conn"],
                              a["sol_conn"], u0, kappa, 1.0)
        if ind.max() >= 1e-14:
            ind = ind / ind.max()
        assert _rel(ind, a["indicator"]) < max(tol, 1e-12) * 100
        if kind == "av":  # the reference's own transfer (2D; it crashes on tetrahedra)
            nod = so.nodal_from_cells(a["av_cell"], a["sol_conn"], meta["nsol"], P1)
            assert _rel(nod, a["av_nodal"]) < 1e-14
    else:
        typ, prm = par[0], float(par[1])
        if typ == "ViscosityIndicator":
            bc = so.sensor_cells(dim, p, a["sol_nodes"], a["geo_coords"], a["geo_conn"],
                                 a["sol_conn"], u0, prm, blend=True)
        elif typ.startswith("Bonanni"):
            g = prob.groups[0]
            bc = so.bonanni([(g.shape, g.order, a["sol_nodes"], a["geo_coords"], a["geo_conn"],
                              a["sol_conn"])], a["u0"], prob.gamma, dim)
        else:
            bc = so.blend_cells(typ, a["sol_conn"], u0, prm)
        assert _rel(bc, a["blend_cell"]) < tol
        nod = so.nodal_from_cells(a["blend_cell"], a["sol_conn"], meta["nsol"], P1)
        assert _rel(nod, a["blend_nodal"]) < 1e-14


def test_cases_exercise_every_branch():
    """The fixtures hold cells on both sides of the sensor's switch-off and nonzero nodal
    fields, for every operator."""
    seen = set()
    for c in stab_cases():
        _, a, meta, kind, par = _case(c)
        key = "av_cell" if kind.startswith("av") else "blend_cell"
        v = a[key]
        assert v.max() > 0.0, c
        seen.add(kind if kind.startswith("av") else par[0])
        if kind.startswith("av"):
            assert (v == 0.0).any() or meta["p"] == 1, c
    assert {"av", "av3d", "LF_Blend", "WongJansen", "ViscosityIndicator", "Bonanni2D",
            "Bonanni3D"} <= seen


def _sensor_weights(t, a, dim):
    """detJ w per cell and point: affine simplices from their vertices, mapped cells
    (t["dVgeo"], bilinear quadrilaterals) per point, as the kernel takes them."""
    if "dVgeo" in t:
        J = np.einsum("aqg,cgx->cqax", t["dVgeo"], a["geo_coords"][a["geo_conn"]])
        return np.linalg.det(J) * t["w"][None, :]
    X = a["geo_coords"][a["geo_conn"][:, :dim + 1]]
    J = np.stack([X[:, k + 1] - X[:, 0] for k in range(dim)], 2) / 2
    return np.linalg.det(J)[:, None] * t["w"][None, :]


def _sensor_numpy(t, a, dim, p, kappa, factor, blend):
    u = a["u0"][:, 0][a["sol_conn"]]
    wj = _sensor_weights(t, a, dim)
    s, r = u @ t["Vn"].T, u @ t["R"].T
    nom, den, vol = (wj * r * r).sum(1), (wj * s * s).sum(1), wj.sum(1)
    Se = np.where(den <= 1e-10, 0.0, nom / np.where(den <= 1e-10, 1.0, den))
    with np.errstate(divide="ignore"):
        se = np.log(Se) / np.log(10.0)
    s0 = 1.0 / p ** 4
    e0 = 1.0 if blend else factor * vol ** (1.0 / dim) / p
    return np.where(se < s0 - kappa, 0.0, np.where(se > s0 + kappa, e0,
                    0.5 * e0 * (1 + np.sin(np.pi * (se - s0) / (2 * kappa)))))


@pytest.mark.parametrize("case,p", [("euler2d_quad_p2_b_bonanni", 2), ("euler2d_quad_p3_b", 3)])
@pytest.mark.parametrize("blend", [False, True])
def test_quad_sensor_tables_match_oracle_above_p1(case, p, blend):
    """Quadrilaterals of order >= 2, where the reference's own value follows the rounding of a
    singular mass matrix's inversion: the host tables against the oracle's projection with a
    regular mass matrix, on the fixtures' bilinear meshes and states (steep fronts)."""
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    g = prob.groups[0]
    assert g.shape == "quad" and g.order == p and meta["p"] == p
    t = stab_tables("quad", p, 4)
    u0 = a["u0"][:, 0]
    for kappa in (0.5, 2.0, 4.0):
        ref = so.sensor_cells(2, p, a["sol_nodes"], a["geo_coords"], a["geo_conn"], a["sol_conn"],
                              u0, kappa, 1.3, blend=blend)
        got = _sensor_numpy(t, a, 2, p, kappa, 1.3, blend)
        assert _rel(got, ref) < 1e-12


def test_quad_mass_matrix_is_singular_above_p1():
    """The reason for the above: the reference's rule of order 2p on the square has fewer points
    than Q_p has modes for p >= 2, so no mass matrix built on it is regular."""
    from pdekit_b200.reference_element import quad_gauss
    assert [len(quad_gauss(2 * p)[1]) for p in (1, 2, 3)] == [4, 8, 12]
    assert [(p + 1) ** 2 for p in (1, 2, 3)] == [4, 9, 16]


@pytest.mark.parametrize("case", [c for c in stab_cases()
                                  if c.endswith("_av") or c.endswith("_visc")])
def test_host_sensor_tables_give_reference_values(case):
    """stab_tables + the kernel's formula (Se from R and Vn, the ramp) in numpy."""
    prob, a, meta, kind, par = _case(case)
    dim, p = meta["dim"], meta["p"]
    g = prob.groups[0]
    t = stab_tables(g.shape, g.order, g.ngeo)
    assert t["nq"] > 0
    u = a["u0"][:, 0][a["sol_conn"]]  # [nc, ndof]
    wj = _sensor_weights(t, a, dim)
    s = u @ t["Vn"].T
    r = u @ t["R"].T
    nom, den, vol = (wj * r * r).sum(1), (wj * s * s).sum(1), wj.sum(1)
    Se = np.where(den <= 1e-10, 0.0, nom / np.where(den <= 1e-10, 1.0, den))
    with np.errstate(divide="ignore"):
        se = np.log(Se) / np.log(10.0)
    kappa = float(par[0] if kind != "blend" else par[1])
    blend = kind == "blend"
    factor = 1.0 if blend else float(par[1])
    s0 = 1.0 / p ** 4
    e0 = 1.0 if blend else factor * vol ** (1.0 / dim) / p
    val = np.where(se < s0 - kappa, 0.0, np.where(se > s0 + kappa, e0,
                   0.5 * e0 * (1 + np.sin(np.pi * (se - s0) / (2 * kappa)))))
    ref = a["blend_cell"] if blend else a["av_cell"]
    assert _rel(val, ref) < TOL[dim]


@pytest.mark.parametrize("shape,p", [("triag", 1), ("triag", 2), ("triag", 3), ("tetra", 2)])
def test_vertex_interpolant_matches_oracle(shape, p):
    from pdekit_b200 import meshgen
    from pdekit_b200.reference_element import tet_nodes
    dim = 2 if shape == "triag" else 3
    nodes = meshgen.equidist_triag_nodes(p) if dim == 2 else tet_nodes(p)
    t = stab_tables(shape, p, dim + 1)
    np.testing.assert_allclose(t["P1"], so.p1_at(dim, nodes), atol=1e-15)


def test_fixture_meta_names_its_operator():
    for c in stab_cases():
        meta = json.load(open(os.path.join(GOLDEN, c, "meta.json")))
        assert meta["stab"].split(":")[0] in ("av", "av3d", "blend", "blend3d")


@pytest.mark.parametrize("case", [c for c in stab_cases() if c.endswith("_bonanni")])
def test_host_bonanni_tables_give_reference_values(case):
    """reference_element.bonanni_tables + the kernel's formula in numpy (per cell: Jacobian from
    dVgeo, |K|, the integrals of V and grad p; over the mesh p_min, p_max, v_dom; the clipped
    ratio) against the reference's cellwise coefficient."""
    from pdekit_b200.reference_element import bonanni_tables

    prob, a, meta, kind, par = _case(case)
    dim = meta["dim"]
    g = prob.groups[0]
    t = bonanni_tables(g.shape, g.order, g.ngeo)
    assert t["nq"] > 0
    u = a["u0"]
    rho = u[:, 0]
    V = u[:, 1:1 + dim] / rho[:, None]
    P = (prob.gamma - 1.0) * (u[:, dim + 1] - 0.5 * rho * (V * V).sum(1))
    X = a["geo_coords"][a["geo_conn"]]  # [nc, ngeo, dim]
    J = np.einsum("aqg,cgx->cqax", t["dVgeo"], X)  # [nc, nq, xi, x]
    jw = np.linalg.det(J) * t["w"][None, :]
    gref = np.einsum("aqn,cn->cqa", t["dV"], P[a["sol_conn"]])
    gp = np.linalg.solve(J, gref[..., None])[..., 0]
    vq = np.einsum("qn,cnd->cqd", t["V"], V[a["sol_conn"]])
    vol = jw.sum(1)
    vint = (jw[..., None] * vq).sum(1)
    pint = (jw[..., None] * gp).sum(1)
    vm, gm = vint / vol[:, None], pint / vol[:, None]
    f = (vm * gm).sum(1) * np.sqrt((vm * vm).sum(1))
    vdom = vint.sum(0) / vol.sum()
    pc = P[a["sol_conn"]]
    delta = (pc.max() - pc.min()) * (vdom @ vdom)
    sc = np.maximum(f / delta, 0.0)
    th = np.minimum(1.0, sc * sc * vol ** (1.0 / dim))
    assert _rel(th, a["blend_cell"]) < TOL[dim]


@pytest.mark.parametrize("p", [1, 2, 3])
def test_quad_sensor_table_separates_the_flagged_modes(p):
    """R maps nodal values to the part of u on the modes the reference flags (the first 2p + 1
    of its tensor Legendre basis): a u on the other modes gives R u = 0, a u on the flagged
    modes gives R u = u at the points."""
    from pdekit_b200.reference_element import _legendre_square, quad_nodes
    t = stab_tables("quad", p, 4)
    Tm, flags = _legendre_square(p, quad_nodes(p))
    rng = np.random.default_rng(p)
    c = rng.standard_normal(len(flags))
    kept, flagged = c * ~flags, c * flags
    assert np.abs(t["R"] @ (Tm @ kept)).max() < 1e-12
    np.testing.assert_allclose(t["R"] @ (Tm @ flagged), t["Vn"] @ (Tm @ flagged), atol=1e-12)
    assert flags.sum() == 2 * p + 1 and flags[:2 * p + 1].all()
