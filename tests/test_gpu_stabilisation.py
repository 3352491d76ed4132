"""Stabilisation on the GPU, through the C ABI, against the reference's own outputs
(tests/golden/*_av, *_lf, *_wj, *_visc): the operators (sensor, normalised indicator,
blending coefficients, cell-to-node transfer) on the reference's state, the residual with the
reference's nodal field handed to the solver (PGLDA artificial viscosity, PGB external
blending coefficient) for the first assemble and the device loop, and the whole chain on the
device (operator -> installed field -> residual)."""

import os

import numpy as np
import pytest

from conftest import GOLDEN, stab_cases
from helpers import rel_err
from golden_io import load_golden
from pdekit_b200.rds import PGRDMethodExplicit, RDSError
from pdekit_b200.stabilisation import ArtificialViscosity, RDBlendingCoeff

pytestmark = pytest.mark.gpu

TOL = 1e-12            # FP64: summation order only
TOL_OP = {2: 1e-12, 3: 1e-8}  # the reference's order-4 tetrahedron rule has ~10 digits


def _setup(case):
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    s = PGRDMethodExplicit(prob.physics, prob.scheme, "fp64").configure_mesh_data(prob)
    s.initialize_work_data()
    s.set_solution(a["u0"])
    kind, *par = meta["stab"].split(":")
    return prob, a, meta, s, kind, par


def _rel(got, ref):
    return np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-300)


@pytest.mark.parametrize("case", stab_cases())
def test_operators_match_reference(case):
    prob, a, meta, s, kind, par = _setup(case)
    tol = TOL_OP[meta["dim"]]
    if kind.startswith("av"):
        kappa, factor = float(par[0]), float(par[1])
        op = ArtificialViscosity().prepare_indicator_operators(s)
        assert _rel(op.compute_artificial_viscosity(kappa=kappa, factor=factor), a["av_cell"]) < tol
        assert _rel(op.compute_indicator_normalized(kappa=kappa), a["indicator"]) < tol * 100
        nod = op.compute_artificial_viscosity_nodal(kappa=kappa, factor=factor, install=False)
        # 2D: the reference's transfer; 3D: the oracle's (the reference's crashes there)
        assert _rel(nod, a["av_nodal"]) < tol
    else:
        typ, prm = par[0], float(par[1])
        op = RDBlendingCoeff().setup(s, typ)
        op.set_param("u_inf" if typ == "WongJansen" else "kappa", prm)
        assert _rel(op.calculate_in_cells(), a["blend_cell"]) < tol
        assert _rel(op.calculate(install=False), a["blend_nodal"]) < tol
    s.close()


def _install_reference_field(s, a, kind):
    if kind.startswith("av"):
        s.set_artificial_viscosity(a["av_nodal"])
    else:
        s.set_blending_coeff(a["blend_nodal"])


@pytest.mark.parametrize("case", stab_cases())
def test_residual_with_field_matches_reference(case):
    prob, a, meta, s, kind, par = _setup(case)
    _install_reference_field(s, a, kind)
    s.assemble_lhs_and_rhs(meta["cfl"])
    res, dt, ws, vol = s.fields()
    assert rel_err(res, a["res1"]) < TOL
    assert rel_err(ws, a["ws1"]) < TOL
    assert rel_err(dt, a["dt1"]) < TOL
    np.testing.assert_allclose(s.compute_residual_norm(), a["norms"][0], rtol=1e-11)
    s.solve()
    assert rel_err(s.solution(), a["u1"]) < TOL
    s.close()


@pytest.mark.parametrize("case", stab_cases())
def test_device_loop_with_field_matches_reference(case):
    prob, a, meta, s, kind, par = _setup(case)
    _install_reference_field(s, a, kind)
    it, hist = s.iterate(meta["cfl"], meta["iters"])
    assert it == meta["iters"]
    assert rel_err(s.solution(), a["uK"]) < TOL
    np.testing.assert_allclose(hist, a["norms"], rtol=1e-11)
    s.close()


@pytest.mark.parametrize("case", [c for c in stab_cases() if "3d" not in c])
def test_field_computed_on_device_gives_reference_residual(case):
    """The reference's example chain (operator at u0, field handed to the solver, assemble)
    entirely on the device."""
    prob, a, meta, s, kind, par = _setup(case)
    if kind == "av":
        ArtificialViscosity().prepare_indicator_operators(s).compute_artificial_viscosity_nodal(
            kappa=float(par[0]), factor=float(par[1]), install=True)
    else:
        op = RDBlendingCoeff().setup(s, par[0])
        op.set_param("u_inf" if par[0] == "WongJansen" else "kappa", float(par[1]))
        op.calculate(install=True)
    s.assemble_lhs_and_rhs(meta["cfl"])
    res, _, _, _ = s.fields()
    assert rel_err(res, a["res1"]) < TOL
    s.close()


def test_removing_the_field_restores_the_plain_residual():
    prob, a, meta, s, kind, par = _setup("burgers_p2_b_lf")
    s.assemble_lhs_and_rhs(meta["cfl"])
    plain = s.fields()[0]
    s.set_blending_coeff(a["blend_nodal"])
    s.iterate(meta["cfl"], 2)          # captured loop with the field
    s.set_solution(a["u0"])
    s.set_blending_coeff(None)
    s.assemble_lhs_and_rhs(meta["cfl"])
    assert np.array_equal(s.fields()[0], plain)
    s.close()


@pytest.mark.parametrize("case,p", [("euler2d_quad_p2_b_bonanni", 2), ("euler2d_quad_p3_b", 3)])
def test_quad_sensor_above_p1_matches_oracle(case, p):
    """Quadrilaterals of order >= 2 (the reference's value follows the rounding of a singular
    mass matrix there): the device sensor against the oracle's regular projection, detJ per
    point on the fixture's bilinear cells."""
    from oracle import stab_oracle as so
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    s = PGRDMethodExplicit(prob.physics, prob.scheme, "fp64").configure_mesh_data(prob)
    s.initialize_work_data()
    s.set_solution(a["u0"])
    op = ArtificialViscosity().prepare_indicator_operators(s)
    for kappa in (0.5, 4.0):
        ref = so.sensor_cells(2, p, a["sol_nodes"], a["geo_coords"], a["geo_conn"],
                              a["sol_conn"], a["u0"][:, 0], kappa, 1.3)
        assert _rel(op.compute_artificial_viscosity(kappa=kappa, factor=1.3), ref) < TOL
    b = RDBlendingCoeff().setup(s, "ViscosityIndicator")
    b.set_param("kappa", 2.0)
    ref = so.sensor_cells(2, p, a["sol_nodes"], a["geo_coords"], a["geo_conn"], a["sol_conn"],
                          a["u0"][:, 0], 2.0, blend=True)
    assert _rel(b.calculate_in_cells(), ref) < TOL
    s.close()


def test_refusals(monkeypatch):
    # the sensor on quadrilaterals needs the geometry tables at its points
    from pdekit_b200 import reference_element as R
    tables = R.stab_tables
    monkeypatch.setattr(R, "stab_tables", lambda *k: {n: v for n, v in tables(*k).items()
                                                       if n != "dVgeo"})
    prob, a, meta = load_golden(os.path.join(GOLDEN, "euler2d_quad_p3_b"))
    s = PGRDMethodExplicit(prob.physics, prob.scheme, "fp64").configure_mesh_data(prob)
    s.initialize_work_data()
    s.set_solution(a["u0"])
    with pytest.raises(RDSError):
        ArtificialViscosity().prepare_indicator_operators(s).compute_artificial_viscosity()
    # LF_Blend works on quadrilaterals (Q1 vertex interpolant for the nodal field)
    nod = RDBlendingCoeff().setup(s, "LF_Blend").calculate(install=True)
    assert nod.shape == (prob.nnodes,) and np.isfinite(nod).all()
    # PGB element Jacobians with an external blending coefficient are not provided
    with pytest.raises(RDSError):
        s.element_jacobians(0)
    with pytest.raises(ValueError):
        s.set_artificial_viscosity(np.zeros(prob.nnodes + 1))
    s.close()
