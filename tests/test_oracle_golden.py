"""The C restatement (oracle/rds_oracle.c) against golden vectors produced by the reference
itself (tests/golden, written by tests/golden/make_golden.py through oracle/ref_harness.cpp)."""

import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_cases
from helpers import rel_err
from oracle.rds_oracle import Oracle
from golden_io import load_golden

TOL = 1e-12  # FP64, summation-order differences only


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_first_assemble(case):
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    o = Oracle(prob)
    assert rel_err(o.vol, a["dual_volume"]) < TOL
    res, ws, dt, bad = o.assemble(a["u0"], meta["cfl"])
    assert bad == 0
    assert rel_err(res, a["res1"]) < TOL
    assert rel_err(ws, a["ws1"]) < TOL
    assert rel_err(dt, a["dt1"]) < TOL


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_iterations(case):
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    o = Oracle(prob)
    u1, _ = o.iterate(a["u0"], meta["cfl"], 1)
    assert rel_err(u1, a["u1"]) < TOL
    uk, norms = o.iterate(a["u0"], meta["cfl"], meta["iters"])
    assert rel_err(uk, a["uK"]) < TOL
    np.testing.assert_allclose(norms, a["norms"], rtol=1e-11, atol=0)


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_rk3tvd(case):
    """Two steps of the third-order TVD Runge-Kutta stepper against the reference's own
    RK3TVD class run on the same solver (state, first-stage residual and dt, norms)."""
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    o = Oracle(prob)
    u, res, dt, norms = o.rk3tvd(a["u0"], meta["cfl"], 2)
    assert rel_err(u, a["u_rk3"]) < TOL
    assert rel_err(res, a["res_rk3"]) < TOL
    assert rel_err(dt, a["dt_rk3"]) < TOL
    np.testing.assert_allclose(norms, a["norms_rk3"], rtol=1e-11, atol=0)


def test_oracle_detects_planted_error():
    """A mistake planted in the oracle's inputs (one wrong table entry) must be caught."""
    prob, a, meta = load_golden(os.path.join(GOLDEN, "burgers_p2_b"))
    prob.groups[0].dVf[0, 0, 0] += 1e-6
    o = Oracle(prob)
    res, _, _, _ = o.assemble(a["u0"], meta["cfl"])
    assert rel_err(res, a["res1"]) > 1e-9
