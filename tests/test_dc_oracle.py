"""The numpy restatement of the mixed form's defect-correction loop (oracle/dc_oracle.py), the
checker of its CUDA kernels, against the C restatement that the golden cases pin to the
reference (CPU only)."""

import dataclasses
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_cases
from golden_io import load_golden
from helpers import rel_err
from oracle.dc_oracle import ScalarCells, dc_iterate
from oracle.rds_oracle import Oracle

SCALAR = [c for c in golden_cases() if c.startswith(("adv", "burgers"))]


@pytest.mark.parametrize("case", SCALAR)
def test_cell_residual_matches_c_restatement(case):
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    cells_only = Oracle(dataclasses.replace(prob, bcs=[]))
    ref = cells_only.assemble(a["u0"], meta["cfl"])[0]
    sc = ScalarCells(prob)
    got = sc.nodal(sc.residual(a["u0"][:, 0])[0], cells_only.vol)
    assert rel_err(got, ref[:, 0]) < 1e-12


@pytest.mark.parametrize("case", ["adv_p1_lda", "adv_p1_n", "adv_p2_b", "adv_p3_lda"])
def test_change_is_exact_for_linear_schemes(case):
    """Advection: the coefficients do not depend on u, so the frozen-coefficient change is the
    exact change of the residual (PGB: with theta of the reference state on both sides)."""
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    sc = ScalarCells(prob)
    ur = a["u0"][:, 0]
    d = 1e-3 * np.sin(17.0 * np.arange(ur.size))
    r0, theta = sc.residual(ur)
    r1 = sc.residual(ur + d)[0]
    got = sc.delta(ur, d, theta)
    if prob.scheme == "b":
        # PGB blends with theta(u): compare the LDA + theta_r N parts of both states
        p = dataclasses.replace(prob, scheme="n")
        sl, sn = ScalarCells(dataclasses.replace(prob, scheme="lda")), ScalarCells(p)
        lda = sl.residual(ur + d)[0] - sl.residual(ur)[0]
        nn = sn.residual(ur + d)[0] - sn.residual(ur)[0]
        ref = lda + theta[:, None] * (nn - lda)
    else:
        ref = r1 - r0
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("case", ["adv_p1_lda", "burgers_p2_b", "adv_p2_strong"])
def test_one_sweep_cycles_are_the_fp64_iteration(case):
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    u_ref, _ = Oracle(prob).iterate(a["u0"], meta["cfl"], 6)
    u = dc_iterate(prob, a["u0"], meta["cfl"], 1, 6)
    assert rel_err(u, u_ref) < 1e-14


@pytest.mark.parametrize("case,cfl,m", [("adv_p1_lda_zero", 0.9, 8), ("burgers_p2_n", 0.5, 8)])
def test_loop_converges_to_the_fp64_fixed_point(case, cfl, m):
    """Run far enough, the correction cycles reach the FP64 scheme's steady state."""
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    o = Oracle(prob)
    u64, _ = o.iterate(a["u0"], cfl, 3000)
    u = dc_iterate(prob, a["u0"], cfl, m, 3000 + 1)
    res = o.assemble(u, cfl)[0]
    res0 = o.assemble(a["u0"], cfl)[0]
    assert np.abs(res).max() <= 1e-9 * np.abs(res0).max()
    assert np.linalg.norm(u - u64) / np.linalg.norm(u64) < 1e-9
