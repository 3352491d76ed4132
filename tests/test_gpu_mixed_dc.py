"""Mixed form, scalar physics: the defect-correction loop on the GPU.

Cycles of one exact FP64 sweep and m - 1 FP32 correction sweeps (rds_cells_scalar_dc.cu and the
gather modes 18 / 19), checked against the FP64 path and the numpy restatement
oracle/dc_oracle.py."""

import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_cases
from golden_io import load_golden
from helpers import rel_err
from oracle.dc_oracle import dc_iterate
from pdekit_b200.rds import PGRDMethodExplicit

pytestmark = pytest.mark.gpu

SCALAR = [c for c in golden_cases() if c.startswith(("adv", "burgers"))]


def _solver(prob, precision, m=None):
    s = PGRDMethodExplicit(prob.physics, prob.scheme, precision)
    s.configure_mesh_data(prob)
    s.initialize_work_data()
    if m is not None:
        s.set_option("mixed_refresh", m)
    return s


@pytest.mark.parametrize("case", ["adv_p1_lda", "burgers_p2_b", "burgers_p3_b", "adv_p2_strong"])
def test_one_sweep_cycles_equal_the_fp64_loop(case):
    """m = 1: every sweep is exact, and the states equal the FP64 loop's bit for bit."""
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    out = []
    for prec, m in (("fp64", None), ("mixed", 1)):
        s = _solver(prob, prec, m)
        s.set_solution(a["u0"])
        it, hist = s.iterate(meta["cfl"], 9)
        assert it == 9
        out.append((s.solution(), hist))
        s.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("case", SCALAR)
def test_correction_sweeps_match_restatement(case):
    """Three cycles of m = 4 (exact sweeps 0, 4, 8; FP32 corrections between) against the FP64
    restatement of the same loop: the FP32 corrections agree to FP32 accuracy relative to the
    change of the state."""
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    s = _solver(prob, "mixed", 4)
    s.set_solution(a["u0"])
    it, _ = s.iterate(meta["cfl"], 9)
    assert it == 9
    u = s.solution()
    s.close()
    u_ref = dc_iterate(prob, a["u0"], meta["cfl"], 4, 9)
    assert rel_err(u - a["u0"], u_ref - a["u0"]) < 2e-6


@pytest.mark.parametrize("case,cfl", [("adv_p1_lda_zero", 0.9), ("burgers_p2_n", 0.5),
                                      ("adv_p2_b", 0.9), ("adv_p3_lda", 0.9)])
@pytest.mark.parametrize("m", [4, 8, 16])
def test_loop_reaches_the_fp64_solution(case, cfl, m):
    """To a 1e-10 drop: the converged state within 1e-9 relative L2 of the FP64 loop's, at most
    1.25x its sweeps; the history holds the exact norms (repeated over the correction sweeps)."""
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    out = {}
    for prec in ("fp64", "mixed"):
        s = _solver(prob, prec, m if prec == "mixed" else None)
        s.set_solution(a["u0"])
        it, hist = s.iterate(cfl, 400000, 1e-10)
        assert (hist[-1] / hist[0]).max() <= 1e-10
        out[prec] = (s.solution(), it, hist)
        s.close()
    (u64, it64, _), (um, itm, hm) = out["fp64"], out["mixed"]
    assert np.linalg.norm(um - u64) / np.linalg.norm(u64) < 1e-9
    assert itm <= 1.25 * it64 + m, (itm, it64)
    assert len(hm) == itm
    assert np.array_equal(hm[1:m], np.repeat(hm[:1], m - 1, axis=0))
