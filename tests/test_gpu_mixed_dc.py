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


FUSABLE = [c for c in SCALAR if "strong" not in c]


@pytest.mark.parametrize("case", FUSABLE)
@pytest.mark.parametrize("m", [4, 24])
def test_fused_correction_sweeps_equal_separate_launches(case, m):
    """The correction sweeps of a cycle in one launch (dc_sweeps_fused, the default on these
    small meshes) against one launch per kernel and sweep: states and exact-sweep norms equal
    bit for bit, including a run that stops inside a cycle."""
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    out = []
    for fuse in (0, 1 << 16):
        s = _solver(prob, "mixed", m)
        s.set_option("mixed_fuse_cells", fuse)
        s.set_solution(a["u0"])
        it, hist = s.iterate(meta["cfl"], 3 * m + 5)
        out.append((it, s.solution(), hist))
        s.close()
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])


def test_fused_barrier_bounded_wait_reports_timeout_and_recovers():
    """With the test option every barrier of the fused sweeps waits for one block more than the
    grid holds: each wait gives up after the given polls, the call reports RDS_ERR_CUDA with the
    bounded-wait message, and the context then runs as a fresh one."""
    from pdekit_b200.rds import RDSError
    prob, a, meta = load_golden(os.path.join(GOLDEN, "burgers_p2_n"))
    s = _solver(prob, "mixed", 8)
    s.set_solution(a["u0"])
    s.set_option("fuse_test_wait", 200)
    with pytest.raises(RDSError) as err:
        s.iterate(meta["cfl"], 16)
    assert err.value.status == 2 and "bounded device wait" in str(err.value)
    s.set_option("fuse_test_wait", 0)
    s.set_solution(a["u0"])
    it, hist = s.iterate(meta["cfl"], 16)
    u = s.solution()
    s.close()
    f = _solver(prob, "mixed", 8)
    f.set_solution(a["u0"])
    it2, hist2 = f.iterate(meta["cfl"], 16)
    assert it == it2 and np.array_equal(u, f.solution()) and np.array_equal(hist, hist2)
    f.close()
