"""GPU parity through the C ABI: the CUDA path against the reference's golden vectors and the
oracle, on the reference's own meshes, tables and states (tests/golden)."""

import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_cases
from helpers import rel_err
from oracle.rds_oracle import Oracle
from golden_io import load_golden
from pdekit_b200.rds import PGRDMethodExplicit, RDSError

pytestmark = pytest.mark.gpu

TOL = 1e-12  # FP64 plain path: summation order only


def _solver(prob, precision="fp64"):
    s = PGRDMethodExplicit(prob.physics, prob.scheme, precision)
    s.configure_mesh_data(prob)
    s.initialize_work_data()
    return s


@pytest.mark.parametrize("case", golden_cases())
def test_first_assemble_matches_reference(case):
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    s = _solver(prob)
    s.set_solution(a["u0"])
    s.assemble_lhs_and_rhs(meta["cfl"])
    res, dt, ws, vol = s.fields()
    assert rel_err(vol, a["dual_volume"]) < TOL
    assert rel_err(res, a["res1"]) < TOL
    assert rel_err(ws, a["ws1"]) < TOL
    assert rel_err(dt, a["dt1"]) < TOL
    norm = s.compute_residual_norm()
    np.testing.assert_allclose(norm, a["norms"][0], rtol=1e-11)
    s.solve()
    assert rel_err(s.solution(), a["u1"]) < TOL
    s.close()


@pytest.mark.parametrize("case", golden_cases())
def test_device_loop_matches_reference(case):
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    s = _solver(prob)
    s.set_solution(a["u0"])
    it, hist = s.iterate(meta["cfl"], meta["iters"])
    assert it == meta["iters"]
    assert rel_err(s.solution(), a["uK"]) < TOL
    np.testing.assert_allclose(hist, a["norms"], rtol=1e-11)
    s.close()


@pytest.mark.parametrize("case", ["burgers_p2_b", "adv_p1_lda", "euler2d_quad_p3_b",
                                  "euler3d_tet_p2_lda"])
def test_bitwise_repeatable(case):
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    outs = []
    for _ in range(2):
        s = _solver(prob)
        s.set_solution(a["u0"])
        s.iterate(meta["cfl"], 7)
        outs.append(s.solution())
        s.close()
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("case", ["burgers_p2_b", "adv_p1_lda", "adv_p2_b", "burgers_p3_b",
                                  "euler2d_tri_p3_b", "euler2d_quad_p3_b",
                                  "euler3d_tet_p2_lda", "adv_p2_strong", "burgers_p2_strong",
                                  "euler2d_tri_p2_farfield", "euler3d_tet_p2_farfield"])
def test_gpu_matches_oracle_many_iterations(case):
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    s = _solver(prob)
    s.set_solution(a["u0"])
    s.iterate(meta["cfl"], 40)
    u_gpu = s.solution()
    s.close()
    u_ref, _ = Oracle(prob).iterate(a["u0"], meta["cfl"], 40)
    assert rel_err(u_gpu, u_ref) < 1e-11


@pytest.mark.parametrize("case", ["burgers_p2_b", "adv_p1_lda", "euler2d_tri_p3_b",
                                  "euler2d_quad_p3_b", "euler3d_tet_p2_lda"])
def test_mixed_precision_close_to_fp64(case):
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    s = _solver(prob, "mixed")
    s.set_solution(a["u0"])
    s.assemble_lhs_and_rhs(meta["cfl"])
    res, dt, ws, vol = s.fields()
    s.close()
    # FP32 interpolation / flux / upwind terms (Euler residuals are differences of large
    # fluxes, so their relative FP32 error is larger)
    tol = 1e-5 if prob.neq == 1 else 1e-3
    assert rel_err(res, a["res1"]) < tol
    assert rel_err(ws, a["ws1"]) < 1e-5


@pytest.mark.parametrize("which", ["config3_small", "config4_small"])
def test_euler_workloads_match_oracle(which):
    """Mixed P3 triangle + P3 quadrilateral channel (two cell groups, our own tables) and the
    P2 tetrahedral bump box, GPU against the oracle over several iterations."""
    from pdekit_b200 import workloads as W

    prob, u0 = W.config3(6, 8, 4) if which == "config3_small" else W.config4(6, 3, 3)
    s = _solver(prob)
    s.set_solution(u0)
    s.assemble_lhs_and_rhs(0.5)
    res, dt, ws, vol = s.fields()
    o = Oracle(prob)
    r_ref, ws_ref, dt_ref, bad = o.assemble(u0, 0.5)
    assert bad == 0
    assert rel_err(vol, o.vol) < 1e-12
    assert rel_err(res, r_ref) < 1e-11
    assert rel_err(ws, ws_ref) < 1e-12
    s.set_solution(u0)
    s.iterate(0.5, 10)
    u_ref, _ = o.iterate(u0, 0.5, 10)
    assert rel_err(s.solution(), u_ref) < 1e-11
    s.close()


@pytest.mark.parametrize("case,cfl", [("adv_p1_lda_zero", 0.9), ("burgers_p2_n", 0.5)])
def test_mixed_loop_reaches_fp64_solution(case, cfl):
    """Mixed form: FP32 cell kernels down to the switch level, then FP64 sweeps to a 1e-10
    drop; the converged state agrees with the FP64 path's converged state to 1e-9 relative L2."""
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    out = {}
    for prec in ("fp64", "mixed"):
        s = _solver(prob, prec)
        s.set_solution(a["u0"])
        it, hist = s.iterate(cfl, 200000, 1e-10)
        assert (hist[-1] / hist[0]).max() <= 1e-10
        out[prec] = (s.solution(), it)
        s.close()
    u64, um = out["fp64"][0], out["mixed"][0]
    assert np.linalg.norm(um - u64) / np.linalg.norm(u64) < 1e-9


# the tensor-core kernel covers the P1 / 6-point, P2 / 7-point and P3 / 16-point rules
@pytest.mark.parametrize("case", [c for c in golden_cases()
                                  if not c.startswith("euler") and "_q6" not in c])
def test_tensor_core_contraction_matches_fp32_path(case):
    """Mixed form: the cell kernel with the basis contractions on the tensor cores (tcgen05,
    3xTF32 split operands, FP32 accumulation) against the CUDA-core FP32 kernel, on the first
    residual and after 40 iterations (both FP32-level: 2e-6 of the largest magnitude)."""
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    out = {}
    for tc in (0, 1):
        s = _solver(prob, "mixed")
        s.set_option("tensor_cores", tc)
        s.set_solution(a["u0"])
        s.assemble_lhs_and_rhs(meta["cfl"])
        res, dt, ws, vol = s.fields()
        s.set_solution(a["u0"])
        s.kernel_timing(True)
        s.run(meta["cfl"], 40)
        names = set(s.kernel_times())
        s.kernel_timing(False)
        assert any(n.endswith("_tc") for n in names) == bool(tc), names
        out[tc] = (res, ws, s.solution())
        s.close()
    for i in range(3):
        ref, got = out[0][i], out[1][i]
        assert np.abs(got - ref).max() <= 2e-6 * np.abs(ref).max(), (case, i)


def test_tensor_core_bounded_wait_reports_timeout_and_recovers():
    """The tensor-core kernel's bounded mbarrier wait: with the test option each CTA waits a few
    tries on a barrier that nothing completes; the call reports the timeout (RDS_ERR_CUDA, the
    bounded-wait message), TMEM is released, and the context then runs as a fresh one."""
    prob, a, meta = load_golden(os.path.join(GOLDEN, "burgers_p2_b"))
    cfl = meta["cfl"]
    s = _solver(prob, "mixed")
    s.set_option("tensor_cores", 1)
    s.set_option("tc_test_wait", 64)
    s.set_solution(a["u0"])
    s.run(cfl, 2)
    with pytest.raises(RDSError) as err:
        s.check()
    assert err.value.status == 2 and "bounded device wait" in str(err.value)
    s.set_option("tc_test_wait", 0)
    s.set_solution(a["u0"])
    s.iterate(cfl, 1, 0.0)  # clears the status word
    s.set_solution(a["u0"])
    s.run(cfl, 3)
    s.check()
    u = s.solution()
    s.close()
    f = _solver(prob, "mixed")
    f.set_option("tensor_cores", 1)
    f.set_solution(a["u0"])
    f.run(cfl, 3)
    assert np.array_equal(u, f.solution())
    f.close()
