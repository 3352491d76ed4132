"""Third-order TVD Runge-Kutta stepping on the GPU (rds_advance_rk3tvd through the C ABI)
against the reference's own RK3TVD class (solver/time/ExplicitTimeStepper.cpp:66-100) run on
the same solver, meshes, tables and states (tests/golden: u_rk3, res_rk3, dt_rk3, norms_rk3)."""

import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_cases
from helpers import rel_err
from oracle.rds_oracle import Oracle
from golden_io import load_golden
from pdekit_b200.rds import RK3TVD, PGRDMethodExplicit, RDSError

pytestmark = pytest.mark.gpu

TOL = 1e-12  # FP64: summation order only


def _solver(prob, precision="fp64"):
    s = PGRDMethodExplicit(prob.physics, prob.scheme, precision)
    s.configure_mesh_data(prob)
    s.initialize_work_data()
    return s


@pytest.mark.parametrize("case", golden_cases())
def test_rk3tvd_matches_reference(case):
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    s = _solver(prob)
    s.set_solution(a["u0"])
    rk3 = RK3TVD()
    rk3.setup(prob.neq, prob.nnodes)
    for step in range(2):
        rk3.advance_in_time(s, meta["cfl"])
        np.testing.assert_allclose(s.compute_residual_norm(), a["norms_rk3"][step], rtol=1e-11)
    assert rel_err(s.solution(), a["u_rk3"]) < TOL
    res, dt, _, _ = s.fields()
    assert rel_err(res, a["res_rk3"]) < TOL
    assert rel_err(dt, a["dt_rk3"]) < TOL
    s.close()


@pytest.mark.parametrize("case", ["burgers_p2_b", "adv_p2_strong", "euler2d_quad_p3_b",
                                  "euler3d_tet_p2_farfield"])
def test_rk3tvd_graph_replay_bitwise(case):
    """Several steps in one call (graph replays) equal the same steps one call at a time, and
    equal the oracle's restatement over three steps."""
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    s1, s2 = _solver(prob), _solver(prob)
    s1.set_solution(a["u0"])
    s2.set_solution(a["u0"])
    s1.advance_rk3tvd(meta["cfl"], 3)
    for _ in range(3):
        s2.advance_rk3tvd(meta["cfl"], 1)
    assert np.array_equal(s1.solution(), s2.solution())
    assert np.array_equal(s1.fields()[0], s2.fields()[0])
    u, res, dt, _ = Oracle(prob).rk3tvd(a["u0"], meta["cfl"], 3)
    assert rel_err(s1.solution(), u) < TOL
    assert rel_err(s1.fields()[0], res) < TOL
    s1.close()
    s2.close()


def test_rk3tvd_cfl_change_recaptures():
    """A second CFL value is honoured (the captured step is rebuilt, not replayed)."""
    prob, a, meta = load_golden(os.path.join(GOLDEN, "burgers_p2_b"))
    s = _solver(prob)
    s.set_solution(a["u0"])
    s.advance_rk3tvd(meta["cfl"], 1)
    s.advance_rk3tvd(0.25, 1)
    o = Oracle(prob)
    u, _, _, _ = o.rk3tvd(a["u0"], meta["cfl"], 1)
    u, _, dt, _ = o.rk3tvd(u, 0.25, 1)
    assert rel_err(s.solution(), u) < TOL
    assert rel_err(s.fields()[1], dt) < TOL
    s.close()


@pytest.mark.parametrize("case", ["burgers_p2_b", "euler2d_tri_p2_n"])
def test_rk3tvd_in_mixed_context_runs_fp64_stages(case):
    """A mixed context's RK3TVD steps run the FP64 cell kernels: the same bits as an FP64
    context's, and the oracle's steps to the usual tolerance."""
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    sm, sd = _solver(prob, "mixed"), _solver(prob)
    for s in (sm, sd):
        s.set_solution(a["u0"])
        s.advance_rk3tvd(meta["cfl"], 2)
    assert np.array_equal(sm.solution(), sd.solution())
    assert np.array_equal(sm.fields()[0], sd.fields()[0])
    u, _, _, _ = Oracle(prob).rk3tvd(a["u0"], meta["cfl"], 2)
    assert rel_err(sm.solution(), u) < TOL
    # the context's own loop still runs in its precision afterwards
    sm.set_solution(a["u0"])
    sm.iterate(meta["cfl"], 3, 0.0)
    sm.close()
    sd.close()
