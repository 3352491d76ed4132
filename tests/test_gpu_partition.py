"""Partitioned single mesh on the GPU: two to four ranks emulated in one process on one GPU
(pdekit_b200.partition.emulate: every rank's phases in turn, the sums over the ranks between
them, so no rank waits for another on the device), against the single-context solver."""

import os

import numpy as np
import pytest

from conftest import GOLDEN
from helpers import rel_err
from pdekit_b200.partition import emulate
from golden_io import load_golden
from pdekit_b200.rds import PGRDMethodExplicit

pytestmark = pytest.mark.gpu


def _single(prob, u0, cfl, iters):
    s = PGRDMethodExplicit(prob.physics, prob.scheme, "fp64").configure_mesh_data(prob)
    s.initialize_work_data()
    s.set_solution(u0)
    _, hist = s.iterate(cfl, iters)
    u = s.solution()
    s.close()
    return u, hist


@pytest.mark.parametrize("case", ["burgers_p2_b", "adv_p2_b", "euler2d_tri_p3_b",
                                  "euler2d_quad_p3_b", "euler3d_tet_p2_lda",
                                  "euler2d_tri_p2_farfield"])
@pytest.mark.parametrize("nparts", [2, 3])
def test_partitioned_matches_single_context(case, nparts):
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    u, norms = emulate(prob, nparts, a["u0"], meta["cfl"], 5)
    u1, hist = _single(prob, a["u0"], meta["cfl"], 5)
    assert rel_err(u, u1) < 1e-12
    np.testing.assert_allclose(norms, hist, rtol=1e-11)


def test_partitioned_larger_mesh_four_ranks():
    from pdekit_b200 import workloads as W

    prob, u0 = W.config2(n=48)
    u, norms = emulate(prob, 4, u0, 0.5, 30)
    u1, hist = _single(prob, u0, 0.5, 30)
    assert rel_err(u, u1) < 1e-11
    np.testing.assert_allclose(norms, hist, rtol=1e-10)


@pytest.mark.parametrize("case", ["burgers_p2_b", "euler2d_tri_p3_b", "euler3d_tet_p2_lda"])
def test_one_rank_graph_steps_match_single_context(case):
    """PartitionedRDS on one rank (no process group): the steps replayed from a CUDA graph, the
    norm summed by the gather's last block (no interface nodes), and steps without the norm's
    sum between them, against the single context."""
    from pdekit_b200.partition import PartitionedRDS

    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    cfl = meta["cfl"]
    u1, hist = _single(prob, a["u0"], cfl, 5)
    pr = PartitionedRDS(prob, 0, 1)
    try:
        pr.set_solution(a["u0"])
        norms = []
        for k in range(5):
            pr.graph_step(cfl, norm=(k % 2 == 0))
            if k % 2 == 0:
                norms.append(pr.norm())
        u = pr.solution_global()
    finally:
        pr.close()
    assert rel_err(u, u1) < 1e-12
    np.testing.assert_allclose(np.array(norms), hist[0::2], rtol=1e-11)
    assert pr.graph_launches > 0


def _single_rk(prob, u0, cfl, nsteps):
    s = PGRDMethodExplicit(prob.physics, prob.scheme, "fp64").configure_mesh_data(prob)
    s.initialize_work_data()
    s.set_solution(u0)
    s.advance_rk3tvd(cfl, nsteps)
    u = s.solution()
    s.close()
    return u


@pytest.mark.parametrize("case", ["burgers_p2_b", "euler2d_tri_p3_b", "euler3d_tet_p2_lda",
                                  "euler2d_tri_p2_farfield"])
@pytest.mark.parametrize("nparts", [2, 3])
def test_partitioned_rk3tvd_matches_single_context(case, nparts):
    """RK3TVD with the exchange in every stage, ranks emulated on one GPU, against the single
    context's device stepper (which the reference's RK3TVD pins)."""
    from pdekit_b200.partition import emulate_rk3tvd

    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    u = emulate_rk3tvd(prob, nparts, a["u0"], meta["cfl"], 2)
    assert rel_err(u, _single_rk(prob, a["u0"], meta["cfl"], 2)) < 1e-12


@pytest.mark.parametrize("case", ["burgers_p2_b", "euler2d_tri_p2_n"])
def test_one_rank_rk3tvd_graph_matches_single_context(case):
    from pdekit_b200.partition import PartitionedRDS

    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    pr = PartitionedRDS(prob, 0, 1)
    try:
        pr.set_solution(a["u0"])
        pr.graph_rk3tvd(meta["cfl"], 3)
        u = pr.solution_global()
    finally:
        pr.close()
    assert rel_err(u, _single_rk(prob, a["u0"], meta["cfl"], 3)) < 1e-13
