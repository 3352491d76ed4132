"""Batched independent problems on the GPU against each problem's own single-problem context.

The batch holds the disjoint union of the problems; every node sums its contributions in the
order of its own context, the per-problem norm reduces the same node blocks in the same order
and each problem stops at its own drop, so states, iteration counts and drops must be equal
bit for bit to the single-problem runs (which the parity tests pin to the oracle)."""

import numpy as np
import pytest

from pdekit_b200 import workloads

pytestmark = pytest.mark.gpu

DROP = 1e-10
CAP = 40000


def _single(prob, u0, cfl, precision, max_iter=CAP, drop=DROP):
    from pdekit_b200.rds import PGRDMethodExplicit

    s = PGRDMethodExplicit(prob.physics, prob.scheme, precision).configure_mesh_data(prob)
    s.initialize_work_data()
    s.set_solution(u0)
    it, hist = s.iterate(cfl, max_iter, drop, raise_on_cap=False)
    u = s.solution()
    s.close()
    return it, u, float((hist[-1] / hist[0]).max())


@pytest.fixture(scope="module")
def batch_case():
    return workloads.config5(nprob=10, seed=17, min_cells=100, max_cells=4000)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_single_problem_runs(batch_case, precision):
    from pdekit_b200.batch import BatchedRDS

    probs, states, cfls, info = batch_case
    b = BatchedRDS(probs, cfls, precision)
    b.set_solutions(states)
    iters, rel = b.iterate(CAP, DROP)
    us = b.solutions()
    b.close()
    assert np.all(rel <= DROP)
    for i, (p, u0, c) in enumerate(zip(probs, states, cfls)):
        it, u, r = _single(p, u0, c, precision)
        assert it == iters[i], (i, info[i])
        assert r == rel[i]
        assert np.array_equal(u, us[i]), (i, info[i], np.abs(u - us[i]).max())


def test_batch_autotune_keeps_results(batch_case):
    from pdekit_b200.batch import BatchedRDS

    probs, states, cfls, info = batch_case
    b = BatchedRDS(probs, cfls, "mixed")
    b.set_solutions(states)
    it0, rel0 = b.iterate(CAP, DROP)
    u0 = b.solutions()
    choices = b.autotune()
    assert len(choices) == 2 * len(b.merged.groups)  # FP32 and FP64 kernels of every group
    for c in choices:
        assert c["tile"] in (64, 128, 256) and c["grid"] >= 1 and c["ms"] > 0
    b.set_solutions(states)
    it1, rel1 = b.iterate(CAP, DROP)
    u1 = b.solutions()
    b.close()
    np.testing.assert_array_equal(it0, it1)
    np.testing.assert_array_equal(rel0, rel1)
    for a, c in zip(u0, u1):
        assert np.array_equal(a, c)


def test_batch_iteration_cap(batch_case):
    from pdekit_b200.batch import BatchedRDS
    from pdekit_b200.rds import RDSError

    probs, states, cfls, info = batch_case
    b = BatchedRDS(probs, cfls, "fp64")
    b.set_solutions(states)
    with pytest.raises(RDSError) as e:
        b.iterate(25, DROP)
    assert e.value.status == 5
    b.set_solutions(states)
    iters, rel = b.iterate(25, DROP, raise_on_cap=False)
    us = b.solutions()
    b.close()
    assert np.all(iters == 25)
    for i in (0, len(probs) - 1):
        it, u, r = _single(probs[i], states[i], cfls[i], "fp64", max_iter=25)
        assert it == 25 and np.array_equal(u, us[i])


def test_batch_tensor_core_cells(batch_case):
    """Batched mixed form with the FP32 cells on the tensor cores: every problem reaches the drop
    and its state agrees with the CUDA-core mixed batch to 1e-9 relative L2 (both finish with
    FP64 sweeps)."""
    from pdekit_b200.batch import BatchedRDS

    probs, states, cfls, info = batch_case
    us = {}
    for tc in (0, 1):
        b = BatchedRDS(probs, cfls, "mixed")
        b.set_option("tensor_cores", tc)
        b.set_solutions(states)
        iters, rel = b.iterate(CAP, DROP)
        assert np.all(rel <= DROP)
        us[tc] = b.solutions()
        b.close()
    for u0, u1 in zip(us[0], us[1]):
        assert np.linalg.norm(u1 - u0) <= 1e-9 * np.linalg.norm(u0)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_rk3tvd_equals_single_problem_steps(batch_case, precision):
    """RK3TVD in a batched context: every problem takes three steps with its own CFL through the
    batch's persistent kernels, bit for bit the steps of its own single-problem context (FP64
    stages in both precisions); a later iterate still runs the batch's own loop."""
    from pdekit_b200.batch import BatchedRDS
    from pdekit_b200.rds import PGRDMethodExplicit

    probs, states, cfls, info = batch_case
    b = BatchedRDS(probs, cfls, precision)
    b.set_solutions(states)
    b.advance_rk3tvd(3)
    got = b.solutions()
    for prob, u0, cfl, ub in zip(probs, states, cfls, got):
        s = PGRDMethodExplicit(prob.physics, prob.scheme, "fp64").configure_mesh_data(prob)
        s.initialize_work_data()
        s.set_solution(u0)
        s.advance_rk3tvd(float(cfl), 3)
        assert np.array_equal(s.solution(), ub)
        s.close()
    # the batch's own loop afterwards: as from a batch that never stepped
    b.set_solutions(states)
    it, _ = b.iterate(200, 0.0, raise_on_cap=False)
    u = b.solutions()
    b.close()
    b2 = BatchedRDS(probs, cfls, precision)
    b2.set_solutions(states)
    it2, _ = b2.iterate(200, 0.0, raise_on_cap=False)
    assert np.array_equal(it, it2)
    assert all(np.array_equal(x, y) for x, y in zip(u, b2.solutions()))
    b2.close()
