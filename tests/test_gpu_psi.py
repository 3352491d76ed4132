"""The PSI scheme on the GPU through the C ABI: the PGN residuals limited by the reference's
residual limiter (src/solver/rdm/cellsplitters/LFResidualLimiter.hpp:37-110) inside the scalar
cell kernels. The reference has no PSI scheme to compare with, so the CUDA path is checked
against the oracle (whose PSI is the limiter restated on its reference-pinned PGN, see
tests/test_psi.py): first assemble, device loop, batched contexts against single ones, and the
refusals."""

import dataclasses
import os

import numpy as np
import pytest

from conftest import GOLDEN
from golden_io import load_golden
from helpers import rel_err
from oracle.rds_oracle import Oracle
from pdekit_b200 import workloads
from pdekit_b200.rds import PGRDMethodExplicit, RDSError

pytestmark = pytest.mark.gpu

TOL = 1e-12  # FP64: summation order only
CASES = ["adv_p1_n", "burgers_p2_n", "burgers_p3_b", "adv_p2_b"]


def _psi(case):
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    return dataclasses.replace(prob, scheme="psi"), a, meta


def _solver(prob, precision="fp64"):
    s = PGRDMethodExplicit(prob.physics, prob.scheme, precision).configure_mesh_data(prob)
    s.initialize_work_data()
    return s


@pytest.mark.parametrize("case", CASES)
def test_psi_matches_oracle(case):
    prob, a, meta = _psi(case)
    o = Oracle(prob)
    s = _solver(prob)
    s.set_solution(a["u0"])
    s.assemble_lhs_and_rhs(meta["cfl"])
    res, dt, ws, vol = s.fields()
    r, w, d, _ = o.assemble(a["u0"], meta["cfl"])
    assert rel_err(res, r) < TOL
    assert rel_err(ws, w) < TOL
    assert rel_err(dt, d) < TOL
    # the limiter changes the residual: PSI differs from PGN somewhere
    n = _solver(dataclasses.replace(prob, scheme="n"))
    n.set_solution(a["u0"])
    n.assemble_lhs_and_rhs(meta["cfl"])
    assert rel_err(n.fields()[0], res) > 1e-6
    n.close()
    s.set_solution(a["u0"])
    it, hist = s.iterate(meta["cfl"], 25)
    uo, no = o.iterate(a["u0"], meta["cfl"], 25)
    assert it == 25
    assert rel_err(s.solution(), uo) < TOL
    np.testing.assert_allclose(hist, no, rtol=1e-11)
    s.close()


def test_psi_batched_equals_single_contexts():
    probs, states, cfls, info = workloads.config5(nprob=6, seed=23, min_cells=100,
                                                  max_cells=3000)
    probs = [dataclasses.replace(p, scheme="psi") for p in probs]
    from pdekit_b200.batch import BatchedRDS

    b = BatchedRDS(probs, cfls, "fp64")
    b.set_solutions(states)
    iters, rel = b.iterate(300, 1e-10, raise_on_cap=False)
    us = b.solutions()
    b.close()
    for i, (p, u0, c) in enumerate(zip(probs, states, cfls)):
        s = _solver(p)
        s.set_solution(u0)
        it, hist = s.iterate(c, 300, 1e-10, raise_on_cap=False)
        assert it == iters[i], (i, info[i])
        assert np.array_equal(s.solution(), us[i]), (i, info[i])
        s.close()


def test_psi_refusals():
    prob, a, meta = _psi("burgers_p2_n")
    with pytest.raises(RDSError):
        _solver(prob, "mixed")
    s = _solver(prob)
    s.set_solution(a["u0"])
    with pytest.raises(RDSError):
        s.element_jacobians(0)
    s.close()
