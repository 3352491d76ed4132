"""Pipelined host-buffer steps (rds_step_host): consecutive calls with different inputs give,
bit for bit, the state and norm of the synchronous sequence set_state, assemble_lhs_and_rhs,
solve, compute_residual_norm, get_state."""

import os

import numpy as np
import pytest

from conftest import GOLDEN
from golden_io import load_golden
from pdekit_b200.rds import PGRDMethodExplicit

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["burgers_p2_b", "euler2d_tri_p3_b", "euler3d_tet_p2_lda"])
def test_pipelined_steps_equal_synchronous_steps(case):
    import torch

    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    cfl, nsteps = meta["cfl"], 5
    u0 = np.asarray(a["u0"], dtype=np.float64).reshape(prob.nnodes, prob.neq)
    rng = np.random.default_rng(1)
    inputs = [u0 * (1.0 + 1e-3 * rng.standard_normal(u0.shape)) for _ in range(nsteps)]

    s = PGRDMethodExplicit(prob.physics, prob.scheme, "fp64").configure_mesh_data(prob)
    s.initialize_work_data()
    ref_u, ref_n = [], []
    for u in inputs:
        s.set_solution(u)
        s.assemble_lhs_and_rhs(cfl)
        s.solve()
        ref_n.append(s.compute_residual_norm())
        ref_u.append(s.solution())

    pin = lambda shape: torch.empty(shape, dtype=torch.float64).pin_memory().numpy()
    ins = [pin(u0.shape) for _ in range(nsteps)]
    outs = [pin(u0.shape) for _ in range(nsteps)]
    norms = [pin((prob.neq,)) for _ in range(nsteps)]
    for i in range(nsteps):
        ins[i][...] = inputs[i]
    for i in range(nsteps):
        s.step_host(ins[i], outs[i], cfl, norms[i])
    s.step_sync()
    for i in range(nsteps):
        assert np.array_equal(outs[i], ref_u[i]), i
        assert np.array_equal(norms[i], ref_n[i]), i
    s.close()


def test_step_host_rejects_wrong_arrays():
    prob, a, meta = load_golden(os.path.join(GOLDEN, "burgers_p2_b"))
    s = PGRDMethodExplicit(prob.physics, prob.scheme, "fp64").configure_mesh_data(prob)
    s.initialize_work_data()
    u = np.zeros((prob.nnodes, prob.neq))
    with pytest.raises(ValueError):
        s.step_host(u[:-1], u.copy(), meta["cfl"])
    with pytest.raises(ValueError):
        s.step_host(u.astype(np.float32), u.copy(), meta["cfl"])
    with pytest.raises(ValueError):
        s.step_host(u, u.copy(), meta["cfl"], np.zeros(prob.neq + 1))
    s.step_sync()
    s.close()
