"""PGLDA element Jacobians on the GPU (rds_element_jacobians) against the oracle, and the linear
advection identity J u = cell residual (pinned to the reference by the golden cases)."""

import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle.rds_oracle import Oracle
from pdekit_b200.problem import load_golden
from pdekit_b200.rds import PGRDMethodExplicit, RDSError

pytestmark = pytest.mark.gpu


def _jacobians(prob, u, scheme="lda"):
    s = PGRDMethodExplicit(prob.physics, scheme, "fp64").configure_mesh_data(prob)
    s.initialize_work_data()
    s.set_solution(u)
    jac = [s.element_jacobians(ig) for ig in range(len(prob.groups))]
    s.close()
    return jac


@pytest.mark.parametrize("case", ["adv_p1_lda", "adv_p3_lda", "burgers_p2_lda", "burgers_p3_b",
                                  "euler2d_tri_p1_lda", "euler2d_tri_p3_b", "euler2d_quad_p3_b",
                                  "euler3d_tet_p2_lda"])
def test_element_jacobians_match_oracle(case):
    prob, a, _ = load_golden(os.path.join(GOLDEN, case))
    prob.scheme = "lda"
    u = np.asarray(a["u0"])
    jac = _jacobians(prob, u)[0]
    o = Oracle(prob)
    ref = np.stack([o.element_jacobian(0, c, u) for c in range(prob.groups[0].ncells)])
    assert jac.shape == ref.shape
    assert np.abs(jac - ref).max() <= 1e-12 * np.abs(ref).max()


def test_linear_advection_identity_on_gpu():
    prob, a, _ = load_golden(os.path.join(GOLDEN, "adv_p3_lda"))
    u = np.random.default_rng(2).standard_normal((prob.nnodes, 1))
    jac = _jacobians(prob, u)[0]
    o = Oracle(prob)
    g = prob.groups[0]
    for c in range(g.ncells):
        res, _ = o.cell_residual(0, c, u)
        un = u[g.sol_conn[c], 0]
        assert np.abs(jac[c] @ un - res[:, 0]).max() <= 1e-12 * np.abs(jac[c]).max() * 4


@pytest.mark.parametrize("case", ["adv_p1_n", "burgers_p2_n", "euler2d_tri_p2_n",
                                  "euler2d_quad_p3_b", "euler3d_tet_p2_lda"])
def test_n_scheme_element_jacobians_match_oracle(case):
    prob, a, _ = load_golden(os.path.join(GOLDEN, case))
    prob.scheme = "n"
    u = np.asarray(a["u0"])
    jac = _jacobians(prob, u, "n")[0]
    o = Oracle(prob)
    o.model.scheme = 1
    ref = np.stack([o.element_jacobian(0, c, u) for c in range(prob.groups[0].ncells)])
    assert np.abs(jac - ref).max() <= 1e-12 * np.abs(ref).max()


def test_element_jacobians_need_pglda_or_pgn():
    prob, a, _ = load_golden(os.path.join(GOLDEN, "burgers_p2_b"))
    s = PGRDMethodExplicit(prob.physics, "b", "fp64").configure_mesh_data(prob)
    s.initialize_work_data()
    with pytest.raises(RDSError) as e:
        s.element_jacobians(0)
    assert e.value.status == 6
    s.close()
