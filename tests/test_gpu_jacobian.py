"""PGLDA / PGN / PGB element Jacobians on the GPU (rds_element_jacobians) and their block-CSR assembly
(rds_jacobian_pattern, rds_assemble_jacobian) against the oracle, and the linear advection
identity J u = cell residual (pinned to the reference by the golden cases)."""

import ctypes as C
import dataclasses
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle.rds_oracle import Oracle
from golden_io import load_golden
from pdekit_b200.rds import PGRDMethodExplicit, RDSError, lib

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


@pytest.mark.parametrize("case", ["adv_p2_b", "burgers_p2_b", "euler2d_tri_p3_b",
                                  "euler2d_quad_p3_b", "euler3d_tet_p2_lda"])
def test_pgb_element_jacobians_match_oracle(case):
    prob, a, _ = load_golden(os.path.join(GOLDEN, case))
    prob.scheme = "b"
    u = np.asarray(a["u0"])
    jac = _jacobians(prob, u, "b")[0]
    o = Oracle(prob)
    o.model.scheme = 2
    ref = np.stack([o.element_jacobian(0, c, u) for c in range(prob.groups[0].ncells)])
    assert np.abs(jac - ref).max() <= 1e-12 * np.abs(ref).max()


def test_element_jacobians_not_in_batched_contexts():
    from pdekit_b200.batch import BatchedRDS

    prob, a, _ = load_golden(os.path.join(GOLDEN, "adv_p1_lda"))
    b = BatchedRDS([prob, prob], np.array([0.9, 0.9]))
    jac = torch_empty(prob.groups[0].ncells * 2 * 9)
    st = lib().rds_element_jacobians(b._ctx, 0, C.c_void_p(jac.data_ptr()))
    assert st == 6
    b.close()


def torch_empty(n):
    import torch

    return torch.empty(n, dtype=torch.float64, device="cuda")


def _dense(row_ptr, col_idx, vals, n, neq):
    A = np.zeros((n * neq, n * neq))
    for v in range(n):
        for k in range(row_ptr[v], row_ptr[v + 1]):
            w = col_idx[k]
            A[v * neq:(v + 1) * neq, w * neq:(w + 1) * neq] = vals[k]
    return A


def _assembled(prob, u, scheme):
    s = PGRDMethodExplicit(prob.physics, scheme, "fp64").configure_mesh_data(prob)
    s.initialize_work_data()
    s.set_solution(u)
    out = s.assemble_jacobian()
    s.close()
    return out


@pytest.mark.parametrize("case,scheme", [("adv_p2_b", "lda"), ("burgers_p2_n", "n"),
                                         ("euler2d_tri_p1_lda", "lda"),
                                         ("euler3d_tet_p2_lda", "n"), ("burgers_p2_b", "b")])
def test_assembled_jacobian_matches_oracle_elements(case, scheme):
    prob, a, _ = load_golden(os.path.join(GOLDEN, case))
    prob.scheme = scheme
    u = np.asarray(a["u0"])
    row_ptr, col_idx, vals = _assembled(prob, u, scheme)
    n, neq = prob.nnodes, prob.neq
    assert row_ptr[0] == 0 and row_ptr[-1] == len(col_idx)
    for v in range(n):
        cols = col_idx[row_ptr[v]:row_ptr[v + 1]]
        assert np.all(np.diff(cols) > 0) and v in cols
    o = Oracle(prob)
    o.model.scheme = {"lda": 0, "n": 1, "b": 2}[scheme]
    g = prob.groups[0]
    ref = np.zeros((n * neq, n * neq))
    for c in range(g.ncells):
        jac = o.element_jacobian(0, c, u)
        d = g.sol_conn[c]
        for m in range(g.ndof):
            for k in range(g.ndof):
                ref[d[m] * neq:(d[m] + 1) * neq, d[k] * neq:(d[k] + 1) * neq] += \
                    jac[m * neq:(m + 1) * neq, k * neq:(k + 1) * neq] / o.vol[d[m]]
    A = _dense(row_ptr, col_idx, vals, n, neq)
    assert np.abs(A - ref).max() <= 1e-12 * np.abs(ref).max()


def test_assembled_advection_jacobian_applies_the_cell_residual():
    """For constant advection (PGLDA) the assembled operator times the state is the nodal
    residual of the cells (the golden cases pin that residual to the reference)."""
    prob, a, meta = load_golden(os.path.join(GOLDEN, "adv_p3_lda"))
    u = np.random.default_rng(4).standard_normal((prob.nnodes, 1))
    row_ptr, col_idx, vals = _assembled(prob, u, "lda")
    A = _dense(row_ptr, col_idx, vals, prob.nnodes, 1)
    cells_only = dataclasses.replace(prob, bcs=[])
    res, _, _, _ = Oracle(cells_only).assemble(u, meta["cfl"])
    assert np.abs(A @ u[:, 0] - res[:, 0]).max() <= 1e-12 * np.abs(A).max() * np.abs(u).max() * 8


JAC_CASES = ["burgers_p2_lda", "burgers_p2_n", "burgers_p2_b", "burgers_p3_b", "adv_p2_b",
             "euler2d_tri_p1_lda", "euler2d_tri_p2_n", "euler2d_tri_p3_b", "euler2d_quad_p3_b",
             "euler3d_tet_p2_lda"]


@pytest.mark.parametrize("case", JAC_CASES)
def test_assembled_jacobian_matches_reference(case):
    """The block-CSR assembly on the GPU against the reference's own Picard-Jacobian cell worker
    (PGRDMPicardJacCellAssemblyWorker: compute_adv_res_and_jacobian of PGLDA / PGN / PGB, entry
    J(m, n) / V(m)), dumped at u0 with the golden case."""
    prob, a, _ = load_golden(os.path.join(GOLDEN, case))
    row_ptr, col_idx, vals = _assembled(prob, np.asarray(a["u0"]), prob.scheme)
    n, neq = prob.nnodes, prob.neq
    A = _dense(row_ptr, col_idx, vals, n, neq)
    ref = np.zeros_like(A)
    ref[a["jac_row"], a["jac_col"]] = a["jac_val"]
    assert np.abs(A - ref).max() <= 1e-12 * np.abs(ref).max()
