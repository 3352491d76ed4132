"""PGLDA element Jacobians of the oracle (oracle/rds_oracle.c rdso_element_jacobian, the
restatement of PGLDA.hpp:316-536), pinned through the reference's residual: for constant
advection the flux interpolant is exact, so J u equals the cell's scheme residual, which the
golden cases pin to the reference itself."""

import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle.rds_oracle import Oracle
from golden_io import load_golden


@pytest.mark.parametrize("case", ["adv_p1_lda", "adv_p1_lda_zero", "adv_p3_lda", "adv_p2_b"])
def test_linear_advection_jacobian_reproduces_residual(case):
    prob, a, _ = load_golden(os.path.join(GOLDEN, case))
    prob.scheme = "lda"
    o = Oracle(prob)
    o.model.scheme = 0  # PGLDA residual for the comparison
    g = prob.groups[0]
    rng = np.random.default_rng(5)
    for u in (np.asarray(a["u0"]), rng.standard_normal((prob.nnodes, 1))):
        worst = 0.0
        for c in range(g.ncells):
            jac = o.element_jacobian(0, c, u)
            res, _ = o.cell_residual(0, c, u)
            un = u.reshape(-1, 1)[g.sol_conn[c]].ravel()
            scale = max(np.abs(res).max(), np.abs(jac).max() * np.abs(un).max())
            diff = np.abs(jac @ un - res.ravel()).max()
            worst = max(worst, diff / scale if scale > 0 else diff)
        assert worst < 1e-13


def test_jacobian_annihilates_constant_states():
    """sum_n grad phi_n = 0, so J maps a constant state to zero (Burgers, Euler)."""
    for case in ("burgers_p2_lda", "euler2d_tri_p1_lda", "euler3d_tet_p2_lda"):
        prob, a, _ = load_golden(os.path.join(GOLDEN, case))
        o = Oracle(prob)
        g = prob.groups[0]
        u = np.asarray(a["u0"]).reshape(-1, prob.neq)
        const = np.tile(u[0], g.ndof)
        jac = o.element_jacobian(0, 0, np.tile(u[0], (prob.nnodes, 1)))
        assert np.abs(jac @ const).max() <= 1e-10 * np.abs(jac).max() * np.abs(const).max()


@pytest.mark.parametrize("case", ["adv_p1_n", "adv_p2_b"])
def test_n_scheme_jacobian_is_the_n_residual_operator(case):
    """Implicit PGN (the plain N scheme): J u equals sum_q w |J| sum_{n != m} K+_m (sum K-)^-1
    K-_n (u_m - u_n), evaluated here from the same frozen upwind coefficients; and J has zero
    row sums (constant states give no residual)."""
    prob, a, _ = load_golden(os.path.join(GOLDEN, case))
    prob.scheme = "n"
    o = Oracle(prob)
    o.model.scheme = 1
    g = prob.groups[0]
    u = np.asarray(a["u0"]).reshape(-1)
    for c in range(g.ncells):
        jac = o.element_jacobian(0, c, u)
        assert np.abs(jac.sum(axis=1)).max() <= 1e-13 * np.abs(jac).max()
        # J u with u_m - u_n differences: sum_n J_mn u_n = sum_n J_mn (u_n - u_m) since rows sum
        # to zero, i.e. only differences of the state enter, as in the N scheme
        un = u[g.sol_conn[c]]
        d = jac @ un - np.array([jac[mm] @ (un - un[mm]) for mm in range(g.ndof)])
        assert np.abs(d).max() <= 1e-12 * max(np.abs(jac).max() * np.abs(un).max(), 1e-300)


@pytest.mark.parametrize("case", ["adv_p2_b", "adv_p1_lda"])
def test_pgb_jacobian_reproduces_the_pgb_residual(case):
    """PGB for constant advection: J(u) u = the blended residual (LDA part plus theta times the
    N part, theta frozen at u); the golden case adv_p2_b pins that residual to the reference."""
    prob, a, _ = load_golden(os.path.join(GOLDEN, case))
    prob.scheme = "b"
    o = Oracle(prob)
    o.model.scheme = 2
    g = prob.groups[0]
    rng = np.random.default_rng(7)
    for u in (np.asarray(a["u0"]).reshape(-1), rng.standard_normal(prob.nnodes)):
        for c in range(g.ncells):
            jac = o.element_jacobian(0, c, u)
            res, _ = o.cell_residual(0, c, u)
            un = u[g.sol_conn[c]]
            scale = max(np.abs(res).max(), np.abs(jac).max() * np.abs(un).max(), 1e-300)
            assert np.abs(jac @ un - res[:, 0]).max() <= 1e-12 * scale


@pytest.mark.parametrize("case", ["burgers_p2_lda", "burgers_p2_n", "burgers_p2_b",
                                  "burgers_p3_b", "adv_p2_b", "euler2d_tri_p1_lda",
                                  "euler2d_tri_p2_n", "euler2d_tri_p3_b", "euler2d_quad_p3_b",
                                  "euler3d_tet_p2_lda"])
def test_element_jacobians_assemble_to_the_reference(case):
    """The oracle's element Jacobians (PGLDA / PGN / PGB), assembled as J(m, n) / V(m), against
    the reference's own Picard-Jacobian cell worker (PGRDMPicardJacCellAssemblyWorker with
    compute_adv_res_and_jacobian, PGLDA.hpp:316-536, PGN.hpp:296, PGB.hpp:503-819) dumped with
    the golden case at u0."""
    prob, a, _ = load_golden(os.path.join(GOLDEN, case))
    o = Oracle(prob)
    n, neq = prob.nnodes, prob.neq
    ref = np.zeros((n * neq, n * neq))
    ref[a["jac_row"], a["jac_col"]] = a["jac_val"]
    got = np.zeros_like(ref)
    u = np.asarray(a["u0"])
    for gi, g in enumerate(prob.groups):
        for c in range(g.ncells):
            jac = o.element_jacobian(gi, c, u)
            d = g.sol_conn[c]
            rows = (d[:, None] * neq + np.arange(neq)[None, :]).ravel()
            got[np.ix_(rows, rows)] += jac / np.repeat(o.vol[d], neq)[:, None]
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
