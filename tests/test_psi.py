"""The PSI scheme on the CPU. The reference has no PSI scheme: its residual limiter
(src/solver/rdm/cellsplitters/LFResidualLimiter.hpp:37-110) serves only its Lax-Friedrichs
schemes, so PSI here is the PGN residuals limited by that limiter and has no reference output
to be pinned on. Checked instead: the oracle's PSI cell residuals against the limiter restated
in numpy on the oracle's PGN residuals (whose PGN is pinned on the reference), the properties
the limiter guarantees (conservation: the node residuals still sum to the cell residual;
positivity: each has the sign of the cell residual; the wave speed is PGN's), and that contexts
refuse the scheme where it is not provided (descriptor validation, no GPU needed)."""

import ctypes
import dataclasses
import os

import numpy as np
import pytest

from conftest import GOLDEN
from golden_io import load_golden
from oracle.rds_oracle import Oracle
from pdekit_b200 import rds

CASES = ["adv_p1_n", "burgers_p2_n", "burgers_p3_b", "adv_p2_b"]


def limit(phi_n, phi):
    """LFResidualLimiter<Physics, 1>::limit_cell_residuals on one cell: where |phi| > 1e-14,
    x_n = std::max(phi_n / phi, 0.0) + 1e-12 and phi_n = x_n / sum x * phi."""
    if not abs(phi) > 1e-14:
        return phi_n.copy()
    r = phi_n / phi
    x = np.where(r < 0.0, 0.0, r) + 1e-12
    return x / x.sum() * phi


@pytest.mark.parametrize("case", CASES)
def test_oracle_psi_is_the_limited_n_scheme(case):
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    on = Oracle(dataclasses.replace(prob, scheme="n"))
    op = Oracle(dataclasses.replace(prob, scheme="psi"))
    g = prob.groups[0]
    limited = 0
    for u in (a["u0"], a["uK"]):
        scale = 0.0
        for c in range(g.ncells):
            rn, wn = on.cell_residual(0, c, u)
            rp, wp = op.cell_residual(0, c, u)
            phi = rn[:, 0].sum()
            scale = max(scale, np.abs(rn).max())
            np.testing.assert_array_equal(wp, wn)
            np.testing.assert_allclose(rp[:, 0], limit(rn[:, 0], phi), rtol=0,
                                       atol=1e-13 * max(abs(phi), 1e-300) + 1e-300)
            if abs(phi) > 1e-14:
                assert abs(rp[:, 0].sum() - phi) <= 1e-13 * abs(phi)
                assert (rp[:, 0] * np.sign(phi) > 0.0).all()
                limited += bool((rn[:, 0] * np.sign(phi) < 0.0).any())
        assert scale > 0.0
    # the limiter changed the distribution somewhere (N residuals of both signs in a cell)
    assert limited > 0


def test_oracle_psi_iterations_stay_finite():
    prob, a, meta = load_golden(os.path.join(GOLDEN, "burgers_p2_n"))
    u, norms = Oracle(dataclasses.replace(prob, scheme="psi")).iterate(a["u0"], meta["cfl"], 20)
    assert np.isfinite(u).all() and np.isfinite(norms).all()


def test_psi_refused_where_not_provided():
    """Euler (the reference's limiter is empty for systems) and mixed precision contexts."""
    L = rds.lib()
    coords = np.zeros((3, 2))
    for physics, neq, precision in [(2, 4, 0), (1, 1, 1), (0, 1, 1)]:
        d = rds._Desc()
        d.physics, d.dim, d.neq, d.scheme, d.precision = physics, 2, neq, rds.SCHEME["psi"], precision
        d.nnodes, d.ngeo_nodes, d.geo_coords = 3, 3, coords.ctypes.data_as(ctypes.c_void_p)
        ctx = ctypes.c_void_p()
        assert L.rds_create(ctypes.byref(ctx), ctypes.byref(d), None) == 6  # RDS_ERR_UNSUPPORTED
        assert b"PSI" in L.rds_last_error(ctx)
        L.rds_destroy(ctx)


def test_oracle_refuses_psi_jacobians():
    prob, a, meta = load_golden(os.path.join(GOLDEN, "burgers_p2_n"))
    with pytest.raises(ValueError):
        Oracle(dataclasses.replace(prob, scheme="psi")).element_jacobian(0, 0, a["u0"])
