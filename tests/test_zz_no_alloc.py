"""The allocation-free residual norm (rds_residual_norm_noalloc) against rds_residual_norm.

rds_residual_norm_noalloc is for callers that may not allocate device memory themselves (their
device memory belongs to another allocator, or their loop cannot take cudaMalloc's implicit
synchronisation); it works from caller-owned device arrays and a fixed scratch array inside the
library. This file runs last so a failure here leaves every other test already run.
"""

import ctypes as C
import os

import numpy as np
import pytest

from conftest import GOLDEN
from pdekit_b200 import reference_element, workloads
from golden_io import load_golden
from pdekit_b200.rds import PGRDMethodExplicit, lib

pytestmark = pytest.mark.gpu

MAX_NODES = 32768 * 256  # RDS_NOALLOC_MAX_NODES in include/rds_b200.h


def _noalloc():
    f = lib().rds_residual_norm_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _device_norm(res, dt):
    """Norm through the allocation-free entry point on device copies of res [n,neq], dt [n]."""
    import torch

    n, neq = res.shape
    d_res = torch.from_numpy(np.ascontiguousarray(res.T)).cuda()  # SoA [neq][n]
    d_dt = torch.from_numpy(np.ascontiguousarray(dt)).cuda()
    d_norm = torch.full((neq,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = _noalloc()(d_res.data_ptr(), d_dt.data_ptr(), n, neq, d_norm.data_ptr(), None)
    assert st == 0
    torch.cuda.synchronize()
    return d_norm.cpu().numpy()


def _problem(which):
    """Scalar (one equation) small and 66-block cases, Euler 2D (4) and Euler 3D (5)."""
    if which == "burgers_64":
        t = reference_element.triag_tables(2, 5)
        n = 64  # 16,641 nodes: 66 blocks of partial sums
        big = workloads.tri_problem("burgers", "b", 2, n, 0.15, 7, workloads.BURGERS_BCS, t)
        u0 = workloads.initial_state(big, "burgers", workloads.sol_coords_tri(n, 0.15, 7, 2))
        return big, u0, 0.5
    prob, a, meta = load_golden(os.path.join(GOLDEN, which))
    return prob, a["u0"], meta["cfl"]


@pytest.mark.parametrize("which", ["burgers_p2_b", "burgers_64", "euler2d_quad_p3_b",
                                   "euler3d_tet_p2_lda"])
def test_noalloc_norm_matches_existing_entry_two_calls(which):
    """Two calls in a row on different residuals; the block split and the summation order are
    those of rds_residual_norm, so the results are equal bit for bit."""
    prob, u0, cfl = _problem(which)
    s = PGRDMethodExplicit(prob.physics, prob.scheme).configure_mesh_data(prob)
    s.initialize_work_data()
    s.set_solution(u0)
    for call in range(2):  # two calls in a row, on different residuals
        s.assemble_lhs_and_rhs(cfl)
        ref = s.compute_residual_norm()
        res, dt, _, _ = s.fields()
        got = _device_norm(res, dt)
        assert got.shape == (prob.neq,)
        np.testing.assert_array_equal(got, ref)
        s.solve()
    s.close()


def test_noalloc_rejects_too_many_nodes():
    import torch

    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    assert _noalloc()(p, p, MAX_NODES + 1, 1, p, None) == 7  # RDS_ERR_TOO_LARGE, nothing launched
    assert _noalloc()(p, p, 10, 6, p, None) == 1  # neq > 5: RDS_ERR_INVALID
