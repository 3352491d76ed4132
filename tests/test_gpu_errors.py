"""Failure paths through the C ABI on the GPU: invalid inputs are rejected with a status and a
message before anything runs, unsupported configurations say so, and the device-side checks
(non-finite norm, non-positive pressure, iteration cap) end the loop with their status codes
instead of faulting or hanging. Also the smallest meshes (two cells) against the oracle."""

import ctypes as C
import dataclasses
import os

import numpy as np
import pytest

from conftest import GOLDEN
from helpers import rel_err
from oracle.rds_oracle import Oracle
from golden_io import load_golden
from pdekit_b200.rds import PGRDMethodExplicit, RDSError, lib

pytestmark = pytest.mark.gpu

INVALID, NONFINITE, NEG_PRESSURE, ITER_CAP, UNSUPPORTED = 1, 3, 4, 5, 6


def _golden(case):
    return load_golden(os.path.join(GOLDEN, case))


def _solver(prob):
    s = PGRDMethodExplicit(prob.physics, prob.scheme, "fp64").configure_mesh_data(prob)
    s.initialize_work_data()
    return s


def _with_group(prob, **kw):
    return dataclasses.replace(prob, groups=[dataclasses.replace(prob.groups[0], **kw)])


@pytest.mark.parametrize("which", ["sol", "geo"])
def test_connectivity_out_of_range(which):
    prob, _, _ = _golden("burgers_p2_b")
    g = prob.groups[0]
    if which == "sol":
        conn = g.sol_conn.copy()
        conn[3, 1] = prob.nnodes
        bad = _with_group(prob, sol_conn=conn)
    else:
        conn = g.geo_conn.copy()
        conn[0, 0] = -1
        bad = _with_group(prob, geo_conn=conn)
    with pytest.raises(RDSError) as e:
        _solver(bad)
    assert e.value.status == INVALID and "out of range" in str(e.value)


def test_node_that_belongs_to_no_cell():
    prob, _, _ = _golden("adv_p1_lda")
    bad = dataclasses.replace(prob, nnodes=prob.nnodes + 1)
    with pytest.raises(RDSError) as e:
        _solver(bad)
    assert e.value.status == INVALID and "belongs to no cell" in str(e.value)


def test_empty_boundary_group_rejected():
    prob, _, _ = _golden("adv_p1_lda")
    b = prob.bcs[0]
    empty = dataclasses.replace(b, sol_conn=b.sol_conn[:0], geo_conn=b.geo_conn[:0],
                                gq=b.gq[:0])
    with pytest.raises(RDSError) as e:
        _solver(dataclasses.replace(prob, bcs=[empty]))
    assert e.value.status == INVALID


def test_euler_only_conditions_rejected_for_scalar_physics():
    prob, _, _ = _golden("adv_p1_lda")
    b = prob.bcs[0]
    for kind in ("WeakWall", "WeakFarfield"):
        wrong = dataclasses.replace(b, kind=kind, gq=np.zeros(1))
        with pytest.raises(RDSError) as e:
            _solver(dataclasses.replace(prob, bcs=[wrong]))
        assert e.value.status == UNSUPPORTED


def test_condition_after_finalize_rejected():
    prob, _, _ = _golden("adv_p1_lda")
    s = _solver(prob)
    with pytest.raises(RDSError) as e:
        s.add_boundary_condition(prob.bcs[0])
    assert e.value.status == INVALID
    s.close()


def test_element_configuration_not_compiled():
    """A quadrature rule the library has no kernel for is reported at the first assembly."""
    prob, a, meta = _golden("adv_p1_lda")
    g = prob.groups[0]
    q = 5  # no P1 triangle kernel with 5 points
    bad = _with_group(prob, w=g.w[:q], V=g.V[:q], dV=g.dV[:, :q], dVgeo=g.dVgeo[:, :q],
                      dVf=g.dVf[:, :q])
    s = _solver(bad)
    s.set_solution(a["u0"])
    with pytest.raises(RDSError) as e:
        s.assemble_lhs_and_rhs(meta["cfl"])
    assert e.value.status == UNSUPPORTED
    s.close()


def test_nonfinite_state_stops_the_loop():
    prob, a, meta = _golden("burgers_p2_n")
    u = np.array(a["u0"], dtype=np.float64)
    u[7] = np.nan
    s = _solver(prob)
    s.set_solution(u)
    with pytest.raises(RDSError) as e:
        s.iterate(meta["cfl"], 50, 1e-10)
    assert e.value.status == NONFINITE
    s.close()


def test_negative_pressure_reported():
    prob, a, meta = _golden("euler2d_tri_p1_lda")
    u = np.array(a["u0"], dtype=np.float64).reshape(prob.nnodes, prob.neq)
    u[5, 3] = -1.0  # energy below the kinetic energy: p < 0
    s = _solver(prob)
    s.set_solution(u)
    with pytest.raises(RDSError) as e:
        s.iterate(meta["cfl"], 3)
    assert e.value.status in (NEG_PRESSURE, NONFINITE)
    s.close()


def test_iteration_cap_reported():
    prob, a, meta = _golden("adv_p1_lda")
    s = _solver(prob)
    s.set_solution(a["u0"])
    with pytest.raises(RDSError) as e:
        s.iterate(meta["cfl"], 7, 1e-30)
    assert e.value.status == ITER_CAP
    it, hist = s.iterate(meta["cfl"], 7, 1e-30, raise_on_cap=False)
    assert it == 7 and np.all(np.isfinite(hist))
    s.close()


def test_interface_out_of_range_rejected():
    prob, _, _ = _golden("adv_p1_lda")
    s = _solver(prob)
    nodes = np.array([prob.nnodes], dtype=np.int32)
    slots = np.array([0], dtype=np.int32)
    owned = np.ones(prob.nnodes, dtype=np.uint8)
    st = lib().rds_set_interface(s._ctx, 1, nodes.ctypes.data_as(C.c_void_p),
                                 slots.ctypes.data_as(C.c_void_p), 1,
                                 owned.ctypes.data_as(C.c_void_p))
    assert st == INVALID
    s.close()


@pytest.mark.parametrize("physics,scheme,p", [("advconst", "lda", 1), ("burgers", "b", 2),
                                              ("burgers", "n", 3)])
def test_two_cell_mesh_matches_oracle(physics, scheme, p):
    from pdekit_b200 import reference_element as R
    from pdekit_b200 import workloads as W

    rule = {1: 4, 2: 5, 3: 8}[p]
    bcs = W.ADV_BCS if physics == "advconst" else W.BURGERS_BCS
    prob = W.tri_problem(physics, scheme, p, 1, 0.0, 1, bcs, R.triag_tables(p, rule))
    assert prob.ncells == 2
    u0 = W.initial_state(prob, "zero" if physics == "advconst" else "burgers", prob.sol_coords)
    s = _solver(prob)
    s.set_solution(u0)
    s.iterate(0.5, 10)
    u_ref, _ = Oracle(prob).iterate(u0, 0.5, 10)
    assert rel_err(s.solution(), u_ref) < 1e-12
    s.close()
