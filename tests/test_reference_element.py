"""Host-side reference-element tables against the reference's own tables (golden) and against
polynomial exactness (CPU)."""

import os

import numpy as np
import pytest

from conftest import GOLDEN
from pdekit_b200 import reference_element as re_
from golden_io import load_golden

CASES = {(1, 4): "adv_p1_lda", (2, 5): "burgers_p2_b", (3, 8): "burgers_p3_b",
         (3, 6): "burgers_p3_q6_b"}


def _match_rows(a, b, tol=1e-13):
    """Permutation mapping rows of a onto rows of b (points of a rule in another order)."""
    perm = []
    for row in a:
        d = np.abs(b - row).max(axis=1)
        k = int(np.argmin(d))
        assert d[k] < tol, (row, d[k])
        perm.append(k)
    assert len(set(perm)) == len(perm)
    return np.asarray(perm)


@pytest.mark.parametrize("p,q", sorted(CASES))
def test_tables_match_reference(p, q):
    _, a, _ = load_golden(os.path.join(GOLDEN, CASES[(p, q)]))
    t = re_.triag_tables(p, q)
    perm = _match_rows(t["qp"], a["qp"])  # same point set, possibly another order
    np.testing.assert_allclose(t["w"], a["w"][perm], rtol=0, atol=1e-14)
    np.testing.assert_allclose(t["V"], a["V"][perm], rtol=0, atol=1e-13)
    for d in range(2):
        np.testing.assert_allclose(t["dV"][d], a[f"dV{d}"][perm], rtol=0, atol=1e-12)
        np.testing.assert_allclose(t["dVgeo"][d], a[f"dVgeo{d}"][perm], rtol=0, atol=1e-13)
        np.testing.assert_allclose(t["dVf"][d], a[f"dVf{d}"][perm], rtol=0, atol=1e-12)
    np.testing.assert_allclose(t["Vsf"], a["Vsf"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(t["fqp"], a["fqp"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(t["fw"], a["fw"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(t["fV"], a["fV"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(t["fdVgeo"][0], a["fdVgeo0"], rtol=0, atol=1e-14)


@pytest.mark.parametrize("order", [1, 2, 4, 5, 8])
def test_triangle_rules_exact(order):
    qp, w = re_.triag_gauss(order)
    assert abs(w.sum() - 2.0) < 1e-14
    # integrate (1+xi)^a (1+eta)^b over the reference triangle exactly:
    # 2^(a+b+2) a! b! / (a+b+2)! on the triangle of area 2
    from math import factorial
    for a_ in range(order + 1):
        for b_ in range(order + 1 - a_):
            exact = 2.0 ** (a_ + b_ + 2) * factorial(a_) * factorial(b_) / factorial(a_ + b_ + 2)
            got = (w * (1 + qp[:, 0]) ** a_ * (1 + qp[:, 1]) ** b_).sum()
            assert abs(got - exact) < 1e-13 * max(1.0, exact), (a_, b_)


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_lagrange_partition_of_unity_and_kronecker(p):
    from pdekit_b200 import meshgen
    nodes = meshgen.equidist_triag_nodes(p)
    V, dV = re_.lagrange_triag(p, nodes)
    np.testing.assert_allclose(V, np.eye(nodes.shape[0]), atol=1e-14)
    qp, _ = re_.triag_gauss(8)
    V, dV = re_.lagrange_triag(p, qp)
    np.testing.assert_allclose(V.sum(axis=1), 1.0, atol=1e-14)
    np.testing.assert_allclose(dV.sum(axis=2), 0.0, atol=1e-12)


@pytest.mark.parametrize("case,order", [("euler2d_quad_p2_b_bonanni", 5),
                                        ("euler2d_quad_p3_b", 8)])
def test_square_rules_match_reference(case, order):
    """quad_gauss against the rule the reference integrated the fixture's cells with (its
    symmetric 8- and 20-point rules, points in the same order). The reference tabulates them
    to 14 - 15 digits."""
    _, a, _ = load_golden(os.path.join(GOLDEN, case))
    qp, w = re_.quad_gauss(order)
    np.testing.assert_allclose(qp, a["qp"], rtol=0, atol=5e-14)
    np.testing.assert_allclose(w, a["w"], rtol=0, atol=5e-14)


@pytest.mark.parametrize("order", range(1, 9))
def test_square_rules_exact(order):
    """Every rule integrates the monomials of its degree exactly on [-1,1]^2 (degree 1, 3, 3, 5,
    5, 7, 7, 9 for orders 1 - 8) and the rule of order 6 is the oracle's closed form."""
    qp, w = re_.quad_gauss(order)
    deg = order if order % 2 else order + 1
    for i in range(deg + 1):
        for j in range(deg + 1 - i):
            ex = (0.0 if i % 2 or j % 2 else 4.0 / ((i + 1) * (j + 1)))
            assert abs(np.sum(w * qp[:, 0] ** i * qp[:, 1] ** j) - ex) < 1e-14
    if order in (4, 6):
        from oracle.stab_oracle import _gauss_quad
        oq, ow = _gauss_quad(order)
        key = lambda q: np.lexsort((q[:, 1], q[:, 0]))
        np.testing.assert_allclose(qp[key(qp)], oq[key(oq)], atol=1e-14)
        np.testing.assert_allclose(w[key(qp)], ow[key(oq)], atol=1e-14)
    with pytest.raises(ValueError):
        re_.quad_gauss(9)


def test_p1_tet_tables_match_reference():
    """P1 tetrahedra with the order-2 rule (4 points) and P1 triangle facets (order 3). The
    reference tabulates the tetrahedron rule's points to about ten digits (5e-11 here)."""
    _, a, _ = load_golden(os.path.join(GOLDEN, "euler3d_tet_p1_lda"))
    t = re_.tet_tables(1, 2)
    perm = _match_rows(t["qp"], a["qp"], tol=1e-10)
    np.testing.assert_allclose(t["w"], a["w"][perm], rtol=0, atol=1e-14)
    np.testing.assert_allclose(t["V"], a["V"][perm], rtol=0, atol=1e-10)
    for d in range(3):
        np.testing.assert_allclose(t["dV"][d], a[f"dV{d}"][perm], rtol=0, atol=1e-12)
        np.testing.assert_allclose(t["dVf"][d], a[f"dVf{d}"][perm], rtol=0, atol=1e-9)
    np.testing.assert_allclose(t["Vsf"], a["Vsf"], rtol=0, atol=1e-13)
    fperm = _match_rows(t["fqp"], a["fqp"])
    np.testing.assert_allclose(t["fw"], a["fw"][fperm], rtol=0, atol=1e-14)


def test_p2_tet_order4_rule_matches_reference():
    """The 11-point order-4 tetrahedron rule (negative centroid weight) against the one the
    reference integrated the fixture with (its points tabulated to about ten digits)."""
    _, a, _ = load_golden(os.path.join(GOLDEN, "euler3d_tet_p2_q4_n"))
    qp, w = re_.tet_gauss(4)
    perm = _match_rows(qp, a["qp"], tol=1e-10)
    np.testing.assert_allclose(w, a["w"][perm], rtol=0, atol=1e-10)
    # exact to degree 4 on the reference tetrahedron (volume 4/3): in barycentric coordinates
    # int l1^a l2^b l3^c = a! b! c! 3! V / (a + b + c + 3)!
    from math import factorial
    lam = (1.0 + qp) / 2.0
    for i in range(5):
        for j in range(5 - i):
            for k in range(5 - i - j):
                got = np.sum(w * lam[:, 0] ** i * lam[:, 1] ** j * lam[:, 2] ** k)
                ex = factorial(i) * factorial(j) * factorial(k) * 6 * (4.0 / 3.0) / \
                    factorial(i + j + k + 3)
                assert abs(got - ex) < 1e-14
