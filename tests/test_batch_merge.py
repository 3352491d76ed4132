"""Host-side batching: the disjoint union of independent problems (no GPU)."""

import numpy as np

from pdekit_b200 import workloads
from pdekit_b200.batch import merge_problems


def _small_batch():
    return workloads.config5(nprob=9, seed=3, min_cells=50, max_cells=800)


def test_node_and_cell_ranges():
    probs, states, cfls, info = _small_batch()
    m = merge_problems(probs)
    assert m.nproblems == len(probs)
    assert m.node_off[0] == 0 and m.node_off[-1] == m.nnodes == sum(p.nnodes for p in probs)
    assert m.ncells == sum(p.ncells for p in probs)
    for g, phys, scheme, pc in m.groups:
        assert pc[0] == 0 and pc[-1] == g.ncells and np.all(np.diff(pc) >= 0)
        for i in range(m.nproblems):
            rows = g.sol_conn[pc[i]:pc[i + 1]]
            if rows.size:
                assert probs[i].physics == phys and probs[i].scheme == scheme
                assert rows.min() >= m.node_off[i] and rows.max() < m.node_off[i + 1]
                geo = g.geo_conn[pc[i]:pc[i + 1]]
                assert geo.min() >= m.geo_off[i] and geo.max() < m.geo_off[i + 1]


def test_union_restores_each_problem():
    probs, _, _, _ = _small_batch()
    m = merge_problems(probs)
    for i, p in enumerate(probs):
        mine = [g.sol_conn[pc[i]:pc[i + 1]] - m.node_off[i] for g, _, _, pc in m.groups
                if pc[i + 1] > pc[i]]
        assert len(mine) == len(p.groups) == 1
        np.testing.assert_array_equal(mine[0], p.groups[0].sol_conn)
        # the problem meets its weak conditions in its own (name) order
        names = [b.name for b, _ in m.bcs
                 if np.any((b.sol_conn >= m.node_off[i]) & (b.sol_conn < m.node_off[i + 1]))]
        assert names == [b.name for b in p.bcs]


def test_bc_facets_and_data_follow_their_problem():
    probs, _, _, _ = _small_batch()
    m = merge_problems(probs)
    for b, phys in m.bcs:
        owner = np.searchsorted(m.node_off, b.sol_conn[:, 0], side="right") - 1
        for f in range(b.nfacets):
            i = owner[f]
            assert np.all((b.sol_conn[f] >= m.node_off[i]) & (b.sol_conn[f] < m.node_off[i + 1]))
            assert probs[i].physics == phys
        assert b.gq.shape == (b.nfacets, b.nfq, 1)


def test_config5_draws():
    probs, states, cfls, info = workloads.config5(nprob=40, seed=5, min_cells=50, max_cells=2000)
    assert len(probs) == len(states) == len(cfls) == 40
    kinds = {i["physics"] for i in info}
    orders = {i["order"] for i in info}
    assert kinds == {"advconst", "burgers"} and orders == {1, 2, 3}
    for p, u, c, i in zip(probs, states, cfls, info):
        assert u.shape == (p.nnodes, 1) and 0.3 <= c <= 0.9
        assert p.scheme == ("lda" if p.physics == "advconst" else "n")
