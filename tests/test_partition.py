"""Partitioned single mesh (pdekit_b200/partition.py) on the CPU: the split itself, and the
per-rank algorithm (partial sums, exchange of the interface nodes, finish on every rank) run
with the C oracle's assemble in place of the GPU kernels, in one process and as two gloo ranks,
against the oracle on the whole mesh."""

import os

import numpy as np
import pytest

from conftest import GOLDEN
from helpers import rel_err
from oracle.rds_oracle import Oracle
from pdekit_b200.partition import partition
from golden_io import load_golden

CASES = ["burgers_p2_b", "adv_p2_b", "euler2d_tri_p3_b", "euler2d_quad_p3_b",
         "euler3d_tet_p2_lda", "euler2d_tri_p2_farfield"]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("nparts", [1, 2, 3])
def test_partition_invariants(case, nparts):
    prob, _, _ = load_golden(os.path.join(GOLDEN, case))
    pt = partition(prob, nparts)
    assert len(pt.parts) == nparts
    for ig, g in enumerate(prob.groups):
        cells = np.sort(np.concatenate([p.cells[ig] for p in pt.parts]))
        assert np.array_equal(cells, np.arange(g.ncells))  # every cell on exactly one rank
    owned = np.zeros(prob.nnodes, dtype=int)
    slot_node = {}
    for p in pt.parts:
        owned[p.nodes] += p.owned
        assert p.problem.nnodes == len(p.nodes)
        for g in p.problem.groups:
            assert g.sol_conn.min() >= 0 and g.sol_conn.max() < p.problem.nnodes
        for ln, sl in zip(p.if_nodes, p.if_slots):
            assert slot_node.setdefault(int(sl), int(p.nodes[ln])) == int(p.nodes[ln])
    assert (owned == 1).all()  # every node counted once in the norm
    assert len(slot_node) == pt.nslots
    for b in prob.bcs:  # every facet on exactly one rank
        n = sum(bb.nfacets for p in pt.parts for bb in p.problem.bcs if bb.name == b.name)
        assert n == b.nfacets


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("nparts", [1, 2, 3])
def test_interface_first_layout(case, nparts):
    """The overlapped step's layout: a rank's interface nodes are its first local nodes, its
    first n_if_groups groups hold exactly the cells touching one, and the other groups touch none
    (so the interface sums need only the first groups and the facets)."""
    prob, _, _ = load_golden(os.path.join(GOLDEN, case))
    pt = partition(prob, nparts)
    for p in pt.parts:
        n_if = len(p.if_nodes)
        assert np.array_equal(p.if_nodes, np.arange(n_if))
        groups = p.problem.groups
        assert 0 <= p.n_if_groups <= len(groups)
        for k, g in enumerate(groups):
            touches = (g.sol_conn < n_if).any(axis=1)
            assert touches.all() if k < p.n_if_groups else not touches.any()
        assert sum(g.ncells for g in groups) == sum(len(c) for c in p.cells)
    if nparts == 1:
        assert pt.nslots == 0 and pt.parts[0].n_if_groups == 0


def test_partition_rejects_strong_conditions():
    prob, _, _ = load_golden(os.path.join(GOLDEN, "adv_p1_strong"))
    with pytest.raises(NotImplementedError):
        partition(prob, 2)


def _rank_oracles(prob, pt):
    """Oracle of every rank with the dual volumes summed over the ranks."""
    ors = [Oracle(p.problem) for p in pt.parts]
    vol = np.zeros(prob.nnodes)
    for p, o in zip(pt.parts, ors):
        vol[p.nodes] += o.vol
    for p, o in zip(pt.parts, ors):
        o.vol[:] = vol[p.nodes]
    return ors


def _finish(p, o, res, ws, u, cfl):
    dt = cfl * o.vol / ws
    u -= dt[:, None] * res
    return ((res * dt[:, None]) ** 2)[p.owned.astype(bool)].sum(axis=0)


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("nparts", [2, 3])
def test_partitioned_algorithm_matches_whole_mesh(case, nparts):
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    cfl, iters = meta["cfl"], 4
    pt = partition(prob, nparts)
    ors = _rank_oracles(prob, pt)
    us = [np.array(a["u0"]).reshape(-1, prob.neq)[p.nodes].copy() for p in pt.parts]
    norms = []
    for _ in range(iters):
        buf = np.zeros((pt.nslots, prob.neq + 1))
        parts = []
        for p, o, u in zip(pt.parts, ors, us):
            res, ws, _, bad = o.assemble(u, cfl)
            assert bad == 0
            parts.append((res, ws))
            buf[p.if_slots, :prob.neq] += res[p.if_nodes]
            buf[p.if_slots, prob.neq] += ws[p.if_nodes]
        sq = np.zeros(prob.neq)
        for p, o, u, (res, ws) in zip(pt.parts, ors, us, parts):
            res[p.if_nodes] = buf[p.if_slots, :prob.neq]
            ws[p.if_nodes] = buf[p.if_slots, prob.neq]
            sq += _finish(p, o, res, ws, u, cfl)
        norms.append(np.sqrt(sq / prob.nnodes))
    u = np.zeros((prob.nnodes, prob.neq))
    for p, ul in zip(pt.parts, us):
        u[p.nodes[p.owned.astype(bool)]] = ul[p.owned.astype(bool)]
    u_ref, n_ref = Oracle(prob).iterate(a["u0"], cfl, iters)
    assert rel_err(u, u_ref) < 1e-12
    np.testing.assert_allclose(np.array(norms), n_ref, rtol=1e-11)


def _gloo_rank(rank, world, port, case, out):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        prob, a, meta = load_golden(os.path.join(GOLDEN, case))
        cfl = meta["cfl"]
        pt = partition(prob, world)
        p = pt.parts[rank]
        o = Oracle(p.problem)
        vol = torch.zeros(prob.nnodes, dtype=torch.float64)
        vol[torch.as_tensor(p.nodes)] = torch.as_tensor(o.vol)
        dist.all_reduce(vol)
        o.vol[:] = vol.numpy()[p.nodes]
        u = np.array(a["u0"]).reshape(-1, prob.neq)[p.nodes].copy()
        slots = torch.as_tensor(p.if_slots.astype(np.int64))
        norms = []
        for _ in range(3):
            res, ws, _, _ = o.assemble(u, cfl)
            buf = torch.zeros((pt.nslots, prob.neq + 1), dtype=torch.float64)
            buf[slots, :prob.neq] = torch.as_tensor(res[p.if_nodes])
            buf[slots, prob.neq] = torch.as_tensor(ws[p.if_nodes])
            dist.all_reduce(buf)
            res[p.if_nodes] = buf.numpy()[p.if_slots, :prob.neq]
            ws[p.if_nodes] = buf.numpy()[p.if_slots, prob.neq]
            sq = torch.as_tensor(_finish(p, o, res, ws, u, cfl))
            dist.all_reduce(sq)
            norms.append(np.sqrt(sq.numpy() / prob.nnodes))
        ug = torch.zeros((prob.nnodes, prob.neq), dtype=torch.float64)
        own = p.owned.astype(bool)
        ug[torch.as_tensor(p.nodes[own])] = torch.as_tensor(u[own])
        dist.all_reduce(ug)
        if rank == 0:
            np.save(out + ".u.npy", ug.numpy())
            np.save(out + ".n.npy", np.array(norms))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", ["burgers_p2_b", "euler2d_tri_p3_b"])
def test_partitioned_two_gloo_ranks(case, tmp_path):
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "r0")
    mp.start_processes(_gloo_rank, args=(2, port, case, out), nprocs=2, join=True,
                       start_method="spawn")
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    u_ref, n_ref = Oracle(prob).iterate(a["u0"], meta["cfl"], 3)
    assert rel_err(np.load(out + ".u.npy"), u_ref) < 1e-12
    np.testing.assert_allclose(np.load(out + ".n.npy"), n_ref, rtol=1e-11)
