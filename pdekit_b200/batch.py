"""Many independent scalar problems solved in one context (batched form of the explicit loop).

The reference solves one problem per PGRDMethodExplicit object
(src/solver/rdm/PGRDMethodExplicit.hpp:417-514). Here P problems of uneven size, of either
scalar physics (constant advection, Burgers), of orders P1-P3 and each with its own CFL, are put
into one context as a disjoint union:

* nodes of problem p occupy [node_off[p], node_off[p+1]); geometry nodes likewise;
* cells of the same (physics, scheme, element type, order, tables) from all problems form one
  cell group, problem by problem, with per-problem cell offsets; one persistent launch per group
  walks the tiles of the problems still iterating;
* weak conditions of the same (name, kind, physics, facet tables) form one facet group; a
  problem meets its conditions in name order, as in its own context.

Every node sees its contributions in the same order as in the problem's own context, so each
problem's iterates, iteration count and norms equal the single-problem run bit for bit.
"""

from __future__ import annotations

import ctypes as C
import dataclasses
import hashlib

import numpy as np

from .problem import BCGroup, CellGroup, Problem
from .rds import (BC_KIND, PHYSICS, PRECISION, SCHEME, SHAPE, RDSError, _BCGroup, _CellGroup,
                  _Desc, _ptr, lib)


def _sig(*arrays) -> str:
    h = hashlib.sha1()
    for a in arrays:
        if a is None:
            h.update(b"none")
        else:
            a = np.ascontiguousarray(a, dtype=np.float64)
            h.update(str(a.shape).encode())
            h.update(a.tobytes())
    return h.hexdigest()


@dataclasses.dataclass
class MergedBatch:
    nnodes: int
    geo_coords: np.ndarray
    node_off: np.ndarray  # [P+1] int32
    geo_off: np.ndarray  # [P+1] int32
    groups: list  # [(CellGroup, physics, scheme, problem_cells [P+1] int32)]
    bcs: list  # [(BCGroup, physics)]
    adv: tuple

    @property
    def nproblems(self):
        return len(self.node_off) - 1

    @property
    def ncells(self):
        return sum(g.ncells for g, _, _, _ in self.groups)


def merge_problems(problems: list) -> MergedBatch:
    """Disjoint union of scalar 2D problems (host arrays only)."""
    if not problems:
        raise ValueError("no problems")
    adv = None
    for p in problems:
        if p.physics not in ("advconst", "burgers") or p.dim != 2 or p.neq != 1:
            raise ValueError("batched problems: scalar 2D physics only")
        if p.physics == "advconst":
            if adv is not None and tuple(adv) != tuple(p.adv):
                raise ValueError("batched advection problems must share the advection vector")
            adv = tuple(p.adv)
    P = len(problems)
    node_off = np.zeros(P + 1, dtype=np.int64)
    geo_off = np.zeros(P + 1, dtype=np.int64)
    for i, p in enumerate(problems):
        node_off[i + 1] = node_off[i] + p.nnodes
        geo_off[i + 1] = geo_off[i] + p.geo_coords.shape[0]
    if node_off[-1] >= 2**31 or geo_off[-1] >= 2**31:
        raise ValueError("more than 2^31 nodes in the batch")
    coords = np.concatenate([np.asarray(p.geo_coords, dtype=np.float64) for p in problems])

    # cell groups by (physics, scheme, shape, order, tables), in order of first appearance
    gkeys, gparts = [], {}
    for i, p in enumerate(problems):
        for g in p.groups:
            key = (p.physics, p.scheme, g.shape, g.order,
                   _sig(g.w, g.V, g.dV, g.dVgeo, g.dVf, g.Vsf, g.wv, g.dVgeo_v))
            if key not in gparts:
                gkeys.append(key)
                gparts[key] = (g, [])
            gparts[key][1].append((i, g))
    groups = []
    for key in gkeys:
        tmpl, parts = gparts[key]
        counts = np.zeros(P, dtype=np.int64)
        sol, geo = [], []
        for i, g in parts:
            counts[i] += g.ncells
            sol.append(np.asarray(g.sol_conn, dtype=np.int64) + node_off[i])
            geo.append(np.asarray(g.geo_conn, dtype=np.int64) + geo_off[i])
        pc = np.zeros(P + 1, dtype=np.int32)
        pc[1:] = np.cumsum(counts)
        mg = dataclasses.replace(tmpl, sol_conn=np.concatenate(sol).astype(np.int32),
                                 geo_conn=np.concatenate(geo).astype(np.int32))
        groups.append((mg, key[0], key[1], pc))

    # weak conditions by (name, kind, physics, facet tables); applied in name order
    bkeys, bparts = [], {}
    for i, p in enumerate(problems):
        for b in p.bcs:
            key = (b.name, b.kind, p.physics, b.order, tuple(b.params),
                   _sig(b.fw, b.fV, b.fVgeo, b.fdVgeo))
            if key not in bparts:
                bkeys.append(key)
                bparts[key] = (b, [])
            bparts[key][1].append((i, b))
    bcs = []
    for key in sorted(bkeys, key=lambda k: (k[0], bkeys.index(k))):
        tmpl, parts = bparts[key]
        mb = dataclasses.replace(
            tmpl,
            sol_conn=np.concatenate([np.asarray(b.sol_conn, np.int64) + node_off[i]
                                     for i, b in parts]).astype(np.int32),
            geo_conn=np.concatenate([np.asarray(b.geo_conn, np.int64) + geo_off[i]
                                     for i, b in parts]).astype(np.int32),
            gq=np.concatenate([b.gq for _, b in parts]))
        bcs.append((mb, key[2]))
    return MergedBatch(nnodes=int(node_off[-1]), geo_coords=coords,
                       node_off=node_off.astype(np.int32), geo_off=geo_off.astype(np.int32),
                       groups=groups, bcs=bcs, adv=adv or (0.0, 0.0, 0.0))


def problem_work(p: Problem) -> float:
    """Relative cost estimate of iterating one problem to its drop: cells x points x dofs (one
    cell kernel step) x order (pseudo-time iterations grow with the order)."""
    return float(sum(g.ncells * g.nq * g.ndof * g.order for g in p.groups))


def shard_problems(problems: list, nranks: int) -> list:
    """Split independent problems over ranks (one GPU each): largest estimated work first, each
    to the least loaded rank. Returns the sorted problem indices of every rank; the problems need
    no exchange between ranks."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    load = [0.0] * nranks
    shards = [[] for _ in range(nranks)]
    order = sorted(range(len(problems)), key=lambda i: (-problem_work(problems[i]), i))
    for i in order:
        r = min(range(nranks), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += problem_work(problems[i])
    return [sorted(sh) for sh in shards]


class BatchedRDS:
    """P independent problems iterated together: persistent cell launches over the active
    problems, one per-problem gather / update / norm / stop test, the loop in one CUDA graph."""

    def __init__(self, problems: list, cfl, precision: str = "fp64"):
        self.problems = list(problems)
        self.precision = precision
        self.merged = m = merge_problems(self.problems)
        P = m.nproblems
        self.cfl = np.ascontiguousarray(np.broadcast_to(np.asarray(cfl, dtype=np.float64), (P,)))
        self._keep = [m.geo_coords, m.node_off, self.cfl]
        self._ctx = None
        L = lib()
        d = _Desc()
        first = self.problems[0]
        d.physics, d.scheme = PHYSICS[first.physics], SCHEME[first.scheme]
        d.precision = PRECISION[precision]
        d.dim, d.neq, d.nnodes = 2, 1, m.nnodes
        d.ngeo_nodes = m.geo_coords.shape[0]
        d.geo_coords = _ptr(m.geo_coords)
        for i, v in enumerate(m.adv):
            d.adv[i] = v
        ctx = C.c_void_p()
        st = L.rds_create(C.byref(ctx), C.byref(d), None)
        self._ctx = ctx
        self._check(st)
        self._check(L.rds_set_problems(self._ctx, P, _ptr(m.node_off), _ptr(self.cfl)))
        for g, phys, scheme, pc in m.groups:
            arrs = [np.ascontiguousarray(g.sol_conn, dtype=np.int32),
                    np.ascontiguousarray(g.geo_conn, dtype=np.int32)] + \
                   [np.ascontiguousarray(x, dtype=np.float64) for x in
                    (g.w, g.V, g.dV, g.dVgeo, g.dVf, g.Vsf)]
            self._keep += arrs + [pc]
            cg = _CellGroup(SHAPE[g.shape], g.order, g.ncells, g.ndof, g.ngeo, g.nq, g.nfl,
                            *[_ptr(a) for a in arrs])
            if g.wv is not None:
                va = [np.ascontiguousarray(g.wv, dtype=np.float64),
                      np.ascontiguousarray(g.dVgeo_v, dtype=np.float64)]
                self._keep += va
                cg.nqv, cg.wv, cg.dVgeo_v = va[0].shape[0], _ptr(va[0]), _ptr(va[1])
            self._check(L.rds_add_batch_cell_group(self._ctx, C.byref(cg), PHYSICS[phys],
                                                   SCHEME[scheme], _ptr(pc)))
        for b, phys in m.bcs:
            arrs = [np.ascontiguousarray(b.sol_conn, dtype=np.int32),
                    np.ascontiguousarray(b.geo_conn, dtype=np.int32)] + \
                   [np.ascontiguousarray(x, dtype=np.float64) for x in
                    (b.fw, b.fV, b.fdVgeo, b.gq)]
            self._keep += arrs
            cb = _BCGroup(BC_KIND[b.kind], b.nfacets, b.nfdof, b.nfgeo, b.nfq,
                          *[_ptr(a) for a in arrs])
            cb.order = b.order
            for k, v in enumerate(b.params[:4]):
                cb.params[k] = v
            self._check(L.rds_add_batch_bc(self._ctx, C.byref(cb), PHYSICS[phys]))
        self._check(L.rds_finalize(self._ctx))

    @property
    def nproblems(self):
        return self.merged.nproblems

    def set_solutions(self, states):
        u = np.concatenate([np.asarray(s, dtype=np.float64).reshape(-1) for s in states])
        if u.shape[0] != self.merged.nnodes:
            raise ValueError("states do not match the problems' node counts")
        self._check(lib().rds_set_state(self._ctx, _ptr(np.ascontiguousarray(u))))

    def solutions(self):
        u = np.empty(self.merged.nnodes)
        self._check(lib().rds_get_state(self._ctx, _ptr(u)))
        o = self.merged.node_off
        return [u[o[i]:o[i + 1]].reshape(-1, 1).copy() for i in range(self.nproblems)]

    def autotune(self):
        """Time tile / grid shapes of every group's persistent kernel; returns the choices."""
        import json

        buf = C.create_string_buffer(1 << 16)
        self._check(lib().rds_autotune(self._ctx, buf, len(buf)))
        return json.loads(buf.value.decode())

    def iterate(self, max_iter: int, drop: float = 1e-10, raise_on_cap=True):
        """Iterate every problem to its own drop; returns (iterations [P], final drop [P])."""
        iters = np.zeros(self.nproblems, dtype=np.int32)
        rel = np.zeros(self.nproblems)
        st = lib().rds_iterate_batch(self._ctx, int(max_iter), float(drop), _ptr(iters),
                                     _ptr(rel))
        if not (st == 5 and not raise_on_cap):
            self._check(st)
        return iters, rel

    def advance_rk3tvd(self, nsteps: int = 1):
        """nsteps RK3TVD steps of every problem, each with its own CFL (the single-problem
        stepper's stages over the batch's kernels, FP64 in both precisions); waits for them."""
        self._check(lib().rds_advance_rk3tvd(self._ctx, 0.0, int(nsteps)))
        self._check(lib().rds_check(self._ctx))

    def set_option(self, key: str, value: float):
        self._check(lib().rds_set_option(self._ctx, key.encode(), float(value)))

    def stream_handle(self) -> int:
        return lib().rds_stream(self._ctx) or 0

    def kernel_timing(self, enable: bool):
        self._check(lib().rds_kernel_timing(self._ctx, int(enable)))

    def kernel_times(self):
        names = (C.c_char * 32 * 64)()
        ms = np.zeros(64)
        cnt = np.zeros(64, dtype=np.int32)
        n = lib().rds_kernel_times(self._ctx, names, _ptr(ms), _ptr(cnt), 64)
        return {names[i].value.decode(): (float(ms[i]), int(cnt[i])) for i in range(n)}

    def launch_count(self) -> int:
        return int(lib().rds_launch_count(self._ctx))

    def _check(self, st):
        if st != 0:
            msg = lib().rds_last_error(self._ctx).decode() if self._ctx else ""
            raise RDSError(st, msg)

    def close(self):
        if self._ctx:
            lib().rds_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
