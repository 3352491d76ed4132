"""Partitioned single mesh: one problem's cells split over ranks (one GPU each), with one
exchange of nodal partial sums per pseudo-time iteration.

The reference runs one mesh per process (its thread pool splits the cell loop,
src/solver/rdm/PGRDMethodExplicit.hpp:270-298). Here the cells are cut into slabs along x of
equal estimated work; each rank builds a context over its cells and the nodes they touch
(renumbered), and every weak boundary facet goes to the lowest rank that holds all of its dofs.
A node that several ranks hold (an interface node) receives partial sums of the residual and of
the wave speed on each of them; per iteration

    rds_assemble_rhs          cells and facets of this rank -> partial res, ws
    rds_pack_interface        partial sums of the interface nodes -> exchange buffer
    sum over the ranks        (NCCL all-reduce of the buffer on the context's stream)
    rds_unpack_interface      full sums back into res, ws
    rds_finish                dt = CFL V / ws, u -= dt res, sum over owned nodes of (res dt)^2
    sum over the ranks        (all-reduce of NEQ doubles) -> norm = sqrt(sum / N)

so every rank updates its copy of an interface node from the same sums. The dual volumes of the
interface nodes are summed over the ranks once, the same way. Results equal the single-context
ones up to the order in which the partial sums of interface nodes are added (rounding).
Strong Dirichlet conditions are not supported in this form (each rank would have to write its
copies of the shared dofs the same way).

The exchange overlaps the interior of the mesh: each rank numbers its interface nodes first and
splits every cell group into the cells touching an interface node and the rest, so that

    interface cells + facets, sums of the interface nodes, pack      (rds_assemble_rhs_cells,
                                                                      rds_gather_rhs)
    sum over the ranks of the buffer  ||  interior cells; the other nodes' sums, dt, update and
                                          norm parts                 (rds_gather_finish)
    unpack, finish of the interface nodes, norm parts of the rank    (rds_finish_nodes)
    sum over the ranks of the norm parts

and a step (its NCCL calls included) is captured once in a CUDA graph and replayed.
"""

from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from .problem import CellGroup, Problem
from .rds import PGRDMethodExplicit, _ptr, lib


@dataclasses.dataclass
class RankPart:
    rank: int
    problem: Problem  # local problem (local node numbering, full geometry coordinates)
    nodes: np.ndarray  # [n_local] global node number of each local node
    if_nodes: np.ndarray  # [n_if] local numbers of the interface nodes
    if_slots: np.ndarray  # [n_if] their slots in the exchange buffer
    owned: np.ndarray  # [n_local] uint8, 1 where this rank counts the node in the norm
    cells: list  # per group: global cell indices of this rank (ascending)
    n_if_groups: int = 0  # local groups [0, n_if_groups) hold the cells touching interface nodes


@dataclasses.dataclass
class Partition:
    parts: list  # RankPart per rank
    nslots: int  # exchange-buffer entries (interface nodes of the whole mesh)
    nnodes: int  # global node count


def _cell_work(g: CellGroup) -> float:
    return float(g.ndof * g.nq)


def partition(prob: Problem, nparts: int) -> Partition:
    """Split the cells of `prob` into `nparts` slabs along x of equal estimated work."""
    if any(b.kind == "StrongDirichlet" for b in prob.bcs):
        raise NotImplementedError("partitioned problems: weak boundary conditions only")
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    xs, ws = [], []
    for g in prob.groups:
        xs.append(prob.geo_coords[g.geo_conn][:, :, 0].mean(axis=1))
        ws.append(np.full(g.ncells, _cell_work(g)))
    x = np.concatenate(xs)
    w = np.concatenate(ws)
    order = np.argsort(x, kind="stable")
    cum = np.cumsum(w[order])
    cut = np.searchsorted(cum, cum[-1] * np.arange(1, nparts) / nparts, side="left")
    rank_of = np.empty(len(x), dtype=np.int64)
    bounds = zip(np.concatenate([[0], cut]), np.concatenate([cut, [len(x)]]))
    for r, (lo, hi) in enumerate(bounds):
        rank_of[order[lo:hi]] = r
    offs = np.cumsum([0] + [g.ncells for g in prob.groups])

    # nodes of every rank, interface nodes and their slots, the owner of every node
    node_sets = []
    for r in range(nparts):
        ns = [g.sol_conn[rank_of[offs[ig]:offs[ig + 1]] == r].ravel()
              for ig, g in enumerate(prob.groups)]
        node_sets.append(np.unique(np.concatenate(ns)))
    count = np.zeros(prob.nnodes, dtype=np.int64)
    first = np.full(prob.nnodes, nparts, dtype=np.int64)
    for r, ns in enumerate(node_sets):
        count[ns] += 1
        first[ns] = np.minimum(first[ns], r)
    iface = np.flatnonzero(count > 1)
    slot_of = np.full(prob.nnodes, -1, dtype=np.int64)
    slot_of[iface] = np.arange(len(iface))

    # the lowest rank that holds all dofs of a facet computes it
    holder = []
    for b in prob.bcs:
        h = np.full(b.nfacets, nparts, dtype=np.int64)
        for r, ns in enumerate(node_sets):
            has = np.isin(b.sol_conn, ns).all(axis=1)
            h = np.where(has & (h == nparts), r, h)
        holder.append(h)

    is_if = np.zeros(prob.nnodes, dtype=bool)
    is_if[iface] = True
    parts = []
    for r, ns in enumerate(node_sets):
        # local numbering: this rank's interface nodes first
        ns = np.concatenate([ns[is_if[ns]], ns[~is_if[ns]]])
        loc = np.full(prob.nnodes, -1, dtype=np.int64)
        loc[ns] = np.arange(len(ns))
        groups_if, groups_in, cells = [], [], []
        for ig, g in enumerate(prob.groups):
            cid = np.flatnonzero(rank_of[offs[ig]:offs[ig + 1]] == r)
            cells.append(cid)
            touch = is_if[g.sol_conn[cid]].any(axis=1)
            for sel, out in ((cid[touch], groups_if), (cid[~touch], groups_in)):
                if len(sel):
                    out.append(dataclasses.replace(
                        g, sol_conn=loc[g.sol_conn[sel]].astype(np.int32),
                        geo_conn=np.ascontiguousarray(g.geo_conn[sel])))
        groups = groups_if + groups_in
        bcs = []
        for b, h in zip(prob.bcs, holder):
            fid = np.flatnonzero(h == r)
            if len(fid) == 0:
                continue
            gq = np.ascontiguousarray(b.gq[fid]) if b.kind == "WeakDirichlet" else b.gq
            bcs.append(dataclasses.replace(
                b, sol_conn=loc[b.sol_conn[fid]].astype(np.int32),
                geo_conn=np.ascontiguousarray(b.geo_conn[fid]), gq=gq))
        local = Problem(physics=prob.physics, scheme=prob.scheme, dim=prob.dim, neq=prob.neq,
                        nnodes=len(ns), geo_coords=prob.geo_coords, groups=groups, bcs=bcs,
                        adv=prob.adv, gamma=prob.gamma)
        n_if = int(is_if[ns].sum())
        ifl = np.arange(n_if)
        parts.append(RankPart(rank=r, problem=local, nodes=ns,
                              if_nodes=ifl.astype(np.int32),
                              if_slots=slot_of[ns[ifl]].astype(np.int32),
                              owned=(first[ns] == r).astype(np.uint8), cells=cells,
                              n_if_groups=len(groups_if)))
    return Partition(parts=parts, nslots=len(iface), nnodes=prob.nnodes)


class RankSolver:
    """The context of one rank of a partitioned problem, driven phase by phase (a multi-rank
    driver interleaves the phases with the sums over the ranks)."""

    def __init__(self, part: RankPart, nslots: int, precision: str = "fp64"):
        import torch

        self.part = part
        p = part.problem
        self.solver = PGRDMethodExplicit(p.physics, p.scheme, precision).configure_mesh_data(p)
        self.solver.initialize_work_data()
        self.nslots = nslots
        dev = torch.device("cuda", torch.cuda.current_device())
        self.buf = torch.zeros((max(nslots, 1), p.neq + 1), dtype=torch.float64, device=dev)
        self.sq = torch.zeros(p.neq, dtype=torch.float64, device=dev)
        self.stream = torch.cuda.ExternalStream(self.solver.stream_handle())
        torch.cuda.synchronize()  # the buffers exist before the context's stream uses them

    def _check(self, st):
        self.solver._check(st)

    def local_volume(self):
        return self.solver.fields()[3]

    def set_volume(self, vol):
        """The dual volumes summed over the ranks, and the interface of this rank."""
        vol = np.ascontiguousarray(vol, dtype=np.float64)
        self._check(lib().rds_set_dual_volume(self.solver._ctx, _ptr(vol)))
        p = self.part
        nodes = np.ascontiguousarray(p.if_nodes, dtype=np.int32)
        slots = np.ascontiguousarray(p.if_slots, dtype=np.int32)
        owned = np.ascontiguousarray(p.owned, dtype=np.uint8)
        self._check(lib().rds_set_interface(self.solver._ctx, len(nodes), _ptr(nodes), _ptr(slots),
                                            self.nslots, _ptr(owned)))

    def set_solution(self, u_global):
        self.solver.set_solution(np.asarray(u_global).reshape(-1, self.part.problem.neq)[
            self.part.nodes])

    def assemble_interface(self):
        """Cells touching interface nodes and the boundary facets, the sums of the interface
        nodes (this rank's parts), those into self.buf."""
        ctx, p = self.solver._ctx, self.part
        if len(p.if_nodes) == 0:
            return  # the facets then run beside the interior cells
        self._check(lib().rds_assemble_rhs_cells(ctx, 0, p.n_if_groups, 1))
        self._check(lib().rds_gather_rhs(ctx, 0, len(p.if_nodes)))
        self._check(lib().rds_pack_interface(ctx, C.c_void_p(self.buf.data_ptr())))

    def assemble_interior(self, cfl: float, norm: bool = True):
        """The other cells, and the other nodes (complete on this rank) finished: their sums,
        dt, update and block sums of (res dt)^2."""
        ctx, p = self.solver._ctx, self.part
        alone = len(p.if_nodes) == 0
        self._check(lib().rds_assemble_rhs_cells(ctx, p.n_if_groups, len(p.problem.groups),
                                                 int(alone)))
        # a rank without interface nodes has its norm part here (no finish after the exchange)
        sq = C.c_void_p(self.sq.data_ptr()) if alone and norm else None
        self._check(lib().rds_gather_finish(ctx, len(p.if_nodes), p.problem.nnodes, float(cfl),
                                            sq))

    # ---- RK3TVD stages (the stage state and residual selected by rk_select)
    def rk_select(self, stage: int):
        """Stage 1-3: the following phases read u_n, u_1, u_2 and write the stage residual;
        0: back to the context's own state and residual."""
        self._check(lib().rds_rk_stage_state(self.solver._ctx, int(stage)))

    def rk_interior(self, cfl: float):
        """The other cells, and the other nodes' sums ending in the stage combination."""
        ctx, p = self.solver._ctx, self.part
        alone = len(p.if_nodes) == 0
        self._check(lib().rds_assemble_rhs_cells(ctx, p.n_if_groups, len(p.problem.groups),
                                                 int(alone)))
        self._check(lib().rds_gather_rk(ctx, len(p.if_nodes), p.problem.nnodes, float(cfl)))

    def rk_interface(self, cfl: float):
        """After the exchange: the interface nodes' summed residual and their combination."""
        ctx, n_if = self.solver._ctx, len(self.part.if_nodes)
        if n_if:
            self._check(lib().rds_unpack_interface(ctx, C.c_void_p(self.buf.data_ptr())))
            self._check(lib().rds_combine_rk(ctx, 0, n_if, float(cfl)))

    def assemble_and_pack(self, cfl: float):
        """This rank's partial sums at the interface nodes into self.buf, the other nodes
        finished."""
        self.assemble_interface()
        self.assemble_interior(cfl)

    def unpack_and_finish(self, cfl: float, norm: bool = True):
        """Full sums of the interface nodes from self.buf, their dt and update, and (norm)
        this rank's norm part (all its owned nodes) into self.sq."""
        ctx, n_if = self.solver._ctx, len(self.part.if_nodes)
        if n_if == 0:
            return  # norm part already summed by assemble_interior
        self._check(lib().rds_unpack_interface(ctx, C.c_void_p(self.buf.data_ptr())))
        sq = C.c_void_p(self.sq.data_ptr()) if norm else None
        self._check(lib().rds_finish_nodes(ctx, float(cfl), 1, 0, n_if, sq))

    def check(self):
        self._check(lib().rds_check(self.solver._ctx))

    def solution(self):
        return self.solver.solution()

    def close(self):
        self.solver.close()


class PartitionedRDS:
    """This rank's part of a problem split over a torch.distributed process group (NCCL, one
    GPU per rank): the exchange buffer and the norm parts are summed with all-reduces on the
    context's stream. Without a process group (one rank) the sums are the rank's own values."""

    def __init__(self, prob: Problem, rank: int, world: int, precision: str = "fp64",
                 group=None):
        import torch
        import torch.distributed as dist

        if dist.is_initialized():
            self._sum = lambda t: dist.all_reduce(t, group=group)
            self._sum_async = lambda t: dist.all_reduce(t, group=group, async_op=True)
            # collectives of other backends (gloo: through the host) cannot be captured
            self._graphs_ok = dist.get_backend(group) == "nccl"
        else:
            self._sum = lambda t: None
            self._sum_async = lambda t: None
            self._graphs_ok = True
        self._graphs = {}  # (cfl, norm) -> (CUDA graph of one step, kernel launches per step)
        self.graph_launches = 0  # kernel launches replayed through the graphs
        self.partition = partition(prob, world)
        part = self.partition.parts[rank]
        self.rank = RankSolver(part, self.partition.nslots, precision)
        idx = torch.as_tensor(part.nodes, device="cuda")
        vol = torch.zeros(prob.nnodes, dtype=torch.float64, device="cuda")
        vol[idx] = torch.as_tensor(self.rank.local_volume(), device="cuda")
        self._sum(vol)
        self.rank.set_volume(vol[idx].cpu().numpy())
        self.nnodes = prob.nnodes

    def set_solution(self, u_global):
        self.rank.set_solution(u_global)

    def step(self, cfl: float, norm: bool = True):
        """One pseudo-time iteration, enqueued: the interface cells and sums, the sum of the
        exchange buffer over the ranks while the interior cells run, then unpack, finish and
        (norm) the sum of the norm parts (they stay on the device, self.rank.sq)."""
        import torch

        with torch.cuda.stream(self.rank.stream):
            self.rank.assemble_interface()
            work = self._sum_async(self.rank.buf) if self.partition.nslots else None
            self.rank.assemble_interior(cfl, norm)
            if work is not None:
                work.wait()
            self.rank.unpack_and_finish(cfl, norm)
            if norm:
                self._sum(self.rank.sq)

    def rk3tvd_step(self, cfl: float):
        """One RK3TVD step (RK3TVD::advance_in_time), enqueued: per stage the interface cells
        and sums, their sum over the ranks while the interior cells run and finish their stage
        combination, then the interface nodes' combination."""
        import torch

        r = self.rank
        with torch.cuda.stream(r.stream):
            for k in (1, 2, 3):
                r.rk_select(k)
                r.assemble_interface()
                work = self._sum_async(r.buf) if self.partition.nslots else None
                r.rk_interior(cfl)
                if work is not None:
                    work.wait()
                r.rk_interface(cfl)
            r.rk_select(0)

    def graph_rk3tvd(self, cfl: float, nsteps: int = 1):
        """nsteps rk3tvd_step through a CUDA graph of one step (captured at the first call for
        this cfl, NCCL calls included); eager where capture is not possible."""
        import torch

        for _ in range(nsteps):
            if not self._graphs_ok:
                self.rk3tvd_step(cfl)
                continue
            key = ("rk3tvd", cfl)
            if key not in self._graphs:
                self.rank.rk_select(0)  # allocates the stage buffers outside the capture
                stream = self.rank.stream
                stream.synchronize()
                n0 = self.rank.solver.launch_count()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=stream):
                    self.rk3tvd_step(cfl)
                self._graphs[key] = (g, self.rank.solver.launch_count() - n0)
            g, n = self._graphs[key]
            with torch.cuda.stream(self.rank.stream):
                g.replay()
            self.graph_launches += n

    def graph_step(self, cfl: float, norm: bool = True):
        """step() through a CUDA graph of one step, captured at the first call for this
        (cfl, norm) (NCCL collectives included) and replayed after; eager where capture is not
        possible."""
        import torch

        if not self._graphs_ok:
            self.step(cfl, norm)
            return
        key = (cfl, norm)
        if key not in self._graphs:
            stream = self.rank.stream
            stream.synchronize()
            n0 = self.rank.solver.launch_count()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=stream):
                self.step(cfl, norm)
            self._graphs[key] = (g, self.rank.solver.launch_count() - n0)
            # the capture ran nothing: the replay below takes the step
        g, n = self._graphs[key]
        with torch.cuda.stream(self.rank.stream):
            g.replay()
        self.graph_launches += n

    def norm(self):
        """sqrt(sum_n (res dt)^2 / N) per equation of the last step."""
        self.rank.stream.synchronize()
        return np.sqrt(self.rank.sq.cpu().numpy() / self.nnodes)

    def iterate(self, cfl: float, max_iter: int, drop: float = 0.0, check_every: int = 16):
        """Up to max_iter steps, stopping at max_eq norm / norm(first step) <= drop (tested
        at the first step and every `check_every` steps); returns (iterations, last norm)."""
        n0 = None
        it = 0
        while it < max_iter:
            self.graph_step(cfl)
            it += 1
            if it == 1 or it % check_every == 0 or it == max_iter:
                nrm = self.norm()
                if not np.all(np.isfinite(nrm)):
                    raise FloatingPointError("non-finite residual norm")
                if n0 is None:
                    n0 = nrm
                if drop > 0 and np.max(nrm / n0) <= drop:
                    break
        self.rank.check()
        return it, self.norm()

    def solution_global(self):
        """The full state (summed over the ranks from the owners' copies)."""
        import torch

        part = self.rank.part
        u = torch.zeros((self.nnodes, part.problem.neq), dtype=torch.float64, device="cuda")
        mine = torch.as_tensor(self.rank.solution(), device="cuda")
        own = torch.as_tensor(part.owned.astype(bool), device="cuda")
        idx = torch.as_tensor(part.nodes, device="cuda")
        u[idx[own]] = mine[own]
        self._sum(u)
        return u.cpu().numpy()

    def close(self):
        self._graphs = {}  # before the process group goes (a graph may hold NCCL calls)
        self.rank.close()


def emulate(prob: Problem, nparts: int, u0, cfl: float, iters: int, precision: str = "fp64"):
    """All ranks of a partitioned problem in one process on one GPU: the phases of every rank
    in turn, the sums over the ranks done between them with the device synchronised (no rank
    ever waits for another on the device). Returns (global state after `iters` steps,
    norms [iters, neq])."""
    import torch

    pt = partition(prob, nparts)
    ranks = [RankSolver(p, pt.nslots, precision) for p in pt.parts]
    vol = np.zeros(prob.nnodes)
    for r in ranks:
        vol[r.part.nodes] += r.local_volume()
    for r in ranks:
        r.set_volume(vol[r.part.nodes])
        r.set_solution(u0)
    norms = np.zeros((iters, prob.neq))
    for it in range(iters):
        for r in ranks:
            r.assemble_and_pack(cfl)
        torch.cuda.synchronize()
        total = sum(r.buf for r in ranks)
        for r in ranks:
            r.buf.copy_(total)
        torch.cuda.synchronize()
        for r in ranks:
            r.unpack_and_finish(cfl)
        torch.cuda.synchronize()
        norms[it] = np.sqrt(sum(r.sq for r in ranks).cpu().numpy() / prob.nnodes)
    for r in ranks:
        r.check()
    u = np.zeros((prob.nnodes, prob.neq))
    for r in ranks:
        own = r.part.owned.astype(bool)
        u[r.part.nodes[own]] = r.solution()[own]
    for r in ranks:
        r.close()
    return u, norms


def emulate_rk3tvd(prob: Problem, nparts: int, u0, cfl: float, nsteps: int,
                   precision: str = "fp64"):
    """RK3TVD steps of a partitioned problem with all ranks in one process on one GPU (as
    `emulate`: every rank's phases in turn, the sums between them with the device synchronised).
    Returns the global state after `nsteps` steps."""
    import torch

    pt = partition(prob, nparts)
    ranks = [RankSolver(p, pt.nslots, precision) for p in pt.parts]
    vol = np.zeros(prob.nnodes)
    for r in ranks:
        vol[r.part.nodes] += r.local_volume()
    for r in ranks:
        r.set_volume(vol[r.part.nodes])
        r.set_solution(u0)
    for _ in range(nsteps):
        for k in (1, 2, 3):
            for r in ranks:
                r.rk_select(k)
                r.assemble_interface()
                r.rk_interior(cfl)
            torch.cuda.synchronize()
            if pt.nslots:
                total = sum(r.buf for r in ranks)
                for r in ranks:
                    r.buf.copy_(total)
            torch.cuda.synchronize()
            for r in ranks:
                r.rk_interface(cfl)
        for r in ranks:
            r.rk_select(0)
    torch.cuda.synchronize()
    for r in ranks:
        r.check()
    u = np.zeros((prob.nnodes, prob.neq))
    for r in ranks:
        own = r.part.owned.astype(bool)
        u[r.part.nodes[own]] = r.solution()[own]
    for r in ranks:
        r.close()
    return u

