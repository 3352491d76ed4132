"""Benchmark of the explicit RDS pseudo-time iteration on B200.

Workload (default): configuration 2 -- 2D inviscid Burgers, [0,1]^2, 512x512 squares split into
P2 triangles (524,288 cells, 1,050,625 nodes), interior jitter 0.15h (seed 7), inflow
u = 1.5 - 2x at y = 0, blended B scheme (PGB), 7-point quadrature, CFL 0.5. A step is one
pseudo-time iteration (assemble_lhs_and_rhs + solve) over the whole mesh.

Metric: cell-residual updates/s = cells x steps / time. Reported:
  value     FP64 plain path, state resident in HBM, L2 flushed before every timed step,
            CUDA events on the library's stream around each step;
  e2e       the same through the reference-facing C ABI with host buffers: every step copies
            the state in from pinned host memory, assembles, solves, reads the residual norm and
            copies the state back out;
  mixed     the mixed-precision path (FP32 interpolation/flux/upwind terms, FP64 accumulation);
  roofline  of the dominant kernel (the cell residual kernel, FP64-bound), against the FP64 FMA
            peak measured on this GPU by the library's micro-kernel, with its HBM fraction;
  cpu_baseline  the reference's own CPU path (oracle/_ref, compiled from the reference sources)
            on a bounded sample of the same workload, all host cores.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
With N > 1 (torchrun), every rank runs its own independent copy of the workload (replicas; the
path has no data exchange between independent problems), timing is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_BYTES = 126 * 2**20
CFL = 0.5
BURGERS_BCS_SPEC = ("WeakDirichlet:inlet:bottom:burgers_inlet,WeakDirichlet:left:left:c1.5,"
                    "WeakDirichlet:right:right:c-0.5")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=512, help="squares per side (512 = configuration 2)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-drop", action="store_true", help="skip the time-to-drop runs")
    ap.add_argument("--drop-max-iter", type=int, default=400000)
    ap.add_argument("--quick", action="store_true",
                    help="only warm-up + timed steps (profiling runs): no e2e, mixed, drop, CPU")
    return ap.parse_args()


def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        import torch

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ------------------------------------------------------------------------------------------------


def build_problem(n):
    from pdekit_b200 import reference_element, workloads

    tables = reference_element.triag_tables(2, 5)
    prob = workloads.tri_problem("burgers", "b", 2, n, 0.15, 7, workloads.BURGERS_BCS, tables)
    u0 = workloads.initial_state(prob, "burgers", workloads.sol_coords_tri(n, 0.15, 7, 2))
    return prob, u0


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        self.out.flush()
        rows = []
        with open(self.out.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


def time_steps(solver, steps, flush):
    """Per-step device time (ms) of `steps` fused iterations, L2 flushed before each step."""
    import torch

    stream = torch.cuda.ExternalStream(solver.stream_handle())
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.zero_()
            ev[k][0].record(stream)
            solver.run(CFL, 1)
            ev[k][1].record(stream)
    stream.synchronize()
    return sum(a.elapsed_time(b) for a, b in ev)


def cpu_reference(n, threads, iters, workdir):
    """Time the reference's own CPU path (oracle/_ref/rds_ref_harness) on the workload's mesh."""
    from pdekit_b200 import meshgen

    harness = os.path.join(ROOT, "oracle", "_ref", "rds_ref_harness")
    if not os.path.exists(harness):
        return None
    msh = os.path.join(workdir, f"burgers_{n}.msh")
    meshgen.write_gmsh22(msh, meshgen.unit_square_tri(n, 0.15, seed=7))
    out = subprocess.run([harness, "time", "burgers", "b", "2", "5", msh, "-", str(iters),
                          str(CFL), "burgers", BURGERS_BCS_SPEC, str(threads)],
                         capture_output=True, text=True, check=True).stdout
    return json.loads(out.strip().splitlines()[-1])


def roofline_cell_kernel(ms_per_launch, ncells, peak_fp64, hbm_gbs):
    """Algorithmic FLOPs and bytes of one launch of the FP64 Burgers P2 PGB cell kernel.

    Per cell (ndof 6, nq 7, nfl 10, affine P1 geometry), counting an FMA as 2 flops:
      flux nodes 10 x (11 + 2) = 130, Jacobian + inverse 28,
      per quadrature point: weights 2, flux divergence 76 + 7, u_q 11, upwind coefficients
      6 x 10, LDA part 2 + 6 x 4, N dissipation 12 + 6 x 6  -> 231, x 7 = 1617,
      blending and output 27            => 1802 flop / cell.
    Bytes per cell (each touched once): dof + vertex indices 9 x 4, coordinates 3 x 16,
      nodal states 6 x 8, contribution writes 6 x 8 + wave speed 8 => 188 B / cell."""
    flop = 1802.0 * ncells
    byts = 188.0 * ncells
    s = ms_per_launch * 1e-3
    achieved = flop / s / 1e12
    return {"bound": "fp64", "achieved": round(achieved, 3), "peak": round(peak_fp64, 3),
            "unit": "TFLOP/s", "frac": round(achieved / peak_fp64, 4),
            "peak_source": "measured in this run: rds_measure_peak (FP64 FMA micro-kernel)",
            "hbm_achieved_gbs": round(byts / s / 1e9, 1), "hbm_peak_gbs": hbm_gbs,
            "hbm_frac": round(byts / s / 1e9 / hbm_gbs, 4),
            "traffic": None, "kernel": "cells_burgers_b", "flop_per_cell": 1802,
            "bytes_per_cell": 188}


def _drop_run(prob, u0, precision, cfl, max_iter, drop=1e-10):
    import torch

    from pdekit_b200.rds import PGRDMethodExplicit

    s = PGRDMethodExplicit(prob.physics, prob.scheme, precision).configure_mesh_data(prob)
    s.initialize_work_data()
    s.set_solution(u0)
    s.iterate(0.1, 3, 0.0)  # builds and uploads the loop graphs outside the timed region
    s.set_solution(u0)
    torch.cuda.synchronize()
    t0 = time.time()
    it, hist = s.iterate(cfl, max_iter, drop, raise_on_cap=False)
    torch.cuda.synchronize()
    sec = time.time() - t0
    rel = float((hist[-1] / hist[0]).max()) if len(hist) else None
    u = s.solution()
    s.close()
    return {"seconds": round(sec, 4), "iterations": int(it), "final_rel_norm": rel,
            "reached": bool(rel is not None and rel <= drop),
            "cell_updates_per_s": prob.ncells * it / sec if sec > 0 else None}, u


def time_to_drop(args, u0_pgb):
    """Time to a 1e-10 drop of max_eq ||res dt|| / ||res dt||(iteration 0), FP64 and mixed.

    configuration 1 (advection P1 64x64, LDA, CFL 0.9) and the configuration-2 mesh with the N
    scheme (Burgers P2 512x512, CFL 0.5) converge to 1e-10; the blended B scheme on the
    configuration-2 mesh stalls near 1e-5 (a property of the scheme's blending on this shock
    problem, reproduced by the reference on smaller meshes), so it is run to a capped iteration
    count and its final drop is reported."""
    from pdekit_b200 import workloads

    out = {}
    cases = [("configuration 1: advection P1 64x64, LDA, CFL 0.9", workloads.config1(64), 0.9,
              args.drop_max_iter),
             (f"configuration-2 mesh with the N scheme: Burgers P2 {args.n}x{args.n}, CFL 0.5",
              workloads.config2(args.n, scheme="n"), 0.5, args.drop_max_iter)]
    for name, (prob, u0), cfl, cap in cases:
        r64, u64 = _drop_run(prob, u0, "fp64", cfl, cap)
        rmx, umx = _drop_run(prob, u0, "mixed", cfl, cap)
        rmx["converged_state_rel_l2_vs_fp64"] = float(np.linalg.norm(umx - u64) /
                                                      np.linalg.norm(u64))
        out[name] = {"cells": prob.ncells, "fp64": r64, "mixed": rmx,
                     "speedup_mixed_vs_fp64": round(r64["seconds"] / rmx["seconds"], 3)}
    prob, u0 = u0_pgb
    r, _ = _drop_run(prob, u0, "fp64", CFL, 4000)
    out[f"configuration 2 (blended B), capped at 4000 iterations"] = {"fp64": r}
    return out


def run_ours(args, rank, world, local):
    import torch

    from pdekit_b200.rds import PGRDMethodExplicit, measure_peak

    torch.cuda.set_device(local)
    prob, u0 = build_problem(args.n)
    ncells = prob.ncells

    solver = PGRDMethodExplicit("burgers", "b", "fp64").configure_mesh_data(prob)
    solver.initialize_work_data()
    solver.set_solution(u0)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")

    # warm-up
    solver.run(CFL, args.warmup)
    torch.cuda.synchronize()
    solver.set_solution(u0)

    launches0 = solver.launch_count()
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t0 = time.time()
        ms = time_steps(solver, args.steps, flush)
        wall = time.time() - t0
    torch.cuda.synchronize()
    barrier(world)
    launches = solver.launch_count() - launches0
    ms = max_over_ranks(ms, world)
    value = ncells * args.steps * world / (ms * 1e-3)

    if args.quick:
        line = {"metric": "cell-residual updates/s", "value": value, "steps": args.steps,
                "ms_per_step": ms / args.steps, "gpu_launches": int(launches), "quick": True}
        solver.close()
        return line

    # per-kernel device time (event timing around every launch, separate pass)
    solver.set_solution(u0)
    solver.kernel_timing(True)
    solver.run(CFL, 50)
    ktimes = solver.kernel_times()
    solver.kernel_timing(False)
    cell_ms, cell_n = ktimes.get("cells_burgers_b", (0.0, 1))
    peak64 = measure_peak("fp64")
    hbm = None
    try:
        hbm = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
    except Exception:
        hbm = 6650.0
    roof = roofline_cell_kernel(cell_ms / cell_n, ncells, peak64, hbm)

    # e2e through the C ABI with host buffers (pinned)
    u_host = torch.from_numpy(np.ascontiguousarray(u0)).pin_memory()
    u_out = torch.empty_like(u_host).pin_memory()
    ke = max(10, args.steps // 10)
    stream = torch.cuda.ExternalStream(solver.stream_handle())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(ke):
        solver.set_solution(u_host.numpy())
        solver.assemble_lhs_and_rhs(CFL)
        solver.solve()
        solver.compute_residual_norm()
        solver.solution(out=u_out.numpy())
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world)
    e2e = {"value": ncells * ke * world / (e2e_ms * 1e-3), "unit": "cell-residual updates/s",
           "h2d_bytes_per_step": int(u_host.numel() * 8),
           "d2h_bytes_per_step": int(u_host.numel() * 8 + 8 * prob.neq), "steps": ke}

    # mixed precision form
    mixed = PGRDMethodExplicit("burgers", "b", "mixed").configure_mesh_data(prob)
    mixed.initialize_work_data()
    mixed.set_solution(u0)
    mixed.run(CFL, args.warmup)
    mixed.set_solution(u0)
    ms_mixed = max_over_ranks(time_steps(mixed, args.steps, flush), world)
    mixed_value = ncells * args.steps * world / (ms_mixed * 1e-3)

    # time to a 1e-10 residual drop, FP64 vs mixed (device loop with the device-side stop test)
    drop = None
    if not args.no_drop and world == 1:
        drop = time_to_drop(args, u0_pgb=(prob, u0))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        with tempfile.TemporaryDirectory() as td:
            r = cpu_reference(args.n, threads, 10, td)
        if r:
            cpu = {"value": r["cell_updates_per_s"], "unit": "cell-residual updates/s",
                   "cores": threads, "kind": "reference",
                   "sample": f"reference PGRDMethodExplicit<Cart2D, Burgers2D, PGB> on the same "
                             f"{args.n}x{args.n} P2 mesh, {r['iters']} iterations after one "
                             f"warm-up assemble, nb_threads={threads}"}

    line = {
        "metric": "cell-residual updates/s", "value": value, "unit": "cell-residual updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "configuration 2: Burgers P2 triangles 512x512 (524,288 cells, "
                               "1,050,625 nodes), blended B scheme, 7-point rule, CFL 0.5",
                   "cells": ncells, "nodes": prob.nnodes,
                   "l2": "flushed (256 MB write) before every timed step",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "e2e": e2e,
        "mixed": {"value": mixed_value, "ms_per_step": ms_mixed / args.steps,
                  "dtype": "f32 interpolation/flux/upwind, f64 accumulation/inverse/norms"},
        "time_to_drop_1e-10": drop,
        "roofline": roof,
        "kernels_ms_per_launch": {k: round(v[0] / v[1], 5) for k, v in ktimes.items()},
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "gpu_launches": int(launches),
        "wall_s_timed_region": round(wall, 3),
    }
    solver.close()
    mixed.close()
    return line


def run_reference(args, rank, world):
    """The reference's own CPU implementation of the path (oracle/_ref) on the host cores."""
    if rank != 0:
        return None
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as td:
        t0 = time.time()
        r = cpu_reference(args.n, threads, max(1, args.steps // 50), td)
        wall = time.time() - t0
    if r is None:
        return {"impl": "reference", "unavailable": "oracle/_ref/rds_ref_harness not built"}
    v = r["cell_updates_per_s"]
    return {"impl": "reference", "metric": "cell-residual updates/s", "value": v,
            "unit": "cell-residual updates/s", "n_gpus": world, "steps": r["iters"],
            "warmup": 1, "ms_per_step": r["seconds"] / r["iters"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "configuration 2: Burgers P2 triangles 512x512 (524,288 "
                                   "cells), blended B scheme, 7-point rule, CFL 0.5",
                       "cells": r["cells"], "nodes": r["nodes"]},
            "cpu_baseline": {"value": v, "unit": "cell-residual updates/s", "cores": threads,
                             "kind": "reference",
                             "sample": f"{r['iters']} iterations of the full mesh, "
                                       f"nb_threads={threads}"},
            "e2e": {"value": v, "unit": "cell-residual updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "wall_s": round(wall, 2)}


def main():
    args = parse()
    rank, world, local = dist_setup(args)
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    else:
        line = run_ours(args, rank, world, local)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
