"""Benchmark of the explicit RDS pseudo-time iteration on B200.

Workloads (--workload, default c2):
  c1  constant advection, P1 triangles 64x64 (8,192 cells), LDA, 6-point rule, CFL 0.9
  c2  Burgers, P2 triangles 512x512 (524,288 cells, 1,050,625 nodes), jitter 0.15h, blended B
      scheme, 7-point rule, CFL 0.5 (the default, the configuration the metric is quoted on)
  c3  Euler 2D bump channel, 500k P3 triangles (16-point rule) + 500k P3 quadrilaterals (5x5
      rule), 6,756,001 nodes, blended B scheme, Mach 0.5, CFL 0.5
  c4  Euler 3D bump box, 786,432 P2 tetrahedra (14-point rule), 1,085,825 nodes, LDA, Mach 0.6
  c5  256 independent advection / Burgers problems (P1-P3 triangles, 1k-200k cells each, own
      CFL) in one context: batched persistent launches, every problem to its own 1e-10 drop
A step of c1-c4 is one pseudo-time iteration (assemble_lhs_and_rhs + solve) over the whole
mesh; a step of c5 is one batched iteration over the problems still iterating.

Metric: cell-residual updates/s = cells x steps / time. Reported:
  value     FP64 plain path, state resident in HBM, L2 flushed before every timed step, CUDA
            events on the library's stream around each step (c5: the batched FP64 loop to the
            1e-10 drop of every problem);
  e2e       the same through the reference-facing C ABI with host buffers: every step copies
            the state in from pinned host memory, assembles, solves, reads the residual norm and
            copies the state back out (rds_step_host: consecutive steps' copies and iterations
            overlap; the synchronous call sequence is reported beside it);
  mixed     the mixed-precision path (FP32 interpolation/flux/upwind terms, FP64 accumulation);
  roofline  of the dominant kernel (the cell residual kernel, FP64-bound), against the FP64 FMA
            peak measured on this GPU by the library's micro-kernel, with its HBM fraction;
  cpu_baseline  the reference's own CPU path (oracle/_ref, compiled from the reference sources)
            on a bounded sample of the same workload, all host cores.

  python bench.py [--workload c1..c5] [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
With N > 1 (torchrun), every rank runs its own independent copy of c1-c4 (replicas, weak
scaling), or with --partition the one mesh split over the ranks with the interface sums
all-reduced every iteration (strong scaling); c5's problems are split over the ranks by
estimated work (strong scaling). Timing is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_BYTES = 126 * 2**20

ADV_SPEC = "WeakDirichlet:inlet_bottom:bottom:sin2pix,WeakDirichlet:inlet_left:left:zero"
BURGERS_SPEC = ("WeakDirichlet:inlet:bottom:burgers_inlet,WeakDirichlet:left:left:c1.5,"
                "WeakDirichlet:right:right:c-0.5")
EULER2D_SPEC = ("WeakWall:bottom_wall_bc:bottom_wall:-,WeakWall:top_wall_bc:top_wall:-,"
                "WeakSubInlet:inlet_bc:inlet:total_temperature=307.6488978;"
                "total_pressure=120195.4453,WeakSubOutlet:outlet_bc:outlet:total_pressure=101325.0")
EULER3D_SPEC = ("WeakWall:bottom_wall_bc:bottom_wall:-,WeakWall:top_wall_bc:top_wall:-,"
                "WeakWall:side_walls_bc:side_walls:-,"
                "WeakSubInlet:inlet_bc:inlet:total_temperature=307.6488978;"
                "total_pressure=120195.4453,WeakSubOutlet:outlet_bc:outlet:total_pressure=101325.0")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="timed steps (default per workload)")
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5"])
    ap.add_argument("--n", type=int, default=512, help="c2: squares per side (512)")
    ap.add_argument("--c5-nprob", type=int, default=256, help="c5: number of problems (256)")
    ap.add_argument("--c5-sequential", action="store_true",
                    help="c5: also time every problem alone through the plain FP64 path")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-drop", action="store_true", help="skip the time-to-drop runs")
    ap.add_argument("--no-configs", action="store_true",
                    help="c2: skip the compact records of configurations 1, 3, 4 and 5")
    ap.add_argument("--drop-max-iter", type=int, default=400000)
    ap.add_argument("--quick", action="store_true",
                    help="only warm-up + timed steps (profiling runs): no e2e, mixed, drop, CPU")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="--quick: precision of the timed steps")
    ap.add_argument("--tensor-cores", action="store_true",
                    help="mixed cells with the basis contractions on the tensor cores")
    ap.add_argument("--stab", default=None, choices=["av", "lf", "wj", "visc"],
                    help="also time the steps with a stabilisation field computed on the device "
                         "(av: artificial viscosity, read by PGLDA; lf / wj / visc: LF_Blend / "
                         "WongJansen / ViscosityIndicator blending coefficient, read by PGB) and "
                         "the operator that computes it")
    ap.add_argument("--partition", action="store_true",
                    help="c1-c4: split the one mesh over the ranks (interface sums all-reduced "
                         "every iteration, strong scaling) instead of one replica per rank")
    return ap.parse_args()


def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

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


def sum_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ------------------------------------------------------------------------------------------------
# Algorithmic work per cell of the cell-residual kernels (FMA = 2 flops)
# ------------------------------------------------------------------------------------------------


def scalar_flops(physics, scheme, ndof, nq, nfl):
    """Scalar 2D kernel on straight-sided triangles (affine geometry), in the form the kernel
    evaluates (flux contracted with invJ once per flux node, k_n = dV0 A + dV1 B):
      flux nodes  nfl x (2 ndof - 1 + 2 + 6)        state at the node, flux, G0/G1 = invJ^T F
      geometry    28                                Jacobian, determinant, inverse
      per point   4 nfl - 1 + 4                     flux divergence, weight, volume, Phi
                  + (2 ndof - 1 for Burgers)        advection speed u_q
                  + 6 + 6 ndof + 3                  A, B; k_n, K+, max |k|, sum K+; 1/sum, e
                  + 2 ndof                          LDA part
                  + (7 ndof for N / B)              N dissipation (O(ndof) form)
      end         27 for B (blending), 5 otherwise
    Configuration 2 (Burgers P2 B, ndof 6, nq 7, nfl 10): 1,316 flop; configuration 1
    (advection P1 LDA, ndof 3, nq 6, nfl 6): 471 flop."""
    fl = nfl * (2 * ndof - 1 + 2 + 6) + 28
    per_q = 4 * nfl - 1 + 4 + 6 + 6 * ndof + 3 + 2 * ndof
    if physics == "burgers":
        per_q += 2 * ndof - 1
    if scheme != "lda":
        per_q += 7 * ndof
    return fl + nq * per_q + (27 if scheme == "b" else 5)


def euler_flops(dim, neq, ndof, nq, nfl, ngeo, scheme, const_jac=None):
    """Count of one Euler cell in the algorithm the kernel evaluates, each quantity counted once
    (the kernel's second evaluation of the upwind factors and point states in its node pass is
    not counted):
      geometry    (1 if const_jac else nq) (2 D^2 ngeo + c_invJ)      c_invJ 10 (2D) / 60 (3D)
      flux nodes  nfl (2 NEQ ndof + c_props + c_flux                  state, properties, flux
                       + 2 NEQ D^2 if const_jac)                      flux contracted with invJ
      points      nq (2 NEQ ndof                                      u_q
                      + 2 NEQ D nfl (const_jac) or 2 NEQ D (D nfl + D)  flux divergence
                      + c_props + c_ac + c_solve + 2)                 state, acoustic factors,
                                                                      (sum K+)^-1 [r, sum K+ u]
      point-node  nq ndof (2 D^2 + c_F + 4 NEQ^2 + NEQ + 11 NEQ       grad phi, upwind factors,
                           + 24 NEQ for N / B)                        sum K+, K+ v (factored),
                                                                      sum K+ du, K+ (u - u_bar)
      c_props 20 / 22, c_flux 12 / 24, c_ac 15 / 17, c_F 58 / 69, c_solve 190 (adjugate) / 165
      (LU) for 2D / 3D. const_jac defaults to straight-sided simplices.
    Configuration 3: 54,786 (P3 triangle, 16 points) and 144,325 (P3 quadrilateral on the bump,
    25 points); configuration 4: 52,116 (P2 tetrahedron, 14 points, LDA)."""
    if const_jac is None:
        const_jac = (dim == 2 and ngeo == 3) or (dim == 3 and ngeo == 4)
    c_invj, c_props, c_flux, c_ac, c_f, c_solve = (10, 20, 12, 15, 58, 190) if dim == 2 else \
        (60, 22, 24, 17, 69, 165)
    f = (1 if const_jac else nq) * (2 * dim * dim * ngeo + c_invj)
    f += nfl * (2 * neq * ndof + c_props + c_flux + (2 * neq * dim * dim if const_jac else 0))
    per_q = 2 * neq * ndof
    per_q += 2 * neq * dim * nfl if const_jac else 2 * neq * dim * (dim * nfl + dim)
    per_q += c_props + c_ac + c_solve + 2
    per_qn = 2 * dim * dim + c_f + 4 * neq * neq + neq + 11 * neq
    if scheme != "lda":
        per_qn += 24 * neq
    return f + nq * per_q + nq * ndof * per_qn


def dc_flops(physics, scheme, ndof, nq, nfl):
    """FP32 correction-sweep kernel of the mixed form's defect-correction loop
    (rds_cells_scalar_dc.cu), per straight-sided triangle:
      geometry    28
      flux nodes  nfl x (2 ndof - 1 + 6 + (2 (ndof - 1) + 4 for Burgers, 2 for advection))
                                                  change of the state and flux, contracted
      points      nq (4 nfl - 1)                  change of the flux divergence
                  + nq (1 + 6 + 3 ndof + ndof + 1 + 2 ndof)    w detJ, A, B, k_n, sum K+, e,
                                                               the K+_n e c accumulation
                  + nq (2 (ndof - 1) + 1) for Burgers           u_q of the reference state
                  + nq (1) for LDA, nq (2 (ndof - 1) + 3 + 2 ndof) + 3 ndof for N / B
    Configuration-2 mesh with the N scheme (ndof 6, nq 7, nfl 10): 1,189 flop."""
    fl = 28
    per_f = 2 * ndof - 1 + 6 + (2 * (ndof - 1) + 4 if physics == "burgers" else 2)
    fl += nfl * per_f + nq * (4 * nfl - 1)
    per_q = 1 + 6 + 3 * ndof + ndof + 1 + 2 * ndof
    if physics == "burgers":
        per_q += 2 * (ndof - 1) + 1
    per_q += 1 if scheme == "lda" else 2 * (ndof - 1) + 3 + 2 * ndof
    fl += nq * per_q
    if scheme != "lda":
        fl += 3 * ndof
    return fl


def cell_bytes(dim, neq, ndof, ngeo):
    """Bytes one cell of the residual kernel moves once: dof and vertex indices, vertex
    coordinates, nodal states, its contributions and its wave speed."""
    return ndof * 4 + ngeo * 4 + ngeo * dim * 8 + 2 * ndof * neq * 8 + 8


def group_work(prob):
    flop = byts = 0.0
    for g in prob.groups:
        if prob.physics in ("advconst", "burgers"):
            f = scalar_flops(prob.physics, prob.scheme, g.ndof, g.nq, g.nfl)
        else:
            f = euler_flops(prob.dim, prob.neq, g.ndof, g.nq, g.nfl, g.ngeo, prob.scheme)
        flop += f * g.ncells
        byts += cell_bytes(prob.dim, prob.neq, g.ndof, g.ngeo) * g.ncells
    return flop, byts


# DRAM bytes (read + write) per launch of the dominant cell kernel(s) of a workload, from one ncu
# capture of the same kernel (cold caches between replays); the summary files give the command.
PROFILED_TRAFFIC = {
    "c1": (0.30771e6, "profiles/dram_traffic_cell_kernels.md"),
    "c2": (31.508736e6 + 0.380416e6, "profiles/cells_burgers_b_p2_512.md"),
    "c3": ((102.96 + 119.78 + 192.94 + 217.37) * 1e6,  # both groups, per iteration
           "profiles/cells_euler_c3_c4.md"),
    "c4": ((91.06 + 268.62) * 1e6, "profiles/cells_euler_c3_c4.md"),
}


def roofline(kernel, ms_per_launch, flop, byts, peak_fp64, hbm_gbs):
    s = ms_per_launch * 1e-3
    achieved = flop / s / 1e12
    return {"bound": "fp64", "achieved": round(achieved, 3), "peak": round(peak_fp64, 3),
            "unit": "TFLOP/s", "frac": round(achieved / peak_fp64, 4),
            "peak_source": "measured in this run: rds_measure_peak (FP64 FMA micro-kernel)",
            "hbm_achieved_gbs": round(byts / s / 1e9, 1), "hbm_peak_gbs": hbm_gbs,
            "hbm_frac": round(byts / s / 1e9 / hbm_gbs, 4), "traffic": None, "kernel": kernel,
            "flop_per_launch": flop, "bytes_per_launch": byts}


def hbm_peak():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
    except Exception:
        return 6650.0


# ------------------------------------------------------------------------------------------------
# Workloads
# ------------------------------------------------------------------------------------------------


def workload(name, args):
    """(problem, initial state, CFL, description, default steps, CPU-sample spec)."""
    from pdekit_b200 import workloads as W

    if name == "c1":
        prob, u0 = W.config1(64)
        return (prob, u0, 0.9, "configuration 1: advection P1 triangles 64x64 (8,192 cells), LDA, "
                "6-point rule, CFL 0.9", 20000,
                dict(mesh=("square", 64, 0.2, 1), p=1, quad=4, init="zero", bcs=ADV_SPEC,
                     iters=200, sample="the full 64x64 mesh"))
    if name == "c2":
        prob, u0 = W.config2(args.n)
        return (prob, u0, 0.5, f"configuration 2: Burgers P2 triangles {args.n}x{args.n} "
                f"({prob.ncells:,} cells, {prob.nnodes:,} nodes), blended B scheme, 7-point rule, "
                "CFL 0.5", 20000,
                dict(mesh=("square", args.n, 0.15, 7), p=2, quad=5, init="burgers",
                     bcs=BURGERS_SPEC, iters=10, sample=f"the full {args.n}x{args.n} mesh"))
    if name == "c3":
        prob, u0 = W.config3()
        return (prob, u0, 0.5, "configuration 3: Euler 2D bump channel, 500,000 P3 triangles "
                "(16-point rule) + 500,000 P3 quadrilaterals (5x5 rule), 6,756,001 nodes, "
                "blended B scheme, Mach 0.5, CFL 0.5", 200,
                dict(mesh=("channel", 125, 250, 125, 3), p=3, quad=8, init="bump2d",
                     bcs=EULER2D_SPEC, iters=2,
                     sample="the same channel with a quarter of the cells per direction: "
                            "125x125 triangle squares + 250x125 quadrilaterals (62,500 cells; "
                            "the reference's own 20-point P8 quadrilateral rule)"))
    if name == "c4":
        prob, u0 = W.config4()
        return (prob, u0, 0.5, "configuration 4: Euler 3D bump box, 128x32x32 hexahedra split "
                "into 786,432 P2 tetrahedra (14-point rule), 1,085,825 nodes, LDA, Mach 0.6, "
                "CFL 0.5", 200,
                dict(mesh=("box", 32, 8, 8, 4), p=2, quad=5, init="bump3d", bcs=EULER3D_SPEC,
                     iters=2, sample="the same box at 32x8x8 hexahedra (12,288 tetrahedra)"))
    raise ValueError(name)


def cpu_reference(prob, spec, threads, workdir):
    """Time the reference's own CPU path (oracle/_ref/rds_ref_harness) on a mesh of the
    workload."""
    from pdekit_b200 import meshgen

    harness = os.path.join(ROOT, "oracle", "_ref", "rds_ref_harness")
    if not os.path.exists(harness):
        return None
    msh = os.path.join(workdir, "mesh.msh")
    m = spec["mesh"]
    if m[0] == "square":
        meshgen.write_gmsh22(msh, meshgen.unit_square_tri(m[1], m[2], seed=m[3]))
    elif m[0] == "channel":
        meshgen.write_gmsh22_mesh(msh, meshgen.channel_2d(m[1], m[2], m[3], jitter=0.0,
                                                          seed=m[4]))
    else:
        meshgen.write_gmsh22_mesh(msh, meshgen.box_tet(m[1], m[2], m[3], jitter=0.1, seed=m[4]))
    cfl = {"advconst": 0.9}.get(prob.physics, 0.5)
    out = subprocess.run([harness, "time", prob.physics, prob.scheme, str(spec["p"]),
                          str(spec["quad"]), msh, "-", str(spec["iters"]), str(cfl), spec["init"],
                          spec["bcs"], str(threads)],
                         capture_output=True, text=True, check=True).stdout
    return json.loads(out.strip().splitlines()[-1])


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


def time_steps(solver, steps, flush, cfl, step=None):
    """Per-step device time (ms) of `steps` fused iterations (or calls of `step`), L2 flushed
    before each step."""
    import torch

    stream = torch.cuda.ExternalStream(solver.stream_handle())
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.zero_()
            ev[k][0].record(stream)
            if step is None:
                solver.run(cfl, 1)
            else:
                step()
            ev[k][1].record(stream)
    stream.synchronize()
    return sum(a.elapsed_time(b) for a, b in ev)


def _drop_run(prob, u0, precision, cfl, max_iter, drop=1e-10):
    import torch

    from pdekit_b200.rds import PGRDMethodExplicit

    s = PGRDMethodExplicit(prob.physics, prob.scheme, precision).configure_mesh_data(prob)
    s.initialize_work_data()
    s.set_solution(u0)
    # the history buffer for max_iter rows and the loop graphs are made outside the timed
    # region (a drop of 1 stops at the first exact sweep)
    s.iterate(cfl, max_iter, 1.0, raise_on_cap=False)
    s.set_solution(u0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    it, hist = s.iterate(cfl, max_iter, drop, raise_on_cap=False)
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    rel = float((hist[-1] / hist[0]).max()) if len(hist) else None
    u = s.solution()
    s.close()
    # microseconds kept: the configuration-1 runs take a few milliseconds
    return {"seconds": round(sec, 6), "iterations": int(it), "final_rel_norm": rel,
            "reached": bool(rel is not None and rel <= drop),
            "cell_updates_per_s": prob.ncells * it / sec if sec > 0 else None}, u


def time_to_drop(args, c2_pgb):
    """Time to a 1e-10 drop of max_eq ||res dt|| / ||res dt||(iteration 0), FP64 and mixed
    (best of 3 runs for the small configuration-1 mesh).

    configuration 1 (advection P1 64x64, LDA, CFL 0.9) and the configuration-2 mesh with the N
    scheme (Burgers P2 512x512, CFL 0.5) converge to 1e-10; the blended B scheme on the
    configuration-2 mesh has not converged after thousands of iterations (its drop is
    reported at a capped iteration count)."""
    from pdekit_b200 import workloads

    out = {}
    cases = [("configuration 1: advection P1 64x64, LDA, CFL 0.9", workloads.config1(64), 0.9),
             (f"configuration-2 mesh with the N scheme: Burgers P2 {args.n}x{args.n}, CFL 0.5",
              workloads.config2(args.n, scheme="n"), 0.5)]
    def best_of(n, prob, u0, prec, cfl):
        runs = [_drop_run(prob, u0, prec, cfl, args.drop_max_iter) for _ in range(n)]
        return min(runs, key=lambda r: r[0]["seconds"])

    for name, (prob, u0), cfl in cases:
        reps = 3 if prob.ncells < 100000 else 1
        r64, u64 = best_of(reps, prob, u0, "fp64", cfl)
        rmx, umx = best_of(reps, prob, u0, "mixed", cfl)
        rmx["converged_state_rel_l2_vs_fp64"] = float(np.linalg.norm(umx - u64) /
                                                      np.linalg.norm(u64))
        out[name] = {"cells": prob.ncells, "fp64": r64, "mixed": rmx,
                     "speedup_mixed_vs_fp64": round(r64["seconds"] / rmx["seconds"], 3)}
    if c2_pgb is not None:
        prob, u0 = c2_pgb
        r, u64 = _drop_run(prob, u0, "fp64", 0.5, 4000)
        rm, um = _drop_run(prob, u0, "mixed", 0.5, 4000)
        rm["state_rel_l2_vs_fp64"] = float(np.linalg.norm(um - u64) / np.linalg.norm(u64))
        out["configuration 2 (blended B), capped at 4000 iterations"] = {"fp64": r, "mixed": rm}
    return out


def loop_rates(prob, u0, cfl, sweeps, world):
    """Sweep rate of the FP64 loop and of the mixed form's loop over the same number of sweeps
    through rds_iterate (one CUDA graph per chunk, no stop test), CUDA events on each solver's
    stream. Scalar physics: the defect-correction loop (an exact FP64 sweep every m sweeps,
    FP32 correction sweeps between); Euler: the FP32 cell kernels. Also the per-kernel device
    times of two cycles of the mixed loop (event timing, separate pass)."""
    import torch

    from pdekit_b200.rds import PGRDMethodExplicit

    out = {}
    for prec in ("fp64", "mixed"):
        s = PGRDMethodExplicit(prob.physics, prob.scheme, prec).configure_mesh_data(prob)
        s.initialize_work_data()
        s.set_solution(u0)
        s.iterate(cfl, 64, 0.0)  # graph capture
        s.set_solution(u0)
        st = torch.cuda.ExternalStream(s.stream_handle())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        done, _ = s.iterate(cfl, sweeps, 0.0)  # the sweeps run (the mixed loop ends on an
        e1.record(st)                          # exact sweep)
        e1.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), world)
        out[prec] = {"value": prob.ncells * done * world / (ms * 1e-3),
                     "ms_per_sweep": ms / done, "sweeps": int(done)}
        if prec == "mixed":
            s.set_solution(u0)
            s.kernel_timing(True)
            # two full cycles of the default period (24): the loop stops at an exact sweep once
            # the next cycle would pass max_iter, so 2 x 24 + 1 sweeps
            s.iterate(cfl, 49, 0.0)
            out["mixed_kernels_ms_per_launch"] = {k: round(v[0] / v[1], 5)
                                                  for k, v in s.kernel_times().items()}
            if any(k.startswith("dc_sweeps") for k in out["mixed_kernels_ms_per_launch"]):
                # a fused launch runs the 23 correction sweeps of a cycle (period 24)
                out["mixed_fused_sweeps_per_launch"] = 23
            s.kernel_timing(False)
        s.close()
    return out


def dc_roofline(prob, kernels):
    """Roofline of the mixed loop's FP32 correction-sweep cell kernel (scalar physics): its
    algorithmic flop per launch (dc_flops) over its event-timed duration, against the FP32 FMA
    peak measured on this GPU."""
    from pdekit_b200.rds import measure_peak

    dc = {k: v for k, v in kernels.items() if k.startswith("cells_") and k.endswith("_dc")}
    if not dc or prob.physics not in ("advconst", "burgers"):
        return None
    ms = sum(dc.values())
    flop = sum(dc_flops(prob.physics, prob.scheme, g.ndof, g.nq, g.nfl) * g.ncells
               for g in prob.groups)
    peak32 = measure_peak("mixed")
    achieved = flop / (ms * 1e-3) / 1e12
    return {"bound": "fp32", "kernel": max(dc, key=dc.get), "achieved": round(achieved, 3),
            "peak": round(peak32, 3), "unit": "TFLOP/s", "frac": round(achieved / peak32, 4),
            "peak_source": "measured in this run: rds_measure_peak (FP32 FMA micro-kernel)",
            "flop_per_launch": flop}


def compact_config(name, args, world):
    """One more configuration in fewer steps than the headline run: value (FP64, L2 flushed
    before every step, CUDA events), e2e (pipelined host-buffer steps), the FP64 and mixed loop
    rates, the roofline of the dominant kernel and the reference's CPU path on its sample."""
    import torch

    from pdekit_b200.rds import PGRDMethodExplicit, measure_peak

    prob, u0, cfl, desc, _, cpu_spec = workload(name, args)
    steps = {"c1": 2000, "c3": 20, "c4": 20}[name]
    s = PGRDMethodExplicit(prob.physics, prob.scheme, "fp64").configure_mesh_data(prob)
    s.initialize_work_data()
    s.set_solution(u0)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")
    s.run(cfl, 3)
    s.set_solution(u0)
    ms = max_over_ranks(time_steps(s, steps, flush, cfl), world)
    s.set_solution(u0)
    s.kernel_timing(True)
    nt = min(20, steps)
    s.run(cfl, nt)
    kt = s.kernel_times()
    s.kernel_timing(False)
    cells = {k: v for k, v in kt.items() if k.startswith("cells_")}
    cell_ms = sum(v[0] for v in cells.values()) / nt
    flop, byts = group_work(prob)
    roof = roofline(max(cells, key=lambda k: cells[k][0]), cell_ms, flop, byts,
                    measure_peak("fp64"), hbm_peak())
    if name in PROFILED_TRAFFIC:
        roof["traffic"], roof["traffic_source"] = PROFILED_TRAFFIC[name]
    # e2e: host buffers every step, pipelined (rds_step_host), host clock
    u_host = torch.from_numpy(np.ascontiguousarray(u0)).pin_memory()
    outs = [torch.empty_like(u_host).pin_memory() for _ in range(2)]
    nrms = [torch.empty(prob.neq, dtype=torch.float64).pin_memory() for _ in range(2)]
    ke = {"c1": 500, "c3": 10, "c4": 10}[name]
    s.step_host(u_host.numpy(), outs[0].numpy(), cfl, nrms[0].numpy())
    s.step_sync()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(ke):
        s.step_host(u_host.numpy(), outs[i % 2].numpy(), cfl, nrms[i % 2].numpy())
    s.step_sync()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3, world)
    s.close()
    rates = loop_rates(prob, u0, cfl, {"c1": 4096, "c3": 64, "c4": 64}[name], world)
    rec = {"workload": desc, "cells": prob.ncells, "nodes": prob.nnodes, "steps": steps,
           "value": prob.ncells * steps * world / (ms * 1e-3), "ms_per_step": ms / steps,
           "e2e": {"value": prob.ncells * ke * world / (e2e_ms * 1e-3), "steps": ke,
                   "h2d_bytes_per_step": int(u_host.numel() * 8),
                   "d2h_bytes_per_step": int(u_host.numel() * 8 + 8 * prob.neq)},
           "loop_fp64": rates["fp64"], "mixed": rates["mixed"],
           "mixed_kernels_ms_per_launch": rates["mixed_kernels_ms_per_launch"],
           "mixed_fused_sweeps_per_launch": rates.get("mixed_fused_sweeps_per_launch"),
           "roofline": roof, "mixed_roofline": dc_roofline(prob, rates["mixed_kernels_ms_per_launch"])}
    if not args.no_cpu:
        threads = os.cpu_count() or 1
        with tempfile.TemporaryDirectory() as td:
            r = cpu_reference(prob, cpu_spec, threads, td)
        if r:
            rec["cpu_baseline"] = {"value": r["cell_updates_per_s"], "cores": threads,
                                   "kind": "reference",
                                   "sample": f"{r['iters']} iterations of {cpu_spec['sample']} "
                                             f"({r['cells']} cells), nb_threads={threads}"}
    return rec


def run_ours(args, rank, world, local):
    import torch

    from pdekit_b200.rds import PGRDMethodExplicit, measure_peak

    torch.cuda.set_device(local)
    if args.workload == "c5":
        return run_batched(args, rank, world, local)
    if args.partition:
        return run_partitioned(args, rank, world, local)
    prob, u0, cfl, desc, default_steps, cpu_spec = workload(args.workload, args)
    steps = args.steps or default_steps
    ncells = prob.ncells

    prec0 = args.precision if args.quick else "fp64"
    solver = PGRDMethodExplicit(prob.physics, prob.scheme, prec0).configure_mesh_data(prob)
    solver.initialize_work_data()
    if args.tensor_cores:
        solver.set_option("tensor_cores", 1)
    solver.set_solution(u0)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")

    # warm-up
    solver.run(cfl, max(args.warmup, 3))
    torch.cuda.synchronize()
    solver.set_solution(u0)

    launches0 = solver.launch_count()
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t0 = time.time()
        ms = time_steps(solver, steps, flush, cfl)
        wall = time.time() - t0
    torch.cuda.synchronize()
    barrier(world)
    launches = solver.launch_count() - launches0
    ms = max_over_ranks(ms, world)
    value = ncells * steps * world / (ms * 1e-3)

    if args.quick:
        line = {"metric": "cell-residual updates/s", "value": value, "steps": steps,
                "ms_per_step": ms / steps, "gpu_launches": int(launches), "quick": True,
                "workload": args.workload, "precision": prec0,
                "tensor_cores": bool(args.tensor_cores)}
        solver.close()
        return line

    # per-kernel device time (event timing around every launch, separate pass)
    solver.set_solution(u0)
    solver.kernel_timing(True)
    iters_timed = min(50, steps)
    solver.run(cfl, iters_timed)
    ktimes = solver.kernel_times()
    solver.kernel_timing(False)
    cell_kernels = {k: v for k, v in ktimes.items() if k.startswith("cells_")}
    kname = max(cell_kernels, key=lambda k: cell_kernels[k][0])
    cell_ms = sum(v[0] for v in cell_kernels.values()) / iters_timed  # all groups, per iteration
    flop, byts = group_work(prob)
    peak64 = measure_peak("fp64")
    roof = roofline(kname, cell_ms, flop, byts, peak64, hbm_peak())
    roof["launches_per_iteration"] = len(prob.groups)
    if args.workload in PROFILED_TRAFFIC and (args.workload != "c2" or args.n == 512):
        roof["traffic"], roof["traffic_source"] = PROFILED_TRAFFIC[args.workload]

    # e2e through the C ABI with host buffers (pinned)
    u_host = torch.from_numpy(np.ascontiguousarray(u0)).pin_memory()
    u_out = torch.empty_like(u_host).pin_memory()
    ke = max(10, min(steps // 10, 200))
    stream = torch.cuda.ExternalStream(solver.stream_handle())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(ke):
        solver.set_solution(u_host.numpy())
        solver.assemble_lhs_and_rhs(cfl)
        solver.solve()
        solver.compute_residual_norm()
        solver.solution(out=u_out.numpy())
    e1.record(stream)
    e1.synchronize()
    sync_ms = max_over_ranks(e0.elapsed_time(e1), world)

    # the same steps pipelined (rds_step_host): every step still uploads its input from pinned
    # host memory and downloads its state and norm; the uploads, downloads and iterations of
    # consecutive steps overlap (two staging buffers, separate copy streams). Host clock around
    # the issued steps and the final wait, the device idle on both sides.
    outs = [torch.empty_like(u_host).pin_memory() for _ in range(2)]
    nrms = [torch.empty(prob.neq, dtype=torch.float64).pin_memory() for _ in range(2)]
    solver.step_host(u_host.numpy(), outs[0].numpy(), cfl, nrms[0].numpy())
    solver.step_sync()
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for i in range(ke):
        solver.step_host(u_host.numpy(), outs[i % 2].numpy(), cfl, nrms[i % 2].numpy())
    solver.step_sync()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3, world)
    e2e = {"value": ncells * ke * world / (e2e_ms * 1e-3), "unit": "cell-residual updates/s",
           "h2d_bytes_per_step": int(u_host.numel() * 8),
           "d2h_bytes_per_step": int(u_host.numel() * 8 + 8 * prob.neq), "steps": ke,
           "api": "rds_step_host (pipelined host-buffer steps), host clock",
           "synchronous_value": ncells * ke * world / (sync_ms * 1e-3),
           "synchronous_api": "rds_set_state + rds_assemble + rds_update + rds_residual_norm + "
                              "rds_get_state per step, CUDA events"}

    # mixed precision form: the defect-correction loop's sweep rate beside the FP64 loop's
    rates = loop_rates(prob, u0, cfl, min(steps, 4096), world)

    # third-order TVD Runge-Kutta steps (three residual passes each, one graph launch)
    solver.set_solution(u0)
    solver.advance_rk3tvd(cfl, max(args.warmup, 3))
    solver.set_solution(u0)
    ms_rk3 = max_over_ranks(time_steps(solver, steps, flush, cfl,
                                       lambda: solver.advance_rk3tvd(cfl, 1)), world)
    solver.set_solution(u0)
    rk3 = {"ms_per_step": ms_rk3 / steps,
           "cell_residual_updates_per_s": 3 * ncells * steps * world / (ms_rk3 * 1e-3),
           "api": "rds_advance_rk3tvd (RK3TVD::advance_in_time), CUDA events"}

    # time to a 1e-10 residual drop, FP64 vs mixed (device loop with the device-side stop test)
    drop = None
    if not args.no_drop and world == 1 and args.workload in ("c1", "c2"):
        drop = time_to_drop(args, (prob, u0) if args.workload == "c2" else None)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        with tempfile.TemporaryDirectory() as td:
            r = cpu_reference(prob, cpu_spec, threads, td)
            # the deterministic one-thread run (the parity reference) beside it; the
            # multi-thread scatter is unsynchronised, so its final norm is compared
            r1 = cpu_reference(prob, cpu_spec, 1, td) if (r and threads > 1) else r
        if r:
            cpu = {"value": r["cell_updates_per_s"], "unit": "cell-residual updates/s",
                   "cores": threads, "kind": "reference",
                   "sample": f"reference PGRDMethodExplicit ({prob.physics}, {prob.scheme}) on "
                             f"{cpu_spec['sample']}, {r['iters']} iterations after one warm-up "
                             f"assemble, nb_threads={threads} ({r['cells']} cells)",
                   "single_thread": {
                       "value": r1["cell_updates_per_s"], "cores": 1,
                       "final_norm_rel_diff_vs_threads":
                           abs(r["norm0"] - r1["norm0"]) / max(abs(r1["norm0"]), 1e-300)}}

    stab = measure_stab(args, solver, prob, u0, cfl, steps, flush, world) if args.stab else None

    line = {
        "metric": "cell-residual updates/s", "value": value, "unit": "cell-residual updates/s",
        "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "cells": ncells, "nodes": prob.nnodes,
                   "l2": "flushed (256 MB write) before every timed step",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "e2e": e2e,
        "mixed": dict(rates["mixed"], loop_fp64=rates["fp64"],
                      speedup_per_sweep_vs_fp64_loop=round(rates["mixed"]["value"] /
                                                           rates["fp64"]["value"], 3),
                      form="defect correction: an exact FP64 sweep every 24 sweeps, FP32 "
                           "correction sweeps between (the cell and facet changes computed from "
                           "the correction itself); rds_iterate, no stop test, CUDA events",
                      kernels_ms_per_launch=rates["mixed_kernels_ms_per_launch"],
                      fused_sweeps_per_launch=rates.get("mixed_fused_sweeps_per_launch"),
                      roofline=dc_roofline(prob, rates["mixed_kernels_ms_per_launch"])),
        "rk3tvd": rk3,
        "time_to_drop_1e-10": drop,
        "roofline": roof,
        "kernels_ms_per_launch": {k: round(v[0] / v[1], 5) for k, v in ktimes.items()},
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "gpu_launches": int(launches),
        "wall_s_timed_region": round(wall, 3),
    }
    if stab:
        line["stabilised"] = stab
    solver.close()
    if args.workload == "c2" and world == 1 and not args.no_configs:
        # the other configurations, compact (the driver records this one line)
        line["configs"] = {k: compact_config(k, args, world) for k in ("c1", "c3", "c4")}
        # configuration 5 with the FP64 plain path (every problem alone) beside the batched loops
        args.c5_sequential = True
        c5 = run_batched(args, rank, world, local)
        line["configs"]["c5"] = {"workload": c5["config"]["workload"], "cells": c5["config"]["cells"],
                                 "value": c5["value"], "gpu_launches": c5["gpu_launches"],
                                 "time_to_drop_1e-10": c5["time_to_drop_1e-10"]}
    return line


def measure_stab(args, solver, prob, u0, cfl, steps, flush, world):
    """The step with a stabilisation field: the operator computes the nodal field from the
    state on the device and installs it (no host copy), then the same timed steps as `value`.
    The operator is timed with CUDA events on the solver's stream (mean of 5 calls after one
    warm-up call)."""
    import torch

    from pdekit_b200 import stabilisation as st

    op, p0, name = {"av": (st.ART_VISC, 5.0, "artificial viscosity (kappa 5, factor 1)"),
                    "lf": (st.BLEND_LF, 0.0, "LF_Blend"),
                    "wj": (st.BLEND_WONG_JANSEN, 1.0, "WongJansen (u_inf 1)"),
                    "visc": (st.BLEND_VISC, 5.0, "ViscosityIndicator (kappa 5)")}[args.stab]
    solver.set_solution(u0)
    stream = torch.cuda.ExternalStream(solver.stream_handle())
    solver.compute_stabilisation(op, p0, 1.0, install=True, cells=False)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(5):
        solver.compute_stabilisation(op, p0, 1.0, install=True, cells=False)
    e1.record(stream)
    e1.synchronize()
    op_ms = max_over_ranks(e0.elapsed_time(e1) / 5, world)
    solver.run(cfl, max(args.warmup, 3))
    torch.cuda.synchronize()
    solver.set_solution(u0)
    solver.compute_stabilisation(op, p0, 1.0, install=True, cells=False)
    launches0 = solver.launch_count()
    ms = max_over_ranks(time_steps(solver, steps, flush, cfl), world)
    launches = solver.launch_count() - launches0
    reads = {"av": "PGLDA", "lf": "PGB", "wj": "PGB", "visc": "PGB"}[args.stab]
    return {"field": name, "read_by": reads,
            "applies": (prob.scheme == "lda") == (reads == "PGLDA"),
            "value": prob.ncells * steps * world / (ms * 1e-3), "ms_per_step": ms / steps,
            "operator_ms": op_ms, "gpu_launches": int(launches)}


def run_partitioned(args, rank, world, local):
    """c1-c4 with the one mesh split over the ranks (pdekit_b200.partition): per step every rank
    assembles the cells at its interface, all-reduces the interface sums while it assembles the
    rest, updates its nodes and all-reduces the norm parts; the step is one CUDA graph replay.
    Strong scaling: value = the whole mesh's cells x steps / the slowest rank's time."""
    import torch

    from pdekit_b200.partition import PartitionedRDS

    prob, u0, cfl, desc, default_steps, _ = workload(args.workload, args)
    steps = args.steps or default_steps
    pr = PartitionedRDS(prob, rank, world)
    pr.set_solution(u0)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")
    for _ in range(max(args.warmup, 3)):
        pr.graph_step(cfl, norm=False)  # captures the graph of the timed steps
    torch.cuda.synchronize()
    pr.set_solution(u0)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    barrier(world)
    torch.cuda.synchronize()
    launches0 = pr.rank.solver.launch_count() + pr.graph_launches
    with ClockSampler(local) as clk:
        with torch.cuda.stream(pr.rank.stream):
            for k in range(steps):
                flush.zero_()
                ev[k][0].record(pr.rank.stream)
                pr.graph_step(cfl, norm=False)  # the work of the fused step (rds_run)
                ev[k][1].record(pr.rank.stream)
        torch.cuda.synchronize()
    barrier(world)
    launches = pr.rank.solver.launch_count() + pr.graph_launches - launches0
    ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), world)
    pr.graph_step(cfl)  # one more step with its norm (reported, not timed)
    norm = pr.norm()
    part = pr.partition.parts[rank]
    line = {"metric": "cell-residual updates/s", "value": prob.ncells * steps / (ms * 1e-3),
            "unit": "cell-residual updates/s", "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": ms / steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "cells": prob.ncells,
                       "l2": "L2 flushed (256 MB write) before every timed step",
                       "parallelism": f"one mesh split over {world} ranks along x "
                                      f"({pr.partition.nslots:,} interface nodes), interface "
                                      "sums all-reduced per step while the interior cells "
                                      "run, one CUDA graph per step; timed steps write the "
                                      "norm's block sums without adding them, like the fused "
                                      "step"},
            "final_norm": [float(x) for x in norm], "clocks": clk.summary(),
            "gpu_launches": int(launches),
            "cells_rank0": int(sum(len(c) for c in part.cells))}
    pr.close()
    return line


def run_batched(args, rank, world, local):
    """Configuration 5: the batched FP64 and mixed loops to every problem's 1e-10 drop."""
    import torch

    from pdekit_b200 import workloads
    from pdekit_b200.batch import BatchedRDS
    from pdekit_b200.rds import PGRDMethodExplicit, measure_peak

    probs, states, cfls, info = workloads.config5(nprob=args.c5_nprob, seed=5)
    total_cells = sum(p.ncells for p in probs)
    if world > 1:
        # one problem set, split over the ranks by estimated work (no exchange between problems)
        from pdekit_b200.batch import shard_problems

        mine = shard_problems(probs, world)[rank]
        probs = [probs[i] for i in mine]
        states = [states[i] for i in mine]
        cfls = cfls[mine]
        info = [info[i] for i in mine]
    cells = sum(p.ncells for p in probs)
    u_host = [torch.from_numpy(np.ascontiguousarray(s)).pin_memory() for s in states]
    res = {}
    launches = 0
    clocks = None
    for prec in ("fp64", "mixed"):
        b = BatchedRDS(probs, cfls, prec)
        b.set_solutions(states)
        tune = b.autotune()
        b.set_solutions(states)
        b.iterate(3, 0.0, raise_on_cap=False)  # graph capture outside the timed region
        barrier(world)
        torch.cuda.synchronize()
        l0 = b.launch_count()
        with ClockSampler(local) as clk:
            t0 = time.time()
            b.set_solutions([u.numpy() for u in u_host])
            iters, rel = b.iterate(args.drop_max_iter, 1e-10, raise_on_cap=False)
            out = b.solutions()
            torch.cuda.synchronize()
            sec = time.time() - t0
        sec = max_over_ranks(sec, world)
        cu = sum_over_ranks(float(sum(p.ncells * int(i) for p, i in zip(probs, iters))), world)
        res[prec] = {"seconds": round(sec, 3),
                     "iterations_max": int(max_over_ranks(float(iters.max()), world)),
                     "iterations_mean": float(iters.mean()), "cell_updates": cu,
                     "cell_updates_per_s": cu / sec,
                     "problems_reached": int(sum_over_ranks(float((rel <= 1e-10).sum()), world)),
                     "autotune": tune}
        res[prec + "_states"] = out
        if prec == "fp64":
            launches = b.launch_count() - l0
            clocks = clk.summary()
        b.close()
    rel_l2 = max_over_ranks(max(float(np.linalg.norm(a - c) / np.linalg.norm(a))
                                for a, c in zip(res["fp64_states"], res["mixed_states"])), world)
    res["speedup_mixed_vs_fp64"] = round(res["fp64"]["seconds"] / res["mixed"]["seconds"], 3)
    del res["fp64_states"], res["mixed_states"]
    seq = None
    if args.c5_sequential and world == 1:
        tot = 0.0
        for p, u0, c in zip(probs, states, cfls):
            s = PGRDMethodExplicit(p.physics, p.scheme, "fp64").configure_mesh_data(p)
            s.initialize_work_data()
            s.set_solution(u0)
            s.iterate(c, args.drop_max_iter, 1.0, raise_on_cap=False)
            s.set_solution(u0)
            torch.cuda.synchronize()
            t0 = time.time()
            s.iterate(c, args.drop_max_iter, 1e-10, raise_on_cap=False)
            torch.cuda.synchronize()
            tot += time.time() - t0
            s.close()
        seq = {"seconds": round(tot, 3),
               "speedup_batched_fp64": round(tot / res["fp64"]["seconds"], 3),
               "speedup_batched_mixed": round(tot / res["mixed"]["seconds"], 3),
               "api": "every problem in its own FP64 context, rds_iterate to its 1e-10 drop, one "
                      "after another (graphs captured before the clock starts)"}
    peak64 = measure_peak("fp64")
    f64 = res["fp64"]
    line = {
        "metric": "cell-residual updates/s", "value": f64["cell_updates_per_s"],
        "unit": "cell-residual updates/s", "n_gpus": world, "steps": f64["iterations_max"],
        "warmup": 3, "ms_per_step": f64["seconds"] * 1e3 / f64["iterations_max"],
        "higher_is_better": True, "scaling": "strong" if world > 1 else "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"configuration 5: {args.c5_nprob} independent problems "
                               f"(advection LDA / Burgers N, P1-P3 triangles, log-uniform "
                               f"1k-200k cells, own CFL), {total_cells:,} cells in total, each "
                               f"to its own 1e-10 drop, batched persistent launches in one CUDA "
                               f"graph",
                   "cells": total_cells, "l2": "inputs larger than L2 (state and contributions)",
                   "parallelism": (f"problems split over {world} GPUs by estimated work, no "
                                   f"exchange") if world > 1 else "single GPU"},
        "e2e": {"value": f64["cell_updates_per_s"], "unit": "cell-residual updates/s",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "note": "the timed region of value already copies every problem's state in from "
                        "pinned host memory and back out"},
        "time_to_drop_1e-10": {"batched_fp64": res["fp64"], "batched_mixed": res["mixed"],
                               "speedup_mixed_vs_fp64": res["speedup_mixed_vs_fp64"],
                               "mixed_vs_fp64_converged_rel_l2_max": rel_l2,
                               "sequential_plain_fp64": seq},
        "roofline": {"bound": "fp64", "peak": round(peak64, 3), "unit": "TFLOP/s",
                     "note": "per-group kernel times of the autotuner are in "
                             "time_to_drop_1e-10.batched_*.autotune"},
        "cpu_baseline": None,
        "clocks": clocks,
        "gpu_launches": int(launches),
    }
    return line


def run_reference(args, rank, world):
    """The reference's own CPU implementation of the path (oracle/_ref) on the host cores."""
    if rank != 0:
        return None
    if args.workload == "c5":
        return {"impl": "reference", "unavailable": "configuration 5 has no reference arm: the "
                "reference solves one problem per solver object"}
    prob, u0, cfl, desc, default_steps, spec = workload(args.workload, args)
    threads = os.cpu_count() or 1
    spec = dict(spec)
    if args.workload == "c2":
        spec["iters"] = max(5, (args.steps or 500) // 50)
    with tempfile.TemporaryDirectory() as td:
        t0 = time.time()
        r = cpu_reference(prob, spec, threads, td)
        wall = time.time() - t0
    if r is None:
        return {"impl": "reference", "unavailable": "oracle/_ref/rds_ref_harness not built"}
    v = r["cell_updates_per_s"]
    return {"impl": "reference", "metric": "cell-residual updates/s", "value": v,
            "unit": "cell-residual updates/s", "n_gpus": world, "steps": r["iters"],
            "warmup": 1, "ms_per_step": r["seconds"] / r["iters"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": desc, "cells": r["cells"], "nodes": r["nodes"],
                       "sample": spec["sample"]},
            "cpu_baseline": {"value": v, "unit": "cell-residual updates/s", "cores": threads,
                             "kind": "reference",
                             "sample": f"{r['iters']} iterations of {spec['sample']}, "
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
