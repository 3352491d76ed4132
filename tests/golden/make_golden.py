"""Regenerate the golden fixtures in tests/golden/<case>/ from the reference itself.

Each case writes a seeded synthetic P1 triangle mesh (Gmsh 2.2, pdekit_b200.meshgen), runs the
reference's own PGRDMethodExplicit through oracle/_ref/rds_ref_harness (the reference sources
compiled in place by oracle/Makefile) and keeps what the harness dumps: the reference's
connectivity, reference-element tables, boundary facets, initial state, and its outputs after
one assemble_lhs_and_rhs (residual, wave speed, dt, dual volume), after one solve, and after
`iters` iterations (state and residual norms).

Needs the reference tree (it runs only where the reference is mounted):
    make -C oracle && python tests/golden/make_golden.py
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from pdekit_b200 import meshgen  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "rds_ref_harness")

ADV_BCS = "WeakDirichlet:inlet_bottom:bottom:sin2pix,WeakDirichlet:inlet_left:left:zero"
BURG_BCS = ("WeakDirichlet:inlet:bottom:burgers_inlet,WeakDirichlet:left:left:c1.5,"
            "WeakDirichlet:right:right:c-0.5")

# name: (physics, scheme, p, quad order, n, jitter, seed, init, bcs, cfl, iters)
CASES = {
    # configuration 1 (advection, P1, LDA, P4 rule, jitter 0.2h, CFL 0.9) on a small mesh
    "adv_p1_lda_zero": ("advconst", "lda", 1, 4, 8, 0.2, 11, "zero", ADV_BCS, 0.9, 5),
    "adv_p1_lda": ("advconst", "lda", 1, 4, 6, 0.2, 12, "smooth", ADV_BCS, 0.9, 3),
    "adv_p1_n": ("advconst", "n", 1, 4, 6, 0.2, 13, "smooth", ADV_BCS, 0.9, 3),
    "adv_p2_b": ("advconst", "b", 2, 5, 5, 0.2, 14, "smooth", ADV_BCS, 0.9, 3),
    "adv_p3_lda": ("advconst", "lda", 3, 8, 4, 0.2, 15, "smooth", ADV_BCS, 0.9, 3),
    # configuration 2 (Burgers, P2, blended B, 7-point rule, jitter 0.15h) on a small mesh
    "burgers_p2_b": ("burgers", "b", 2, 5, 6, 0.15, 21, "burgers", BURG_BCS, 0.5, 4),
    "burgers_p2_n": ("burgers", "n", 2, 5, 5, 0.15, 22, "burgers", BURG_BCS, 0.5, 3),
    "burgers_p2_lda": ("burgers", "lda", 2, 5, 5, 0.15, 23, "burgers", BURG_BCS, 0.5, 3),
    "burgers_p1_b": ("burgers", "b", 1, 4, 6, 0.2, 24, "burgers", BURG_BCS, 0.5, 3),
    "burgers_p3_b": ("burgers", "b", 3, 8, 4, 0.2, 25, "burgers", BURG_BCS, 0.5, 3),
}


def make(name, spec):
    physics, scheme, p, quad, n, jit, seed, init, bcs, cfl, iters = spec
    out = os.path.join(HERE, name)
    if os.path.isdir(out):
        shutil.rmtree(out)
    os.makedirs(out)
    mesh = meshgen.unit_square_tri(n, jit, seed=seed)
    msh = os.path.join(out, "mesh.msh")
    meshgen.write_gmsh22(msh, mesh)
    cmd = [HARNESS, "dump", physics, scheme, str(p), str(quad), msh, out, str(iters), str(cfl),
           init, bcs]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)


def main(argv):
    if not os.path.exists(HARNESS):
        raise SystemExit(f"{HARNESS} missing: run `make -C oracle` with the reference mounted")
    names = argv or list(CASES)
    for name in names:
        make(name, CASES[name])
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1:])
