"""Regenerate the golden fixtures in tests/golden/<case>/ from the reference itself.

Each case writes a seeded synthetic P1 triangle mesh (Gmsh 2.2, pdekit_b200.meshgen), runs the
reference's own PGRDMethodExplicit through oracle/_ref/rds_ref_harness (the reference sources
compiled in place by oracle/Makefile) and keeps what the harness dumps: the reference's
connectivity, reference-element tables, boundary facets, initial state, and its outputs after
one assemble_lhs_and_rhs (residual, wave speed, dt, dual volume), after one solve, after
`iters` iterations (state and residual norms), and after two steps of its RK3TVD stepper (state,
first-stage residual and dt, norms). The cases in JACOBIAN_CASES also hold the reference's
Picard-linearised implicit assembly at u0 (jac_row / jac_col / jac_val: the summed J(m, n) / V(m)
entries of its PGRDMPicardJacCellAssemblyWorker; jac_rhs: -res / V).

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

EULER2D_BCS = ("WeakWall:bottom_wall_bc:bottom_wall:-,WeakWall:top_wall_bc:top_wall:-,"
               "WeakSubInlet:inlet_bc:inlet:total_temperature=307.6488978;"
               "total_pressure=120195.4453,"
               "WeakSubOutlet:outlet_bc:outlet:total_pressure=101325.0")
EULER3D_BCS = ("WeakWall:bottom_wall_bc:bottom_wall:-,WeakWall:top_wall_bc:top_wall:-,"
               "WeakWall:side_walls_bc:side_walls:-,"
               "WeakSubInlet:inlet_bc:inlet:total_temperature=307.6488978;"
               "total_pressure=120195.4453,"
               "WeakSubOutlet:outlet_bc:outlet:total_pressure=101325.0")

# WeakFarfield with the bump freestream as reference state (conservative variables), and
# StrongDirichlet inflow (the strong condition precedes the weak left inflow in name order, so
# the weak condition sees the overwritten corner state)
FAR2D = "state=1.204780419|206.7048679|0|271049.8994"
FAR3D = "state=1.143916132|233.0856257|0|0|259331.1534"
EULER2D_FAR_BCS = ("WeakWall:bottom_wall_bc:bottom_wall:-,WeakFarfield:farfield_bc:top_wall:" + FAR2D
                   + ",WeakSubInlet:inlet_bc:inlet:total_temperature=307.6488978;"
                   "total_pressure=120195.4453,"
                   "WeakSubOutlet:outlet_bc:outlet:total_pressure=101325.0")
EULER3D_FAR_BCS = ("WeakWall:bottom_wall_bc:bottom_wall:-,WeakFarfield:farfield_bc:top_wall:" + FAR3D
                   + ",WeakFarfield:side_bc:side_walls:" + FAR3D
                   + ",WeakSubInlet:inlet_bc:inlet:total_temperature=307.6488978;"
                   "total_pressure=120195.4453,"
                   "WeakSubOutlet:outlet_bc:outlet:total_pressure=101325.0")
# WeakSymmetry (reflected momentum) and WeakSuperInlet (wave speed only) of the Euler registry
EULER2D_SYM_BCS = ("WeakWall:bottom_wall_bc:bottom_wall:-,WeakSymmetry:symmetry_bc:top_wall:-,"
                   "WeakSuperInlet:inlet_bc:inlet:-,"
                   "WeakSubOutlet:outlet_bc:outlet:total_pressure=101325.0")
EULER3D_SYM_BCS = ("WeakWall:bottom_wall_bc:bottom_wall:-,WeakSymmetry:symmetry_top_bc:top_wall:-,"
                   "WeakSymmetry:symmetry_side_bc:side_walls:-,"
                   "WeakSubInlet:inlet_bc:inlet:total_temperature=307.6488978;"
                   "total_pressure=120195.4453,WeakSuperInlet:outlet_bc:outlet:-")
ADV_STRONG_BCS = "StrongDirichlet:inlet_bottom:bottom:sin2pix,WeakDirichlet:inlet_left:left:zero"
BURG_STRONG_BCS = ("WeakDirichlet:inlet:bottom:burgers_inlet,StrongDirichlet:left:left:c1.5,"
                   "WeakDirichlet:right:right:c-0.5")

# name: (physics, scheme, p, quad order, n, jitter, seed, init, bcs, cfl, iters)
# n is the squares per side of the unit square, or a tuple naming another mesh:
#   ("channel_tri", nx, ny) / ("channel_quad", nx, ny): bump channel [-1.5,1.5] x [0,1]
#   ("box_tet", nx, ny, nz): bump box [-2,2] x [0,1]^2, hexahedra split into 6 tetrahedra
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
    # configuration 3 (Euler 2D bump channel, P3 triangles / P3 quadrilaterals, blended B)
    "euler2d_tri_p3_b": ("euler2d", "b", 3, 8, ("channel_tri", 4, 3), 0.15, 31, "bump2d",
                         EULER2D_BCS, 0.5, 3),
    "euler2d_quad_p3_b": ("euler2d", "b", 3, 8, ("channel_quad", 4, 3), 0.15, 32, "bump2d",
                          EULER2D_BCS, 0.5, 3),
    "euler2d_tri_p1_lda": ("euler2d", "lda", 1, 4, ("channel_tri", 5, 3), 0.15, 33, "bump2d",
                           EULER2D_BCS, 0.5, 3),
    "euler2d_tri_p2_n": ("euler2d", "n", 2, 5, ("channel_tri", 4, 3), 0.15, 34, "bump2d",
                         EULER2D_BCS, 0.5, 3),
    # configuration 4 (Euler 3D bump box, P2 tetrahedra, LDA)
    "euler3d_tet_p2_lda": ("euler3d", "lda", 2, 5, ("box_tet", 3, 2, 2), 0.1, 41, "bump3d",
                           EULER3D_BCS, 0.5, 3),
    # the other two conditions of the reference's registry (bc/RDMBCManager.hpp:57-89);
    # WeakFarfield only with Euler (the reference's scalar instantiation crashes in the harness)
    "adv_p2_strong": ("advconst", "lda", 2, 5, 5, 0.2, 16, "smooth", ADV_STRONG_BCS, 0.9, 3),
    "adv_p1_strong": ("advconst", "n", 1, 4, 6, 0.2, 18, "smooth", ADV_STRONG_BCS, 0.9, 3),
    "burgers_p2_strong": ("burgers", "b", 2, 5, 5, 0.15, 26, "burgers", BURG_STRONG_BCS, 0.5, 3),
    "euler2d_tri_p2_farfield": ("euler2d", "n", 2, 5, ("channel_tri", 4, 3), 0.15, 35, "bump2d",
                                EULER2D_FAR_BCS, 0.5, 3),
    "euler3d_tet_p2_farfield": ("euler3d", "lda", 2, 5, ("box_tet", 3, 2, 2), 0.1, 42, "bump3d",
                                EULER3D_FAR_BCS, 0.5, 3),
    "euler2d_tri_p2_symmetry": ("euler2d", "b", 2, 5, ("channel_tri", 4, 3), 0.15, 36, "bump2d",
                                EULER2D_SYM_BCS, 0.5, 3),
    "euler3d_tet_p2_symmetry": ("euler3d", "n", 2, 5, ("box_tet", 3, 2, 2), 0.1, 43, "bump3d",
                                EULER3D_SYM_BCS, 0.5, 3),
    # stabilisation fields computed at u0 by the reference's own operators (a steep front, so
    # that the sensor is zero in some cells and on its ramp in others): nodal artificial
    # viscosity into PGLDA, nodal blending coefficients into PGB; optional 12th entry
    "burgers_p2_lda_av": ("burgers", "lda", 2, 5, 8, 0.15, 51, "steep", BURG_BCS, 0.5, 3,
                          "av:2.0:1.0"),
    "adv_p1_lda_av": ("advconst", "lda", 1, 4, 8, 0.2, 52, "steep", ADV_BCS, 0.9, 3,
                      "av:3.0:0.5"),
    "burgers_p3_lda_av": ("burgers", "lda", 3, 8, 5, 0.15, 53, "steep", BURG_BCS, 0.5, 3,
                          "av:2.0:1.0"),
    "burgers_p2_b_lf": ("burgers", "b", 2, 5, 8, 0.15, 54, "steep", BURG_BCS, 0.5, 3,
                        "blend:LF_Blend:0"),
    "burgers_p2_b_wj": ("burgers", "b", 2, 5, 8, 0.15, 55, "steep", BURG_BCS, 0.5, 3,
                        "blend:WongJansen:1.0"),
    "adv_p2_b_visc": ("advconst", "b", 2, 5, 8, 0.2, 56, "steep", ADV_BCS, 0.9, 3,
                      "blend:ViscosityIndicator:2.0"),
    "euler2d_tri_p2_lda_av": ("euler2d", "lda", 2, 5, ("channel_tri", 6, 3), 0.15, 57,
                              "bump2d_jump", EULER2D_BCS, 0.5, 3, "av:4.0:1.0"),
    "euler2d_tri_p3_b_lf": ("euler2d", "b", 3, 8, ("channel_tri", 5, 3), 0.15, 58, "bump2d_jump",
                            EULER2D_BCS, 0.5, 3, "blend:LF_Blend:0"),
    # the reference's cell-to-node transfer crashes on tetrahedral meshes: the cellwise values
    # come from the reference, the nodal field handed to its solver from the oracle's transfer
    "euler3d_tet_p2_lda_av": ("euler3d", "lda", 2, 5, ("box_tet", 4, 2, 2), 0.1, 59,
                              "bump3d_jump", EULER3D_BCS, 0.5, 3, "av3d:4.0:1.0"),
    # Bonanni's pressure-based blending coefficient into PGB (3D: cellwise values from the
    # reference, the nodal field from the oracle's transfer, as for the viscosity above)
    "euler2d_tri_p2_b_bonanni": ("euler2d", "b", 2, 5, ("channel_tri", 5, 3), 0.15, 61,
                                 "bump2d_jump", EULER2D_BCS, 0.5, 3, "blend:Bonanni2D:0"),
    "euler2d_tri_p3_b_bonanni": ("euler2d", "b", 3, 8, ("channel_tri", 4, 3), 0.15, 62,
                                 "bump2d_jump", EULER2D_BCS, 0.5, 3, "blend:Bonanni2D:0"),
    "euler2d_quad_p2_b_bonanni": ("euler2d", "b", 2, 5, ("channel_quad", 5, 3), 0.15, 63,
                                  "bump2d_jump", EULER2D_BCS, 0.5, 3, "blend:Bonanni2D:0"),
    "euler3d_tet_p2_b_bonanni": ("euler3d", "b", 2, 5, ("box_tet", 4, 2, 2), 0.1, 64,
                                 "bump3d_jump", EULER3D_BCS, 0.5, 3, "blend3d:Bonanni3D:0"),
    # rules the reference's own examples use: P3 triangles with the order-6 rule (12 points,
    # examples/testcases-rdm/Burgers-RDS-2D.cpp), P1 tetrahedra with the order-2 rule (4 points,
    # Bump-RDS-3D-Explicit.cpp)
    "burgers_p3_q6_b": ("burgers", "b", 3, 6, 5, 0.15, 67, "burgers", BURG_BCS, 0.5, 3),
    "adv_p3_q6_n": ("advconst", "n", 3, 6, 5, 0.2, 68, "smooth", ADV_BCS, 0.9, 3),
    "euler3d_tet_p1_lda": ("euler3d", "lda", 1, 2, ("box_tet", 4, 2, 2), 0.1, 69, "bump3d",
                           EULER3D_BCS, 0.5, 3),
    "euler3d_tet_p1_b": ("euler3d", "b", 1, 2, ("box_tet", 4, 2, 2), 0.1, 70, "bump3d",
                         EULER3D_BCS, 0.5, 3),
    # Euler 2D P3 triangles with the order-6 rule and P1 quadrilaterals with the order-3 rule
    # (the 2 x 2 Gauss rule)
    "euler2d_tri_p3_q6_b": ("euler2d", "b", 3, 6, ("channel_tri", 4, 3), 0.15, 72, "bump2d",
                            EULER2D_BCS, 0.5, 3),
    "euler2d_quad_p1_q3_lda": ("euler2d", "lda", 1, 3, ("channel_quad", 6, 3), 0.15, 73,
                               "bump2d", EULER2D_BCS, 0.5, 3),
    # P2 tetrahedra with the order-4 rule (11 points; examples/testcases-rdm/OneraM6-RDS.cpp)
    "euler3d_tet_p2_q4_n": ("euler3d", "n", 2, 4, ("box_tet", 3, 2, 2), 0.1, 71, "bump3d",
                            EULER3D_BCS, 0.5, 3),
    # the smoothness sensor on bilinear quadrilaterals (detJ varies inside the cell); P1 only:
    # at p >= 2 the reference's rule of order 2p has fewer points than the cell has modes, its
    # modal mass matrix is singular and the sensor follows the rounding of its inversion
    "euler2d_quad_p1_lda_av": ("euler2d", "lda", 1, 5, ("channel_quad", 8, 4), 0.15, 65,
                               "bump2d_jump", EULER2D_BCS, 0.5, 3, "av:4.0:1.0"),
    "euler2d_quad_p1_b_visc": ("euler2d", "b", 1, 5, ("channel_quad", 8, 4), 0.15, 66,
                               "bump2d_jump", EULER2D_BCS, 0.5, 3,
                               "blend:ViscosityIndicator:1.5"),
}


# cases that also dump the reference's assembled element Jacobians (RDS_HARNESS_JACOBIAN)
JACOBIAN_CASES = {"burgers_p2_lda", "burgers_p2_n", "burgers_p2_b", "burgers_p3_b", "adv_p2_b",
                  "euler2d_tri_p1_lda", "euler2d_tri_p2_n", "euler2d_tri_p3_b",
                  "euler2d_quad_p3_b", "euler3d_tet_p2_lda"}


def make(name, spec):
    physics, scheme, p, quad, n, jit, seed, init, bcs, cfl, iters = spec[:11]
    stab = spec[11] if len(spec) > 11 else "none"
    out = os.path.join(HERE, name)
    if os.path.isdir(out):
        shutil.rmtree(out)
    os.makedirs(out)
    msh = os.path.join(out, "mesh.msh")
    if isinstance(n, tuple):
        if n[0] == "channel_tri":
            mesh = meshgen.channel_2d(n[1], 0, n[2], x0=-1.5, xm=1.5, x1=1.5, jitter=jit,
                                      seed=seed)
        elif n[0] == "channel_quad":
            mesh = meshgen.channel_2d(0, n[1], n[2], x0=-1.5, xm=-1.5, x1=1.5, jitter=jit,
                                      seed=seed)
        else:
            mesh = meshgen.box_tet(n[1], n[2], n[3], jitter=jit, seed=seed)
        meshgen.write_gmsh22_mesh(msh, mesh)
    else:
        meshgen.write_gmsh22(msh, meshgen.unit_square_tri(n, jit, seed=seed))
    cmd = [HARNESS, "dump", physics, scheme, str(p), str(quad), msh, out, str(iters), str(cfl),
           init, bcs, "1"]
    env = dict(os.environ)
    env.pop("RDS_HARNESS_NO_RK3", None)
    if name in JACOBIAN_CASES:
        env["RDS_HARNESS_JACOBIAN"] = "1"
    else:
        env.pop("RDS_HARNESS_JACOBIAN", None)
    if not (stab.startswith("av3d:") or stab.startswith("blend3d:")):
        subprocess.run(cmd + [stab], check=True, stdout=subprocess.DEVNULL, env=env)
        return
    # two passes: the reference's cellwise field, then the solver with the nodal field
    import json
    import numpy as np
    from oracle import stab_oracle
    blend = stab.startswith("blend3d:")
    _, a1, a2 = stab.split(":")
    tmp = out + "_cells"
    os.makedirs(tmp, exist_ok=True)
    first = f"blendcells:{a1}:{a2}" if blend else f"avcells:{a1}:{a2}"
    subprocess.run(cmd[:7] + [tmp] + cmd[8:] + [first], check=True, stdout=subprocess.DEVNULL)
    meta = json.load(open(os.path.join(tmp, "meta.json")))
    shp = meta["arrays"]
    rd = lambda n, t: np.fromfile(os.path.join(tmp, f"{n}.{t}"),
                                  dtype=np.float64 if t == "f64" else np.int32).reshape(shp[n])
    sol_conn, sol_nodes = rd("sol_conn", "i32"), rd("sol_nodes", "f64")
    cells = ("blend_cell",) if blend else ("av_cell", "indicator")
    nodal = stab_oracle.nodal_from_cells(rd(cells[0], "f64"), sol_conn, meta["nsol"],
                                         stab_oracle.p1_at(meta["dim"], sol_nodes))
    field = os.path.join(tmp, "field.f64")
    nodal.tofile(field)
    second = f"blendfield:{field}" if blend else f"avfield:{field}"
    subprocess.run(cmd + [second], check=True, stdout=subprocess.DEVNULL)
    meta2 = json.load(open(os.path.join(out, "meta.json")))
    for n in cells:
        shutil.copy(os.path.join(tmp, f"{n}.f64"), os.path.join(out, f"{n}.f64"))
        meta2["arrays"][n] = shp[n]
    meta2["stab"] = stab
    json.dump(meta2, open(os.path.join(out, "meta.json"), "w"), indent=1)
    shutil.rmtree(tmp)


def main(argv):
    if not os.path.exists(HARNESS):
        raise SystemExit(f"{HARNESS} missing: run `make -C oracle` with the reference mounted")
    names = argv or list(CASES)
    for name in names:
        make(name, CASES[name])
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1:])
