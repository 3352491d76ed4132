"""Host-side mirror of pdekit's explicit RDS solver interface over the librds_b200 C ABI.

`PGRDMethodExplicit` keeps the reference's call sequence and names
(src/solver/rdm/PGRDMethodExplicit.hpp:38-93, src/solver/rdm/RDMethod.hpp:60-139):

    scheme = PGRDMethodExplicit(physics="burgers", scheme="b")
    scheme.configure_mesh_data(problem)      # mesh, geometry and solution dofs, tables
    scheme.add_boundary_condition(...)       # optional, weak BCs (or carried by the problem)
    scheme.initialize_work_data()            # -> rds_finalize (gather lists, dual volumes)
    scheme.set_solution(u)                   # SolverVecFn::solution
    scheme.assemble_lhs_and_rhs(cfl); scheme.solve()
    scheme.compute_residual_norm()

Every call goes through librds_b200.so; there is no CPU fallback. If the library is absent the
import fails loudly.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .problem import Problem

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librds_b200.so")

PHYSICS = {"advconst": 0, "burgers": 1, "euler2d": 2, "euler3d": 3}
SCHEME = {"lda": 0, "n": 1, "b": 2, "psi": 3}
PRECISION = {"fp64": 0, "mixed": 1}
SHAPE = {"line": 2, "triag": 3, "quad": 4, "tetra": 10}
BC_KIND = {"WeakDirichlet": 0, "WeakWall": 1, "WeakSubInlet": 2, "WeakSubOutlet": 3,
           "WeakFarfield": 4, "StrongDirichlet": 5,
           "WeakSuperInlet": 6, "WeakSymmetry": 7}

STATUS = {0: "OK", 1: "INVALID", 2: "CUDA", 3: "NONFINITE", 4: "NEG_PRESSURE", 5: "ITER_CAP",
          6: "UNSUPPORTED", 7: "TOO_LARGE"}

# Symbols the C ABI exports (include/rds_b200.h).
EXPORTS = ["rds_create", "rds_add_cell_group", "rds_add_bc", "rds_finalize", "rds_set_state",
           "rds_get_state", "rds_assemble", "rds_assemble_rhs", "rds_update",
           "rds_residual_norm", "rds_get_fields", "rds_iterate", "rds_stream",
           "rds_kernel_timing", "rds_kernel_times", "rds_launch_count", "rds_destroy",
           "rds_last_error", "rds_version", "rds_run", "rds_measure_peak", "rds_set_option",
           "rds_set_problems", "rds_add_batch_cell_group", "rds_add_batch_bc",
           "rds_iterate_batch", "rds_autotune", "rds_residual_norm_noalloc",
           "rds_set_blending_coeff", "rds_set_artificial_viscosity", "rds_set_stab_tables",
           "rds_compute_stabilisation", "rds_advance_rk3tvd"]


class RDSError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"rds status {STATUS.get(status, status)}: {msg}")
        self.status = status


class _Desc(C.Structure):
    _fields_ = [("physics", C.c_int), ("scheme", C.c_int), ("precision", C.c_int),
                ("dim", C.c_int), ("neq", C.c_int), ("nnodes", C.c_int),
                ("ngeo_nodes", C.c_int), ("geo_coords", C.c_void_p),
                ("adv", C.c_double * 3), ("gamma", C.c_double)]


class _CellGroup(C.Structure):
    _fields_ = [("shape", C.c_int), ("order", C.c_int), ("ncells", C.c_int), ("ndof", C.c_int),
                ("ngeo", C.c_int), ("nq", C.c_int), ("nfl", C.c_int),
                ("sol_conn", C.c_void_p), ("geo_conn", C.c_void_p), ("w", C.c_void_p),
                ("V", C.c_void_p), ("dV", C.c_void_p), ("dVgeo", C.c_void_p),
                ("dVf", C.c_void_p), ("Vsf", C.c_void_p), ("nqv", C.c_int),
                ("wv", C.c_void_p), ("dVgeo_v", C.c_void_p)]


class _BCGroup(C.Structure):
    _fields_ = [("kind", C.c_int), ("nfacets", C.c_int), ("nfdof", C.c_int),
                ("nfgeo", C.c_int), ("nfq", C.c_int), ("sol_conn", C.c_void_p),
                ("geo_conn", C.c_void_p), ("fw", C.c_void_p), ("fV", C.c_void_p),
                ("fdVgeo", C.c_void_p), ("gq", C.c_void_p), ("order", C.c_int),
                ("params", C.c_double * 4)]


_lib = None


def lib():
    """Load librds_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m pdekit_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, ip, dp = C.c_void_p, C.c_int, C.c_double
    sig = {
        "rds_create": ([C.POINTER(vp), vp, vp], ip),
        "rds_add_cell_group": ([vp, vp], ip),
        "rds_add_bc": ([vp, vp], ip),
        "rds_finalize": ([vp], ip),
        "rds_set_state": ([vp, vp], ip),
        "rds_get_state": ([vp, vp], ip),
        "rds_assemble": ([vp, dp], ip),
        "rds_assemble_rhs": ([vp], ip),
        "rds_update": ([vp], ip),
        "rds_residual_norm": ([vp, vp], ip),
        "rds_get_fields": ([vp, vp, vp, vp, vp], ip),
        "rds_iterate": ([vp, dp, ip, dp, C.POINTER(ip), vp], ip),
        "rds_stream": ([vp], vp),
        "rds_kernel_timing": ([vp, ip], ip),
        "rds_kernel_times": ([vp, vp, vp, vp, ip], ip),
        "rds_launch_count": ([vp], C.c_longlong),
        "rds_destroy": ([vp], ip),
        "rds_last_error": ([vp], C.c_char_p),
        "rds_version": ([], C.c_char_p),
        "rds_run": ([vp, dp, ip], ip),
        "rds_advance_rk3tvd": ([vp, dp, ip], ip),
        "rds_measure_peak": ([ip, vp], ip),
        "rds_set_option": ([vp, C.c_char_p, dp], ip),
        "rds_set_problems": ([vp, ip, vp, vp], ip),
        "rds_add_batch_cell_group": ([vp, vp, ip, ip, vp], ip),
        "rds_add_batch_bc": ([vp, vp, ip], ip),
        "rds_iterate_batch": ([vp, ip, dp, vp, vp], ip),
        "rds_autotune": ([vp, C.c_char_p, ip], ip),
        "rds_set_dual_volume": ([vp, vp], ip),
        "rds_set_interface": ([vp, ip, vp, vp, ip, vp], ip),
        "rds_pack_interface": ([vp, vp], ip),
        "rds_unpack_interface": ([vp, vp], ip),
        "rds_finish": ([vp, dp, ip, vp], ip),
        "rds_assemble_rhs_cells": ([vp, ip, ip, ip], ip),
        "rds_gather_rhs": ([vp, ip, ip], ip),
        "rds_gather_finish": ([vp, ip, ip, dp, vp], ip),
        "rds_rk_stage_state": ([vp, ip], ip),
        "rds_gather_rk": ([vp, ip, ip, dp], ip),
        "rds_combine_rk": ([vp, ip, ip, dp], ip),
        "rds_finish_nodes": ([vp, dp, ip, ip, ip, vp], ip),
        "rds_check": ([vp], ip),
        "rds_element_jacobians": ([vp, ip, vp], ip),
        "rds_jacobian_pattern": ([vp, vp, vp, vp], ip),
        "rds_assemble_jacobian": ([vp, vp], ip),
        "rds_step_host": ([vp, vp, vp, dp, vp], ip),
        "rds_step_sync": ([vp], ip),
        "rds_set_blending_coeff": ([vp, vp], ip),
        "rds_set_artificial_viscosity": ([vp, vp], ip),
        "rds_set_stab_tables": ([vp, ip, ip, vp, vp, vp, ip, vp], ip),
        "rds_set_bonanni_tables": ([vp, ip, ip, vp, vp, vp, vp], ip),
        "rds_set_stab_geo_tables": ([vp, ip, ip, vp], ip),
        "rds_compute_stabilisation": ([vp, ip, dp, dp, ip, vp, vp], ip),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def measure_peak(precision: str = "fp64") -> float:
    """Measured CUDA-core FMA peak of the current GPU in TFLOP/s."""
    out = np.zeros(1)
    st = lib().rds_measure_peak(PRECISION[precision], _ptr(out))
    if st != 0:
        raise RDSError(st, "rds_measure_peak failed")
    return float(out[0])


class PGRDMethodExplicit:
    """GPU drop-in for PGRDMethodExplicit<MeshConfig, Physics, Scheme> (one CUDA context)."""

    def __init__(self, physics: str = "burgers", scheme: str = "b", precision: str = "fp64"):
        self.physics, self.scheme, self.precision = physics, scheme, precision
        self._ctx = None
        self._keep = []
        self.problem = None

    # ---- set-up -------------------------------------------------------------------------------
    def configure_mesh_data(self, prob: Problem):
        """RDMethod::configure_mesh_data + the reference tables of initialize_work_data."""
        L = lib()
        if prob.physics != self.physics or prob.scheme != self.scheme:
            # the problem description carries its physics; the scheme tag can be overridden
            prob = Problem(**{**prob.__dict__, "physics": self.physics, "scheme": self.scheme})
        self.problem = prob
        coords = np.ascontiguousarray(prob.geo_coords, dtype=np.float64)
        self._keep.append(coords)
        d = _Desc()
        d.physics = PHYSICS[self.physics]
        d.scheme = SCHEME[self.scheme]
        d.precision = PRECISION[self.precision]
        d.dim, d.neq, d.nnodes = prob.dim, prob.neq, prob.nnodes
        d.ngeo_nodes = coords.shape[0]
        d.geo_coords = _ptr(coords)
        for i, v in enumerate(prob.adv):
            d.adv[i] = v
        d.gamma = prob.gamma
        ctx = C.c_void_p()
        st = L.rds_create(C.byref(ctx), C.byref(d), None)
        self._ctx = ctx
        self._check(st)
        for g in prob.groups:
            arrs = [np.ascontiguousarray(g.sol_conn, dtype=np.int32),
                    np.ascontiguousarray(g.geo_conn, dtype=np.int32)] + \
                   [np.ascontiguousarray(x, dtype=np.float64) for x in
                    (g.w, g.V, g.dV, g.dVgeo, g.dVf, g.Vsf)]
            self._keep += arrs
            cg = _CellGroup(SHAPE[g.shape], g.order, g.ncells, g.ndof, g.ngeo, g.nq, g.nfl,
                            *[_ptr(a) for a in arrs])
            if g.wv is not None:
                va = [np.ascontiguousarray(g.wv, dtype=np.float64),
                      np.ascontiguousarray(g.dVgeo_v, dtype=np.float64)]
                self._keep += va
                cg.nqv, cg.wv, cg.dVgeo_v = va[0].shape[0], _ptr(va[0]), _ptr(va[1])
            self._check(L.rds_add_cell_group(self._ctx, C.byref(cg)))
        for b in prob.bcs:
            self.add_boundary_condition(b)
        return self

    def add_boundary_condition(self, b):
        """RDMethod::add_boundary_condition with its boundary data (`b.gq`: the boundary state
        at the facet quadrature points for WeakDirichlet, the reference state for WeakFarfield,
        the values of the facet dofs for StrongDirichlet)."""
        arrs = [np.ascontiguousarray(b.sol_conn, dtype=np.int32),
                np.ascontiguousarray(b.geo_conn, dtype=np.int32)] + \
               [np.ascontiguousarray(x, dtype=np.float64) for x in (b.fw, b.fV, b.fdVgeo, b.gq)]
        self._keep += arrs
        cb = _BCGroup(BC_KIND[b.kind], b.nfacets, b.nfdof, b.nfgeo, b.nfq,
                      *[_ptr(a) for a in arrs])
        cb.order = b.order
        for k, v in enumerate(b.params[:4]):
            cb.params[k] = v
        self._check(lib().rds_add_bc(self._ctx, C.byref(cb)))

    def initialize_work_data(self):
        self._check(lib().rds_finalize(self._ctx))
        # tables of the stabilisation operators: the vertex interpolant of every group, the
        # smoothness sensor's where it is defined (affine simplices, bilinear quadrilaterals)
        from .reference_element import bonanni_tables, stab_tables
        for ig, g in enumerate(self.problem.groups):
            t = stab_tables(g.shape, g.order, g.ngeo)
            arrs = [t[k] for k in ("w", "Vn", "R", "P1")]
            self._keep += arrs
            self._check(lib().rds_set_stab_tables(self._ctx, ig, t["nq"], *[_ptr(a) for a in arrs[:3]],
                                                  t["P1"].shape[1], _ptr(arrs[3])))
            if t["nq"] and "dVgeo" in t:
                self._keep.append(t["dVgeo"])
                self._check(lib().rds_set_stab_geo_tables(self._ctx, ig, t["dVgeo"].shape[2],
                                                          _ptr(t["dVgeo"])))
            if self.problem.neq > 1:  # Bonanni's coefficient (Euler)
                b = bonanni_tables(g.shape, g.order, g.ngeo)
                if b["nq"]:
                    arrs = [b[k] for k in ("w", "V", "dV", "dVgeo")]
                    self._keep += arrs
                    self._check(lib().rds_set_bonanni_tables(self._ctx, ig, b["nq"],
                                                             *[_ptr(a) for a in arrs]))
        return self

    # ---- stabilisation fields (RDMethod::set_blending_coeff / set_artificial_viscosity) -------
    def set_blending_coeff(self, theta):
        """External nodal blending coefficient [nnodes] read by PGB cells (None removes it)."""
        self._check(lib().rds_set_blending_coeff(self._ctx, None if theta is None else
                                                 _ptr(self._nodal(theta, "theta"))))

    def set_artificial_viscosity(self, eps):
        """Nodal artificial viscosity [nnodes] added by PGLDA cells (None removes it)."""
        self._check(lib().rds_set_artificial_viscosity(self._ctx, None if eps is None else
                                                       _ptr(self._nodal(eps, "eps"))))

    def compute_stabilisation(self, op: int, p0: float = 0.0, p1: float = 1.0,
                              install: bool = False, cells: bool = True, nodes: bool = False):
        """Operator `op` (RDS_STAB_*) on the current state: (cell values [total cells] or None,
        nodal field [nnodes] or None); install=True makes the nodal field the solver's
        artificial viscosity / blending coefficient."""
        nc = sum(g.ncells for g in self.problem.groups)
        cv = np.empty(nc) if cells else None
        nv = np.empty(self.problem.nnodes) if nodes else None
        self._check(lib().rds_compute_stabilisation(
            self._ctx, int(op), float(p0), float(p1), int(bool(install)),
            None if cv is None else _ptr(cv), None if nv is None else _ptr(nv)))
        return cv, nv

    def _nodal(self, a, name):
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        if a.size != self.problem.nnodes:
            raise ValueError(f"{name} must hold {self.problem.nnodes} nodal values")
        return a

    # ---- fields -------------------------------------------------------------------------------
    def set_solution(self, u):
        p = self.problem
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(p.nnodes, p.neq)
        self._check(lib().rds_set_state(self._ctx, _ptr(u)))

    def solution(self, out=None):
        p = self.problem
        u = np.empty((p.nnodes, p.neq)) if out is None else out
        self._check(lib().rds_get_state(self._ctx, _ptr(u)))
        return u

    def fields(self):
        """(residual [n,neq], dt [n], nodal wave speed [n], dual volume [n])."""
        p = self.problem
        res = np.empty((p.nnodes, p.neq))
        dt, ws, vol = np.empty(p.nnodes), np.empty(p.nnodes), np.empty(p.nnodes)
        self._check(lib().rds_get_fields(self._ctx, _ptr(res), _ptr(dt), _ptr(ws), _ptr(vol)))
        return res, dt, ws, vol

    # ---- iteration ----------------------------------------------------------------------------
    def assemble_lhs_and_rhs(self, cfl: float):
        self._check(lib().rds_assemble(self._ctx, float(cfl)))

    def assemble_rhs(self):
        self._check(lib().rds_assemble_rhs(self._ctx))

    def solve(self):
        self._check(lib().rds_update(self._ctx))

    def compute_residual_norm(self):
        out = np.zeros(self.problem.neq)
        self._check(lib().rds_residual_norm(self._ctx, _ptr(out)))
        return out

    def iterate(self, cfl: float, max_iter: int, drop: float = 0.0, raise_on_cap=True):
        """Device loop of assemble_lhs_and_rhs + solve; returns (iterations, norm history)."""
        hist = np.zeros((max_iter, self.problem.neq))
        done = C.c_int(0)
        st = lib().rds_iterate(self._ctx, float(cfl), int(max_iter), float(drop),
                               C.byref(done), _ptr(hist))
        if st == 5 and not raise_on_cap:
            return done.value, hist[:done.value]
        self._check(st)
        return done.value, hist[:done.value]

    def element_jacobians(self, group: int = 0):
        """PGLDA element Jacobians [ncells, ndof * neq, ndof * neq] of a cell group at the
        current state (computed on the GPU, copied to the host)."""
        import torch

        g = self.problem.groups[group]
        nr = g.ndof * self.problem.neq
        jac = torch.empty((g.ncells, nr, nr), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        self._check(lib().rds_element_jacobians(self._ctx, int(group), C.c_void_p(jac.data_ptr())))
        torch.cuda.ExternalStream(self.stream_handle()).synchronize()
        self._check(lib().rds_check(self._ctx))
        return jac.cpu().numpy()

    def assemble_jacobian(self):
        """Block-CSR Jacobian at the current state: (row_ptr [n + 1], col_idx [nnzb],
        values [nnzb, neq, neq]), block (v, w) divided by the dual volume of v."""
        import torch

        nnzb = C.c_int64(0)
        self._check(lib().rds_jacobian_pattern(self._ctx, C.byref(nnzb), None, None))
        row_ptr = np.zeros(self.problem.nnodes + 1, dtype=np.int32)
        col_idx = np.zeros(nnzb.value, dtype=np.int32)
        self._check(lib().rds_jacobian_pattern(self._ctx, C.byref(nnzb), _ptr(row_ptr),
                                               _ptr(col_idx)))
        neq = self.problem.neq
        vals = torch.empty((nnzb.value, neq, neq), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        self._check(lib().rds_assemble_jacobian(self._ctx, C.c_void_p(vals.data_ptr())))
        torch.cuda.ExternalStream(self.stream_handle()).synchronize()
        self._check(lib().rds_check(self._ctx))
        return row_ptr, col_idx, vals.cpu().numpy()

    def step_host(self, u_in, u_out, cfl: float, norm=None):
        """One pipelined step on host arrays (pinned for overlap): returns without waiting;
        call step_sync() before reading u_out / norm or reusing u_in. The arrays are used in
        place (no copies): float64, C-contiguous, nnodes x neq values (norm: neq)."""
        p = self.problem
        for nm, a, n in (("u_in", u_in, p.nnodes * p.neq), ("u_out", u_out, p.nnodes * p.neq),
                         ("norm", norm, p.neq)):
            if a is None and nm == "norm":
                continue
            if (not isinstance(a, np.ndarray) or a.dtype != np.float64
                    or not a.flags.c_contiguous or a.size != n):
                raise ValueError(f"step_host: {nm} must be a C-contiguous float64 array of "
                                 f"{n} values")
        self._check(lib().rds_step_host(self._ctx, _ptr(u_in), _ptr(u_out), float(cfl),
                                        None if norm is None else _ptr(norm)))

    def step_sync(self):
        self._check(lib().rds_step_sync(self._ctx))

    def set_option(self, key: str, value: float):
        self._check(lib().rds_set_option(self._ctx, key.encode(), float(value)))

    def check(self):
        """Waits for the context's stream and raises the status the device recorded (a
        non-finite norm, a non-positive pressure, a bounded wait that gave up)."""
        self._check(lib().rds_check(self._ctx))

    def run(self, cfl: float, n: int):
        """Enqueue n fused iterations without waiting (for event timing on stream_handle())."""
        self._check(lib().rds_run(self._ctx, float(cfl), int(n)))

    def advance_rk3tvd(self, cfl: float, nsteps: int = 1):
        """nsteps third-order TVD Runge-Kutta steps on the device (enqueued without waiting);
        afterwards residual and dt are those of the last step's first stage."""
        self._check(lib().rds_advance_rk3tvd(self._ctx, float(cfl), int(nsteps)))

    # ---- diagnostics --------------------------------------------------------------------------
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


class ExplicitEuler:
    """Forward-Euler pseudo-time stepper over a solver (solver/time/ExplicitTimeStepper.cpp:
    36-40): assemble_lhs_and_rhs(CFL) then solve()."""

    def setup(self, nb_fields: int, nb_entries: int):
        pass

    def advance_in_time(self, scheme: PGRDMethodExplicit, CFL: float):
        scheme.assemble_lhs_and_rhs(CFL)
        scheme.solve()


class RK3TVD:
    """Third-order TVD Runge-Kutta stepper (solver/time/ExplicitTimeStepper.cpp:46-100). The
    three stages run on the device in one graph launch (rds_advance_rk3tvd); the stage states
    live in the solver's context, so setup() has nothing to allocate."""

    def setup(self, nb_fields: int, nb_entries: int):
        pass

    def advance_in_time(self, scheme: PGRDMethodExplicit, CFL: float):
        scheme.advance_rk3tvd(CFL, 1)
