"""ctypes front end of the C restatement (rds_oracle.c) -- TEST ORACLE ONLY.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, where it is
the checker. It consumes the same problem description (pdekit_b200.problem.Problem) as the
GPU path so both run on identical inputs.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "librds_oracle.so")
HARNESS_PATH = os.path.join(_HERE, "_ref", "rds_ref_harness")

PHYSICS = {"advconst": 0, "burgers": 1, "euler2d": 2, "euler3d": 3}
SCHEME = {"lda": 0, "n": 1, "b": 2, "psi": 3}
BC_KIND = {"WeakDirichlet": 0, "WeakWall": 1, "WeakSubInlet": 2, "WeakSubOutlet": 3,
           "WeakFarfield": 4, "StrongDirichlet": 5,
           "WeakSuperInlet": 6, "WeakSymmetry": 7}


class _Model(C.Structure):
    _fields_ = [("physics", C.c_int), ("scheme", C.c_int), ("dim", C.c_int), ("neq", C.c_int),
                ("adv", C.c_double * 3), ("gamma", C.c_double), ("gas_R", C.c_double)]


class _Cells(C.Structure):
    _fields_ = [("ncells", C.c_int), ("ndof", C.c_int), ("ngeo", C.c_int), ("nq", C.c_int),
                ("nfl", C.c_int), ("sol_conn", C.c_void_p), ("geo_conn", C.c_void_p),
                ("w", C.c_void_p), ("V", C.c_void_p), ("dV", C.c_void_p),
                ("dVgeo", C.c_void_p), ("dVf", C.c_void_p), ("Vsf", C.c_void_p),
                ("nqv", C.c_int), ("wv", C.c_void_p), ("dVgeo_v", C.c_void_p)]


class _BC(C.Structure):
    _fields_ = [("kind", C.c_int), ("nfacets", C.c_int), ("nfdof", C.c_int), ("nfgeo", C.c_int),
                ("nfq", C.c_int), ("sol_conn", C.c_void_p), ("geo_conn", C.c_void_p),
                ("fw", C.c_void_p), ("fV", C.c_void_p), ("fdVgeo", C.c_void_p),
                ("gq", C.c_void_p), ("order", C.c_int), ("params", C.c_double * 4)]


def build() -> None:
    """Compile the C restatement (gcc) into oracle/_ref/."""
    subprocess.run(["make", "-C", _HERE, "port"], check=True, capture_output=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.rdso_dual_volume.argtypes = [vp, vp, C.c_int, C.c_int, vp, vp]
        L.rdso_assemble.argtypes = [vp, vp, C.c_int, vp, C.c_int, C.c_int, vp, vp, vp, C.c_double,
                                    vp, vp, vp]
        L.rdso_assemble.restype = C.c_int
        L.rdso_update.argtypes = [C.c_int, C.c_int, vp, vp, vp]
        L.rdso_residual_norm.argtypes = [C.c_int, C.c_int, vp, vp, vp]
        L.rdso_cell_residual.argtypes = [vp, vp, vp, vp, vp, vp]
        L.rdso_element_jacobian.argtypes = [vp, vp, vp, vp, vp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Oracle:
    """Holds the ctypes structs for one problem; arrays are kept alive on the instance."""

    def __init__(self, prob):
        self.prob = prob
        self._keep = []
        m = _Model()
        m.physics = PHYSICS[prob.physics]
        m.scheme = SCHEME[prob.scheme]
        m.dim = prob.dim
        m.neq = prob.neq
        for i, v in enumerate(prob.adv):
            m.adv[i] = v
        m.gamma = prob.gamma
        m.gas_R = 287.05
        self.model = m
        self.groups = (_Cells * len(prob.groups))()
        for i, g in enumerate(prob.groups):
            arrs = [np.ascontiguousarray(x) for x in
                    (g.sol_conn, g.geo_conn, g.w, g.V, g.dV, g.dVgeo, g.dVf, g.Vsf)]
            self._keep += arrs
            c = self.groups[i]
            c.ncells, c.ndof, c.ngeo, c.nq, c.nfl = g.ncells, g.ndof, g.ngeo, g.nq, g.nfl
            (c.sol_conn, c.geo_conn, c.w, c.V, c.dV, c.dVgeo, c.dVf, c.Vsf) = [_p(a) for a in arrs]
            if g.wv is not None:
                va = [np.ascontiguousarray(g.wv, dtype=np.float64),
                      np.ascontiguousarray(g.dVgeo_v, dtype=np.float64)]
                self._keep += va
                c.nqv, c.wv, c.dVgeo_v = va[0].shape[0], _p(va[0]), _p(va[1])
        nb = max(1, len(prob.bcs))
        self.bcs = (_BC * nb)()
        for i, b in enumerate(prob.bcs):
            arrs = [np.ascontiguousarray(x) for x in
                    (b.sol_conn, b.geo_conn, b.fw, b.fV, b.fdVgeo, b.gq)]
            self._keep += arrs
            s = self.bcs[i]
            s.kind, s.nfacets, s.nfdof, s.nfgeo, s.nfq = (BC_KIND[b.kind], b.nfacets, b.nfdof,
                                                          b.nfgeo, b.nfq)
            s.order = b.order
            for k, v in enumerate(b.params[:4]):
                s.params[k] = v
            (s.sol_conn, s.geo_conn, s.fw, s.fV, s.fdVgeo, s.gq) = [_p(a) for a in arrs]
        self.coords = np.ascontiguousarray(prob.geo_coords, dtype=np.float64)
        self.vol = np.zeros(prob.nnodes)
        lib().rdso_dual_volume(C.byref(self.model), self.groups, len(prob.groups), prob.nnodes,
                               _p(self.coords), _p(self.vol))

    def _assemble_inplace(self, u, cfl):
        prob = self.prob
        res = np.zeros_like(u)
        ws = np.zeros(prob.nnodes)
        dt = np.zeros(prob.nnodes)
        bad = lib().rdso_assemble(C.byref(self.model), self.groups, len(prob.groups), self.bcs,
                                  len(prob.bcs), prob.nnodes, _p(self.coords), _p(self.vol),
                                  _p(u), float(cfl), _p(res), _p(ws), _p(dt))
        return res, ws, dt, bad

    def assemble(self, u, cfl):
        """Returns (res [n,neq], ws [n], dt [n], nbad); `u` is not modified (the state after
        the strong conditions is `self.last_state`)."""
        prob = self.prob
        u = np.array(u, dtype=np.float64).reshape(prob.nnodes, prob.neq)
        out = self._assemble_inplace(u, cfl)
        self.last_state = u
        return out

    def iterate(self, u, cfl, iters):
        """iters x (assemble + solve). Returns (u, norms [iters, neq])."""
        prob = self.prob
        u = np.array(u, dtype=np.float64).reshape(prob.nnodes, prob.neq)
        norms = np.zeros((iters, prob.neq))
        for it in range(iters):
            res, ws, dt, _ = self._assemble_inplace(u, cfl)
            nrm = np.zeros(prob.neq)
            lib().rdso_residual_norm(prob.nnodes, prob.neq, _p(res), _p(dt), _p(nrm))
            norms[it] = nrm
            lib().rdso_update(prob.nnodes, prob.neq, _p(dt), _p(res), _p(u))
        return u, norms

    def rk3tvd(self, u, cfl, steps):
        """`steps` x RK3TVD::advance_in_time (solver/time/ExplicitTimeStepper.cpp:66-100).
        Every stage assembles at its own state (cells and conditions read it; strong conditions
        overwrite it) and the later stages reuse the first stage's dt. Returns (u, residual and
        dt of the last step's first stage, norms [steps, neq] after each step)."""
        prob = self.prob
        un = np.array(u, dtype=np.float64).reshape(prob.nnodes, prob.neq)
        norms = np.zeros((steps, prob.neq))
        for k in range(steps):
            res_n, _, dt, _ = self._assemble_inplace(un, cfl)
            d = dt[:, None]
            u1 = un - d * res_n
            r, _, _, _ = self._assemble_inplace(u1, cfl)
            u2 = 3. / 4. * un + 1. / 4. * u1 - 1. / 4. * (d * r)
            r, _, _, _ = self._assemble_inplace(u2, cfl)
            un = 1. / 3. * un + 2. / 3 * u2 - 2. / 3. * (d * r)
            lib().rdso_residual_norm(prob.nnodes, prob.neq, _p(res_n), _p(dt), _p(norms[k]))
        return un, res_n, dt, norms

    def cell_residual(self, group, cell, u):
        """Scheme residual [ndof, neq] and wave speed [ndof] of one cell from the state u."""
        prob, g = self.prob, self.prob.groups[group]
        X = np.ascontiguousarray(prob.geo_coords[g.geo_conn[cell]], dtype=np.float64)
        un = np.ascontiguousarray(np.asarray(u).reshape(-1, prob.neq)[g.sol_conn[cell]])
        res = np.zeros((g.ndof, prob.neq))
        ws = np.zeros(g.ndof)
        lib().rdso_cell_residual(C.byref(self.model), C.byref(self.groups[group]), _p(X), _p(un),
                                 _p(res), _p(ws))
        return res, ws

    def element_jacobian(self, group, cell, u):
        """Element Jacobian [ndof * neq, ndof * neq] of one cell at the state u (PGLDA, or PGN
        when the problem's scheme is "n")."""
        if self.prob.scheme == "psi":
            raise ValueError("no element Jacobians for the PSI scheme")
        prob, g = self.prob, self.prob.groups[group]
        X = np.ascontiguousarray(prob.geo_coords[g.geo_conn[cell]], dtype=np.float64)
        un = np.ascontiguousarray(np.asarray(u).reshape(-1, prob.neq)[g.sol_conn[cell]])
        nr = g.ndof * prob.neq
        jac = np.zeros((nr, nr))
        lib().rdso_element_jacobian(C.byref(self.model), C.byref(self.groups[group]), _p(X),
                                    _p(un), _p(jac))
        return jac
