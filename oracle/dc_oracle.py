"""Test oracle (CPU, numpy, FP64) of the mixed form's defect-correction loop.

Test infrastructure only: the tests import it as the checker of the CUDA path
(pdekit_b200/csrc/rds_cells_scalar_dc.cu and the loop in rds_api.cu); the library never does.

The loop has no counterpart in the reference, which iterates in FP64 only. What it restates
here is the library's own linearisation of the reference's scalar cell residual:

  ScalarCells.residual(u)   the cell residual of PGLDA / PGN / PGB on straight-sided triangles,
                            following src/solver/rdm/cellsplitters/PGLDA.hpp:171-310,
                            PGN.hpp:154-289, PGB.hpp:314-498 (checked against the C
                            restatement oracle/rds_oracle.c, which the golden cases pin to the
                            reference), plus the blending coefficient theta of each cell;
  ScalarCells.delta(ur, d)  its change from ur to ur + d with the distribution coefficients
                            (K+, beta, theta) of ur and the flux change exact in d;
  dc_iterate(...)           cycles of one exact sweep (the reference's assemble + solve, by the
                            C restatement) and m - 1 correction sweeps
                            u -= dt(ur) [R_cells(ur) + delta(ur, u - ur) / V + R_bc(u)].
"""

from __future__ import annotations

import dataclasses

import numpy as np

from .rds_oracle import Oracle


class ScalarCells:
    """Scalar cell residuals of one straight-sided triangle group, vectorised over cells."""

    def __init__(self, prob, group=0):
        assert prob.physics in ("advconst", "burgers") and prob.dim == 2
        g = prob.groups[group]
        assert g.ngeo == 3, "straight-sided triangles only"
        self.prob, self.g = prob, g
        X = prob.geo_coords[g.geo_conn]  # [nc, 3, 2]
        J = np.einsum("dg,cgk->cdk", g.dVgeo[:, 0, :], X)
        det = J[:, 0, 0] * J[:, 1, 1] - J[:, 0, 1] * J[:, 1, 0]
        self.ij00, self.ij11 = J[:, 1, 1] / det, J[:, 0, 0] / det
        self.ij01, self.ij10 = -J[:, 0, 1] / det, -J[:, 1, 0] / det
        self.wj = g.w[None, :] * det[:, None]  # [nc, nq]

    def _coeffs(self, uc):
        """Upwind coefficients at the points for cell states uc [nc, ndof]: K+ [nc, nq, ndof]."""
        g, p = self.g, self.prob
        if p.physics == "burgers":
            ax, ay = uc @ g.V.T, 1.0  # u_q
        else:
            ax, ay = p.adv[0], p.adv[1]
        A = ax * self.ij00[:, None] + ay * self.ij10[:, None]
        B = ax * self.ij01[:, None] + ay * self.ij11[:, None]
        k = g.dV[0][None] * A[..., None] + g.dV[1][None] * B[..., None]
        return np.maximum(k, 0.0)

    def _divergence(self, F0, F1):
        """d F_d / d x_d at the points from flux-node values F0, F1 [nc, nfl]."""
        g = self.g
        G0 = self.ij00[:, None] * F0 + self.ij10[:, None] * F1
        G1 = self.ij01[:, None] * F0 + self.ij11[:, None] * F1
        return G0 @ g.dVf[0].T + G1 @ g.dVf[1].T

    def _flux(self, s):
        p = self.prob
        if p.physics == "burgers":
            return 0.5 * s * s, s
        return p.adv[0] * s, p.adv[1] * s

    def _schemes(self, kp, r, uc):
        """LDA part, N dissipation [nc, ndof] for K+ kp, point values r [nc, nq], states uc."""
        S = kp.sum(-1)
        ek = (self.wj / S)[..., None] * kp
        lda = np.einsum("cqn,cq->cn", ek, r)
        tk = np.einsum("cqm,cm->cq", kp, uc)
        diss = np.einsum("cqn,cqn->cn", ek, uc[:, None, :] * S[..., None] - tk[..., None])
        return lda, diss

    def residual(self, u):
        """(cell contributions [nc, ndof], theta [nc]) at the nodal state u [nnodes]."""
        g, scheme = self.g, self.prob.scheme
        uc = u[g.sol_conn]
        r = self._divergence(*self._flux(uc @ g.Vsf.T))
        lda, diss = self._schemes(self._coeffs(uc), r, uc)
        phi = (self.wj * r).sum(-1)
        theta = np.abs(phi) / (np.abs(lda + diss).sum(-1) + 1.0e-6)
        if scheme == "lda":
            return lda, theta
        if scheme == "n":
            return lda + diss, theta
        return lda + theta[:, None] * diss, theta

    def delta(self, ur, d, theta):
        """Change of the cell contributions from ur to ur + d with the coefficients of ur
        (K+, beta and, for PGB, the blending coefficient theta of ur)."""
        g, p = self.g, self.prob
        urc, dc = ur[g.sol_conn], d[g.sol_conn]
        sr, ds = urc @ g.Vsf.T, dc @ g.Vsf.T
        if p.physics == "burgers":
            dF0, dF1 = ds * (sr + 0.5 * ds), ds
        else:
            dF0, dF1 = p.adv[0] * ds, p.adv[1] * ds
        lda, diss = self._schemes(self._coeffs(urc), self._divergence(dF0, dF1), dc)
        if p.scheme == "lda":
            return lda
        if p.scheme == "n":
            return lda + diss
        return lda + theta[:, None] * diss

    def nodal(self, contrib, vol):
        out = np.zeros(self.prob.nnodes)
        np.add.at(out, self.g.sol_conn, contrib)
        return out / vol


def dc_iterate(prob, u0, cfl, m, nsweeps):
    """nsweeps sweeps of the defect-correction loop from u0 (FP64 throughout): an exact sweep
    (C restatement assemble + update) at sweeps 0, m, 2m, ...; correction sweeps in between.
    Returns the state after the sweeps."""
    full = Oracle(prob)
    cells_only = Oracle(dataclasses.replace(prob, bcs=[]))
    sc = ScalarCells(prob)
    u = np.array(u0, dtype=np.float64).reshape(-1).copy()
    # the cells read the state as the sweep finds it; strong Dirichlet conditions overwrite
    # their dofs after the cells (full.last_state), and the update starts from that state
    for k in range(nsweeps):
        if k % m == 0:
            rc = cells_only.assemble(u[:, None], cfl)[0][:, 0]
            theta = sc.residual(u)[1]
            res, _, dt, _ = full.assemble(u[:, None], cfl)
            ur, dtr, rcell = full.last_state[:, 0].copy(), dt.copy(), rc
            u = ur - dtr * res[:, 0]
            continue
        rc = cells_only.assemble(u[:, None], cfl)[0][:, 0]
        dcell = sc.nodal(sc.delta(ur, u - ur, theta), full.vol)
        rall = full.assemble(u[:, None], cfl)[0][:, 0]
        inc = rcell + dcell + (rall - rc)
        u = full.last_state[:, 0] - dtr * inc
    return u[:, None]
