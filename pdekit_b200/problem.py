"""Problem description shared by the GPU solver and its checkers.

A problem is what the reference's RDMethod is configured with before the pseudo-time loop
(src/solver/rdm/RDMethod.hpp:159-243): the physics and scheme (template arguments of
PGRDMethodExplicit), geometry node coordinates, one group of cells per element type with its
reference-element tables (FEValues: V, dV, quadrature weights; FluxSpaceMetric: dVf, Vsf), and
one group of boundary facets per weak boundary condition with its facet tables and the
boundary state at the facet quadrature points.

All arrays are host numpy arrays; layouts are row-major, derivative tables are stacked
[dim][rows][cols], connectivities are int32 [entities][local nodes].
"""

from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class CellGroup:
    sol_conn: np.ndarray  # [ncells, ndof] int32
    geo_conn: np.ndarray  # [ncells, ngeo] int32
    w: np.ndarray  # [nq]
    V: np.ndarray  # [nq, ndof]
    dV: np.ndarray  # [dim, nq, ndof]
    dVgeo: np.ndarray  # [dim, nq, ngeo]
    dVf: np.ndarray  # [dim, nq, nfl]
    Vsf: np.ndarray  # [nfl, ndof]
    shape: str = "triag"
    order: int = 1
    wv: np.ndarray = None  # [nqv] dual-volume rule (Gauss rule of the cell order), optional
    dVgeo_v: np.ndarray = None  # [dim, nqv, ngeo]

    @property
    def ncells(self):
        return self.sol_conn.shape[0]

    @property
    def ndof(self):
        return self.sol_conn.shape[1]

    @property
    def ngeo(self):
        return self.geo_conn.shape[1]

    @property
    def nq(self):
        return self.w.shape[0]

    @property
    def nfl(self):
        return self.Vsf.shape[0]


@dataclasses.dataclass
class BCGroup:
    kind: str  # WeakDirichlet | WeakWall | WeakSubInlet | WeakSubOutlet | WeakFarfield |
    # WeakSuperInlet | WeakSymmetry |
    # StrongDirichlet
    name: str
    sol_conn: np.ndarray  # [nfacets, nfdof] int32
    geo_conn: np.ndarray  # [nfacets, nfgeo] int32
    fw: np.ndarray  # [nfq]
    fV: np.ndarray  # [nfq, nfdof]
    fVgeo: np.ndarray  # [nfq, nfgeo]
    fdVgeo: np.ndarray  # [dim-1, nfq, nfgeo]
    # WeakDirichlet: [nfacets, nfq, neq] boundary state at the facet quadrature points;
    # WeakFarfield: [neq] reference state (conservative); StrongDirichlet: [nfacets, nfdof, neq]
    # values the facet dofs take (facet by facet, a shared dof keeps the later value)
    gq: np.ndarray
    order: int = 1  # polynomial order of the facet's solution basis
    params: tuple = (0.0, 0.0, 0.0, 0.0)  # WeakSubInlet: (T_tot, p_tot); WeakSubOutlet: (p,)

    @property
    def nfacets(self):
        return self.sol_conn.shape[0]

    @property
    def nfdof(self):
        return self.sol_conn.shape[1]

    @property
    def nfgeo(self):
        return self.geo_conn.shape[1]

    @property
    def nfq(self):
        return self.fw.shape[0]

    def quadrature_coords(self, geo_coords):
        """Physical coordinates of the facet quadrature points [nfacets, nfq, dim]."""
        X = geo_coords[self.geo_conn]  # [nf, nfgeo, dim]
        return np.einsum("qg,fgd->fqd", self.fVgeo, X)


@dataclasses.dataclass
class Problem:
    physics: str  # advconst | burgers | euler2d | euler3d
    scheme: str  # lda | n | b
    dim: int
    neq: int
    nnodes: int
    geo_coords: np.ndarray  # [ngeo_nodes, dim]
    groups: list
    bcs: list
    adv: tuple = (0.0, 0.0, 0.0)
    gamma: float = 1.4

    @property
    def ncells(self):
        return sum(g.ncells for g in self.groups)


ADV_CONST_DIR = (0.5 / np.sqrt(1.25), 1.0 / np.sqrt(1.25), 0.0)
