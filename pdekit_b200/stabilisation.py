"""Stabilisation operators with the reference's class interface, on the GPU solver's state.

The reference computes these fields on the host from a solution function and hands them to
the solver (examples/testcases-rdm/Burgers-RDS-2D.cpp:121-176):

    ArtificialViscosity<MeshConfig> av;  av.prepare_indicator_operators(sol_dofs);
    av.compute_artificial_viscosity_nodal(mesh, sol_dofs, u, art_visc_nodal);
    scheme->set_artificial_viscosity(art_visc_nodal);

    RDBlendingCoeff<MeshConfig> bc;  bc.setup(sol_dofs, "LF_Blend");
    bc.calculate(mesh, sol_dofs, u, blending_coeff);  scheme->set_blending_coeff(blending_coeff);

Here the state, the mesh and the fields stay on the device: the operators take the solver
(`PGRDMethodExplicit`), read its current state, and with install=True make the nodal field the
solver's own in the same call (no host round trip). The values are returned as numpy arrays
when asked for. Cell values are in the solver's cell order (groups in order).

* ArtificialViscosity (src/solver/art_visc/ArtificialViscosity.hpp): the Persson-Peraire
  smoothness sensor of the first state component, kappa (default 5) and factor (default 1);
  affine triangles (orders 1-3), tetrahedra (orders 1-2) and bilinear quadrilaterals (orders
  1-3; from order 2 the reference's own value there follows the rounding of a singular mass
  matrix, and the sensor takes the projection every regular mass matrix gives).
* RDBlendingCoeff (src/solver/rdm/blending_coeff/RDBlendingCoeff.hpp): "LF_Blend" (any cell
  type), "ViscosityIndicator" (param "kappa", the sensor as a coefficient in [0, 1]; the
  sensor's cells), "WongJansen" (param "u_inf", default 1e-14; any cell type), "Bonanni2D" /
  "Bonanni3D" (Euler; the pressure-based coefficient, no parameters; straight-sided cells).
"""

from __future__ import annotations

from .rds import PGRDMethodExplicit

# rds_stab_op (include/rds_b200.h)
ART_VISC, INDICATOR, BLEND_LF, BLEND_VISC, BLEND_WONG_JANSEN, BLEND_BONANNI = range(6)


class ArtificialViscosity:
    def __init__(self):
        self.solver = None

    def prepare_indicator_operators(self, solver: PGRDMethodExplicit):
        """Bind to a configured solver (its initialize_work_data set the sensor tables)."""
        self.solver = solver
        return self

    def _s(self, solver):
        s = solver if solver is not None else self.solver
        if s is None:
            raise RuntimeError("prepare_indicator_operators(solver) first")
        return s

    def compute_artificial_viscosity(self, solver=None, kappa: float = 5.0, factor: float = 1.0):
        """Cellwise viscosity [total cells]."""
        return self._s(solver).compute_stabilisation(ART_VISC, kappa, factor)[0]

    def compute_indicator(self, solver=None, kappa: float = 5.0):
        """Cellwise viscosity with factor 1 (the reference's compute_indicator)."""
        return self.compute_artificial_viscosity(solver, kappa, 1.0)

    def compute_indicator_normalized(self, solver=None, kappa: float = 5.0):
        """compute_indicator divided by its maximum (unless that is below 1e-14)."""
        return self._s(solver).compute_stabilisation(INDICATOR, kappa)[0]

    def compute_artificial_viscosity_nodal(self, solver=None, kappa: float = 5.0,
                                           factor: float = 1.0, install: bool = True):
        """Nodal viscosity [nnodes]; install=True also makes it the solver's artificial
        viscosity (set_artificial_viscosity)."""
        return self._s(solver).compute_stabilisation(ART_VISC, kappa, factor, install=install,
                                                     cells=False, nodes=True)[1]


class RDBlendingCoeff:
    _TYPES = {"LF_Blend": BLEND_LF, "ViscosityIndicator": BLEND_VISC,
              "WongJansen": BLEND_WONG_JANSEN, "Bonanni2D": BLEND_BONANNI,
              "Bonanni3D": BLEND_BONANNI}

    def __init__(self):
        self.solver, self.op = None, None
        self.params = {"kappa": 5.0, "u_inf": 1.e-14}

    def setup(self, solver: PGRDMethodExplicit, coeff_type: str):
        if coeff_type not in self._TYPES:
            raise ValueError(f"blending coefficient type {coeff_type!r} is not provided "
                             f"(have {sorted(self._TYPES)})")
        if coeff_type.startswith("Bonanni") and solver.problem.dim != int(coeff_type[-2]):
            raise ValueError(f"{coeff_type} on a {solver.problem.dim}D problem")
        self.solver, self.op = solver, self._TYPES[coeff_type]
        return self

    def set_param(self, name: str, value: float):
        """'kappa' (ViscosityIndicator) or 'u_inf' (WongJansen); others are ignored, as in the
        reference."""
        if name in self.params:
            self.params[name] = float(value)

    def _p0(self):
        return self.params["u_inf"] if self.op == BLEND_WONG_JANSEN else self.params["kappa"]

    def calculate(self, install: bool = True):
        """Nodal coefficient [nnodes]; install=True also makes it the solver's blending
        coefficient (set_blending_coeff)."""
        return self.solver.compute_stabilisation(self.op, self._p0(), 1.0, install=install,
                                                 cells=False, nodes=True)[1]

    def calculate_in_cells(self):
        """Cellwise coefficient [total cells]."""
        return self.solver.compute_stabilisation(self.op, self._p0(), 1.0)[0]

    def clear(self):
        self.solver, self.op = None, None
