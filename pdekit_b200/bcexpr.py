"""Named boundary-state expressions of the benchmark configurations.

The reference's WeakDirichletBC takes a function pointer g(x, u, eq)
(src/solver/rdm/bc/RDMBCBase.hpp:112-114) and evaluates it at every facet quadrature point
(src/solver/rdm/bc/WeakDirichletBC.hpp:225-228). The configurations' inflow data depend on the
coordinates only, so the host evaluates them once at setup and hands the values to the device.
"""

from __future__ import annotations

import numpy as np


def evaluate(name: str, xq: np.ndarray, neq: int) -> np.ndarray:
    """Values [..., neq] of the named expression at coordinates xq [..., dim]."""
    x = xq[..., 0]
    if name == "zero":
        v = np.zeros_like(x)
    elif name == "sin2pix":
        v = np.sin(2.0 * np.pi * x)
    elif name == "burgers_inlet":
        v = 1.5 - 2.0 * x
    elif name == "c1.5":
        v = np.full_like(x, 1.5)
    elif name == "c-0.5":
        v = np.full_like(x, -0.5)
    else:
        raise ValueError(f"unknown boundary expression {name!r}")
    out = np.zeros(x.shape + (neq,))
    out[..., 0] = v
    return out
