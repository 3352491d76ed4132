"""Shared checks for the parity tests."""

import numpy as np


def rel_err(got, ref):
    """max |got - ref| normalised by max |ref| (per-node errors relative to the field scale:
    near-zero entries make a per-entry relative error ill-conditioned)."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    scale = np.abs(ref).max()
    if scale == 0.0:
        return float(np.abs(got).max())
    return float(np.abs(got - ref).max() / scale)
