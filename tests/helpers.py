"""Shared checks for the parity tests."""

import numpy as np


def rel_err(got, ref):
    """max |got - ref| / max |ref|, per equation (column) for [nodes, neq] fields, worst
    equation returned. Per-node relative errors are ill-conditioned where a residual crosses
    zero, and the Euler variables differ in scale by orders of magnitude (density vs energy),
    so each equation is normalised by its own largest value."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    if got.ndim == 1:
        got, ref = got[:, None], ref[:, None]
    worst = 0.0
    for e in range(ref.shape[1]):
        scale = np.abs(ref[:, e]).max()
        err = np.abs(got[:, e] - ref[:, e]).max()
        worst = max(worst, err / scale if scale > 0.0 else err)
    return float(worst)
