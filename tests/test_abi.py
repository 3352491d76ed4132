"""The C-ABI library loads and exports every entry point include/rds_b200.h declares (CPU)."""

import ctypes
import os
import re

from conftest import ROOT
from pdekit_b200 import rds


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "rds_b200.h")).read()
    return sorted(set(re.findall(r"^RDS_API\s+[^(]*?\b(rds_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_abi():
    names = declared_symbols()
    assert "rds_create" in names and "rds_iterate" in names
    assert set(rds.EXPORTS) <= set(names)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(rds.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), f"{name} declared in include/rds_b200.h but not exported"


def test_version_string():
    assert b"sm_100a" in rds.lib().rds_version()


def test_invalid_descriptor_rejected_before_any_device_call():
    """rds_create validates the descriptor first (no GPU needed to see the error)."""
    import numpy as np

    L = rds.lib()
    coords = np.zeros((3, 2))
    for physics, dim, neq, scheme, nnodes in [(9, 2, 1, 0, 3), (1, 3, 1, 0, 3), (2, 2, 1, 0, 3),
                                              (1, 2, 1, 7, 3), (1, 2, 1, 0, 0)]:
        d = rds._Desc()
        d.physics, d.dim, d.neq, d.scheme, d.precision = physics, dim, neq, scheme, 0
        d.nnodes, d.ngeo_nodes, d.geo_coords = nnodes, 3, coords.ctypes.data_as(ctypes.c_void_p)
        ctx = ctypes.c_void_p()
        assert L.rds_create(ctypes.byref(ctx), ctypes.byref(d), None) == 1  # RDS_ERR_INVALID
        assert b"invalid descriptor" in L.rds_last_error(ctx)
        L.rds_destroy(ctx)
    assert L.rds_create(None, None, None) == 1


def test_steppers_reject_missing_context():
    """The stepping entry points check their context before touching the device."""
    L = rds.lib()
    assert L.rds_advance_rk3tvd(None, 0.5, 1) == 1  # RDS_ERR_INVALID
    assert L.rds_run(None, 0.5, 1) == 1
