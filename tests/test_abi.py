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
