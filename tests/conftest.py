import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def _stab(d):
    import json
    return json.load(open(os.path.join(GOLDEN, d, "meta.json"))).get("stab", "none")


def golden_cases():
    """Cases without a stabilisation field (the plain residual path)."""
    return sorted(d for d in os.listdir(GOLDEN)
                  if os.path.exists(os.path.join(GOLDEN, d, "meta.json")) and _stab(d) == "none")


def stab_cases():
    """Cases whose solver had a stabilisation field computed by the reference's operators."""
    return sorted(d for d in os.listdir(GOLDEN)
                  if os.path.exists(os.path.join(GOLDEN, d, "meta.json")) and _stab(d) != "none")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
