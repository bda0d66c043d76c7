"""Shared fixtures.  `-m "not gpu"` runs on any CPU box; `-m gpu` needs a B200."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "tests" / "golden"))

import __graft_entry__ as graft  # noqa: E402

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a) device")


@pytest.fixture(scope="session")
def b2p():
    return graft.load_package()


@pytest.fixture(scope="session")
def lpgen(b2p):
    return b2p.lpgen


@pytest.fixture(scope="session")
def oracle():
    from oracle_lib import OracleLib
    return OracleLib()


@pytest.fixture(scope="session")
def reflib():
    from oracle_lib import RefLib, REF_DIR
    if not (REF_DIR / "libbharatopt_ref.so").exists():
        pytest.skip("compiled reference (oracle/_ref/libbharatopt_ref.so) not present")
    return RefLib()


@pytest.fixture(scope="session")
def golden():
    npz = np.load(GOLDEN / "ref_traces.npz")
    meta = json.loads((GOLDEN / "ref_traces.json").read_text())
    highs = json.loads((GOLDEN / "highs_objectives.json").read_text())
    return {"arrays": npz, "meta": meta, "highs": highs}


@pytest.fixture(scope="session")
def ctx(b2p):
    c = b2p.Context(0)
    yield c
    c.close()


class _Std:
    """Standard-form LP view over golden arrays."""

    def __init__(self, arrays, key):
        for f in ("rowptr", "colidx", "vals", "b", "c", "lb", "ub", "is_eq"):
            setattr(self, f, np.ascontiguousarray(arrays[f"{key}/sf_{f}"]))
        self.m = len(self.b)
        self.n = len(self.c)
        self.name = key


@pytest.fixture(scope="session")
def golden_std(golden):
    return lambda key: _Std(golden["arrays"], key)
