"""The C-ABI library loads and exports every symbol include/b2p.h declares (CPU only)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    src = (ROOT / "include" / "b2p.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(b2p_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("b2p_device_info", "b2p_ctx_create", "b2p_upload_lp", "b2p_solve", "b2p_spmv",
              "b2p_batch_upload", "b2p_batch_solve", "b2p_mlp_train_epoch"):
        assert s in syms


def test_library_exports_every_declared_symbol(b2p):
    lib = b2p.lib()
    for s in declared_symbols():
        assert hasattr(lib, s), f"libb2p.so does not export {s}"
    assert set(declared_symbols()) <= set(b2p.SIGNATURES), "ctypes mirror misses a declared symbol"


def test_params_defaults_mirror_reference_options(b2p):
    p = b2p.default_params()
    # FirstOrderSolverOptions defaults, include/bharatopt/first_order_solver.hpp:29-38
    assert p.max_iterations == 50000 and p.check_frequency == 100 and p.adaptive_step_size == 1
    assert p.feasibility_tolerance == 1e-7 and p.primal_step_size == 0.01 and p.dual_step_size == 0.01
    assert p.engine == 0 and p.eps_rel_kkt == 1e-6


def test_struct_layouts_match_header(b2p):
    # field counts of the C structs, so a header edit without a mirror edit fails here
    src = (ROOT / "include" / "b2p.h").read_text()
    for cname, py in (("b2p_params", b2p.Params), ("b2p_result", b2p.Result)):
        body = re.search(r"typedef struct \{([^}]*)\}\s*" + cname + ";", src).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        n = len([ln for ln in body.split(";") if ln.strip()])
        assert n == len(py._fields_), (cname, n, len(py._fields_))


@pytest.mark.skipif(Path("/dev/nvidia0").exists(), reason="a GPU is present")
def test_no_gpu_is_an_error_not_a_fallback(b2p):
    with pytest.raises(b2p.B2PError) as e:
        b2p.Context(0)
    assert e.value.code == b2p.GPU_UNAVAILABLE
