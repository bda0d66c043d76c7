"""ctypes mirror of the libb2p C ABI (include/b2p.h).

This is the Python face the tests and the benchmark use; the product
boundary itself is the C ABI and the C++ drop-in under dropin/.  There is no
CPU fallback anywhere in this module: without libb2p.so or without a usable
GPU every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import lpgen  # noqa: F401  (workload generators)
from . import warmstart  # noqa: F401  (learned warm start orchestration)

_HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("B2P_LIB", _HERE / "libb2p.so"))

OK, GPU_UNAVAILABLE, GPU_UNINITIALIZED, OUT_OF_MEMORY, INVALID_ARGUMENT, EXECUTION_FAILED, NO_LP, TIMEOUT, TOO_LARGE = range(9)
DOT_NOALLOC_MAX_N = 8388608
STATUS_NAMES = ["OPTIMAL", "MAX_ITERATIONS", "NUMERICAL_FAILURE", "INFEASIBLE_DETECTED", "UNBOUNDED_DETECTED",
                "INTERRUPTED"]
CALL_NAMES = ["OK", "GPU_UNAVAILABLE", "GPU_UNINITIALIZED", "OUT_OF_MEMORY", "INVALID_ARGUMENT", "EXECUTION_FAILED",
              "NO_LP", "TIMEOUT", "TOO_LARGE"]
ENGINES = {"reference": 0, "halpern": 1}
PRECISIONS = {"fp64": 0, "fp32": 1}


class DeviceInfo(C.Structure):
    _fields_ = [("is_available", C.c_int), ("device_name", C.c_char * 128), ("total_memory_bytes", C.c_size_t),
                ("free_memory_bytes", C.c_size_t), ("compute_capability_major", C.c_int),
                ("compute_capability_minor", C.c_int), ("multiprocessor_count", C.c_int),
                ("l2_cache_bytes", C.c_int), ("status_message", C.c_char * 256)]


class Timing(C.Structure):
    _fields_ = [("h2d_time_ms", C.c_double), ("kernel_time_ms", C.c_double), ("d2h_time_ms", C.c_double),
                ("sync_time_ms", C.c_double), ("total_gpu_time_ms", C.c_double)]


class Params(C.Structure):
    _fields_ = [("engine", C.c_int), ("precision", C.c_int), ("max_iterations", C.c_int64),
                ("feasibility_tolerance", C.c_double), ("primal_step_size", C.c_double),
                ("dual_step_size", C.c_double), ("adaptive_step_size", C.c_int), ("check_frequency", C.c_int64),
                ("eps_rel_kkt", C.c_double), ("check_every", C.c_int), ("ruiz_iterations", C.c_int),
                ("reflection", C.c_double), ("restart_sufficient", C.c_double), ("restart_necessary", C.c_double),
                ("restart_artificial", C.c_double), ("primal_weight", C.c_double), ("step_safety", C.c_double),
                ("refinement_rounds", C.c_int), ("time_limit_s", C.c_double),
                ("lanes_per_row", C.c_int), ("eps_objective", C.c_double), ("eps_infeasible", C.c_double)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int64), ("restarts", C.c_int64),
                ("primal_objective", C.c_double), ("dual_objective", C.c_double),
                ("rel_primal_residual", C.c_double), ("rel_dual_residual", C.c_double), ("rel_gap", C.c_double),
                ("rel_kkt", C.c_double), ("constraint_violation", C.c_double), ("bound_violation", C.c_double),
                ("max_primal_delta", C.c_double), ("max_dual_delta", C.c_double), ("used_average", C.c_int),
                ("refinement_rounds_done", C.c_int), ("primal_weight", C.c_double), ("step_size", C.c_double),
                ("solve_time_ms", C.c_double), ("kernel_time_ms", C.c_double), ("transfer_time_ms", C.c_double),
                ("kernel_launches", C.c_int64)]


_P = C.c_void_p
_I32P = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_I64P = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_F64P = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_F32P = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_U8P = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_U16P = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")

# name -> (restype, argtypes); every symbol declared in include/b2p.h
SIGNATURES = {
    "b2p_device_info": (C.c_int, [C.c_int, C.POINTER(DeviceInfo)]),
    "b2p_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "b2p_ctx_destroy": (C.c_int, [_P]),
    "b2p_last_error": (C.c_char_p, [_P]),
    "b2p_params_default": (None, [C.POINTER(Params)]),
    "b2p_ctx_set_stream": (C.c_int, [_P, _P]),
    "b2p_kernel_timing": (C.c_int, [_P, C.POINTER(Params), C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                    C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "b2p_spmv": (C.c_int, [_P, C.c_int, C.c_int, _I32P, _I32P, _F64P, _F64P, _F64P, C.POINTER(Timing)]),
    "b2p_spmv_t": (C.c_int, [_P, C.c_int, C.c_int, _I32P, _I32P, _F64P, _F64P, _F64P, C.POINTER(Timing)]),
    "b2p_vector_op": (C.c_int, [_P, C.c_int, C.c_size_t, C.c_double, _F64P, _P, _F64P, C.POINTER(Timing)]),
    "b2p_dot": (C.c_int, [_P, C.c_size_t, _F64P, _F64P, C.POINTER(C.c_double), C.POINTER(Timing)]),
    "b2p_norm2": (C.c_int, [_P, C.c_size_t, _F64P, C.POINTER(C.c_double), C.POINTER(Timing)]),
    "b2p_dot_noalloc": (C.c_int, [_P, _P, C.c_size_t, _P, _P]),
    "b2p_upload_lp": (C.c_int, [_P, C.c_int, C.c_int, C.c_int64, _I32P, _I32P, _F64P, _F64P, _F64P, _F64P, _F64P,
                                _U8P]),
    "b2p_solve": (C.c_int, [_P, C.POINTER(Params), _P, _P, C.POINTER(Result), _P, _P]),
    "b2p_batch_upload": (C.c_int, [_P, C.c_int, _I32P, _I32P, _I64P, _I32P, _I32P, _F64P, C.c_int, _I32P, _F64P,
                                   _F64P, _F64P, _F64P, _U8P]),
    "b2p_batch_solve": (C.c_int, [_P, C.POINTER(Params), _P, _P, _P, _P, _P, _P, _P, _P, _P, C.POINTER(Result)]),
    "b2p_batch_objectives": (C.c_int, [_P, _P, _P, _P]),
    "b2p_batch_trace": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int), _P, _P]),
    "b2p_mps_read": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    "b2p_mps_free": (None, [_P]),
    "b2p_mps_dims": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int64),
                               C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int),
                               C.POINTER(C.c_int64)]),
    "b2p_mps_model": (C.c_int, [_P, _I32P, _I32P, _F64P, C.c_char_p, _U8P, _F64P, _F64P, _F64P, _F64P, _F64P,
                                _U8P]),
    "b2p_mps_standard_form": (C.c_int, [_P, _I32P, _I32P, _F64P, _F64P, _F64P, _F64P, _F64P, _U8P]),
    "b2p_upload_mps": (C.c_int, [_P, _P]),
    "b2p_mlp_create": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_uint64]),
    "b2p_mlp_train_epoch": (C.c_int, [_P, _F32P, _F32P, C.c_int, C.c_int, C.c_float, C.POINTER(C.c_float)]),
    "b2p_mlp_infer": (C.c_int, [_P, _F32P, C.c_int, _F32P]),
    "b2p_mlp_get_params": (C.c_int, [_P, _F32P]),
    "b2p_mlp_set_params": (C.c_int, [_P, _F32P]),
    "b2p_mlp_gradient": (C.c_int, [_P, _F32P, _F32P, C.c_int, C.POINTER(C.c_float), _F32P]),
    "b2p_gemm_bf16": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, _U16P, C.c_int, _U16P, C.c_int, _F32P]),
    "b2p_mlp_dataset_from_batch": (C.c_int, [_P, _F32P, C.c_int]),
    "b2p_mlp_train": (C.c_int, [_P, C.c_int, C.c_int, C.c_float, C.c_float, C.c_uint64, C.POINTER(C.c_float)]),
    "b2p_mlp_get_normalization": (C.c_int, [_P, _F32P, _F32P, _F32P, _F32P]),
    "b2p_mlp_set_normalization": (C.c_int, [_P, _F32P, _F32P, _F32P, _F32P]),
    "b2p_batch_solve_learned": (C.c_int, [_P, C.POINTER(Params), _F32P, C.c_int, _P, _P, _P, _P, _P, _P,
                                          C.POINTER(Result)]),
}

_lib = None


def lib(path: Path | None = None):
    """Load libb2p.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path or LIB_PATH)
    if not p.exists():
        raise RuntimeError(f"libb2p.so not built at {p}; run `python __graft_entry__.py`")
    L = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


class B2PError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{CALL_NAMES[code] if 0 <= code < len(CALL_NAMES) else code}: {msg}")
        self.code = code


def device_info(device: int = 0) -> dict:
    info = DeviceInfo()
    st = lib().b2p_device_info(device, C.byref(info))
    return {"status": st, "is_available": bool(info.is_available), "name": info.device_name.decode(),
            "total_memory_bytes": info.total_memory_bytes, "free_memory_bytes": info.free_memory_bytes,
            "cc": (info.compute_capability_major, info.compute_capability_minor),
            "sm_count": info.multiprocessor_count, "l2_bytes": info.l2_cache_bytes,
            "message": info.status_message.decode()}


class MpsFile:
    """An MPS file read by the library (b2p_mps_read): its model as parsed, its
    standard form, and the handle b2p_upload_mps takes.  Host code only; needs no GPU."""

    def __init__(self, path):
        self._h = C.c_void_p()
        err = C.create_string_buffer(512)
        st = lib().b2p_mps_read(str(path).encode(), C.byref(self._h), err, 512)
        if st != OK:
            raise B2PError(st, err.value.decode())
        m, n, mx, sm = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        nnz, snnz = C.c_int64(), C.c_int64()
        off = C.c_double()
        lib().b2p_mps_dims(self._h, C.byref(m), C.byref(n), C.byref(nnz), C.byref(mx), C.byref(off), C.byref(sm),
                           C.byref(snnz))
        self.m, self.n, self.nnz, self.maximize, self.obj_offset = m.value, n.value, nnz.value, bool(mx.value), off.value
        self.std_m, self.std_nnz = sm.value, snnz.value

    def model(self) -> dict:
        """Rows as parsed: CSR (columns ascending), row type 'L' / 'G' / 'E', ranged flag, rhs
        (the lower end of a ranged row), range upper end; columns: cost, bounds, kind
        (0 continuous, 1 integer, 2 binary)."""
        m, n, z = self.m, self.n, self.nnz
        out = dict(rowptr=np.zeros(m + 1, np.int32), colidx=np.zeros(z, np.int32), vals=np.zeros(z),
                   row_type=C.create_string_buffer(m + 1), ranged=np.zeros(m, np.uint8), rhs=np.zeros(m),
                   range_upper=np.zeros(m), obj=np.zeros(n), lb=np.zeros(n), ub=np.zeros(n),
                   col_type=np.zeros(n, np.uint8))
        lib().b2p_mps_model(self._h, *[out[k] for k in ("rowptr", "colidx", "vals", "row_type", "ranged", "rhs",
                                                         "range_upper", "obj", "lb", "ub", "col_type")])
        out["row_type"] = out["row_type"].raw[:m].decode()
        return out

    def standard_form(self):
        """lpgen.StdLP of the file (ranged rows written as two <= rows)."""
        from .lpgen import StdLP
        m, n, z = self.std_m, self.n, self.std_nnz
        a = dict(rowptr=np.zeros(m + 1, np.int32), colidx=np.zeros(z, np.int32), vals=np.zeros(z), b=np.zeros(m),
                 c=np.zeros(n), lb=np.zeros(n), ub=np.zeros(n), is_eq=np.zeros(m, np.uint8))
        lib().b2p_mps_standard_form(self._h, *[a[k] for k in ("rowptr", "colidx", "vals", "b", "c", "lb", "ub",
                                                              "is_eq")])
        return StdLP(m, n, a["rowptr"], a["colidx"], a["vals"], a["b"], a["c"], a["lb"], a["ub"], a["is_eq"],
                     name="mps")

    def close(self):
        if self._h:
            lib().b2p_mps_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def default_params(**kw) -> Params:
    p = Params()
    lib().b2p_params_default(C.byref(p))
    for k, v in kw.items():
        if k == "engine":
            v = ENGINES[v] if isinstance(v, str) else v
        if k == "precision":
            v = PRECISIONS[v] if isinstance(v, str) else v
        if k == "eps":
            k = "eps_rel_kkt"
        setattr(p, k, v)
    return p


def _result_dict(r: Result) -> dict:
    d = {name: getattr(r, name) for name, _ in Result._fields_}
    d["status"] = STATUS_NAMES[r.status] if 0 <= r.status < len(STATUS_NAMES) else r.status
    return d


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Context:
    """One libb2p context (one CUDA stream, one uploaded LP, optional batch and MLP)."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        st = lib().b2p_ctx_create(device, C.byref(self._h))
        if st != OK:
            raise B2PError(st, device_info(device)["message"])

    def close(self):
        if self._h:
            lib().b2p_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != OK:
            raise B2PError(st, lib().b2p_last_error(self._h).decode())

    def set_stream(self, stream_handle):
        """Issue all work on an existing cudaStream_t (an int handle, e.g. torch's
        `torch.cuda.current_stream().cuda_stream`); None restores the context's own."""
        self._check(lib().b2p_ctx_set_stream(self._h, C.c_void_p(stream_handle) if stream_handle else None))

    def kernel_timing(self, reps=20, **params):
        p = default_params(**params)
        vals = [C.c_double() for _ in range(4)]
        self._check(lib().b2p_kernel_timing(self._h, C.byref(p), reps, *[C.byref(v) for v in vals]))
        return {"primal_ms": vals[0].value, "dual_ms": vals[1].value, "primal_bytes": vals[2].value,
                "dual_bytes": vals[3].value}

    # ---- GpuBackend primitives
    def spmv(self, m, n, rowptr, colidx, vals, x, transpose=False):
        out = np.zeros(n if transpose else m)
        t = Timing()
        f = lib().b2p_spmv_t if transpose else lib().b2p_spmv
        self._check(f(self._h, m, n, np.ascontiguousarray(rowptr, np.int32), np.ascontiguousarray(colidx, np.int32),
                      np.ascontiguousarray(vals, np.float64), np.ascontiguousarray(x, np.float64), out, C.byref(t)))
        return out, {k: getattr(t, k) for k, _ in Timing._fields_}

    def vector_op(self, op, a, b=None, alpha=0.0):
        codes = {"add": 0, "sub": 1, "scale": 2, "axpy": 3}
        a = np.ascontiguousarray(a, np.float64)
        out = np.zeros_like(a)
        bb = None if b is None else np.ascontiguousarray(b, np.float64)
        self._check(lib().b2p_vector_op(self._h, codes[op], a.size, alpha, a, _ptr(bb), out, None))
        return out

    def dot(self, a, b):
        r = C.c_double()
        self._check(lib().b2p_dot(self._h, len(a), np.ascontiguousarray(a, np.float64),
                                  np.ascontiguousarray(b, np.float64), C.byref(r), None))
        return r.value

    def norm2(self, a):
        r = C.c_double()
        self._check(lib().b2p_norm2(self._h, len(a), np.ascontiguousarray(a, np.float64), C.byref(r), None))
        return r.value

    # ---- single LP
    def upload(self, lp):
        """Upload a standard-form LP (lpgen.StdLP or any object with the same fields)."""
        self.m, self.n = int(lp.m), int(lp.n)
        self._check(lib().b2p_upload_lp(self._h, lp.m, lp.n, int(lp.rowptr[-1]),
                                        np.ascontiguousarray(lp.rowptr, np.int32),
                                        np.ascontiguousarray(lp.colidx, np.int32),
                                        np.ascontiguousarray(lp.vals, np.float64),
                                        np.ascontiguousarray(lp.b, np.float64),
                                        np.ascontiguousarray(lp.c, np.float64),
                                        np.ascontiguousarray(lp.lb, np.float64),
                                        np.ascontiguousarray(lp.ub, np.float64),
                                        np.ascontiguousarray(lp.is_eq, np.uint8)))

    def upload_mps(self, mps):
        """Upload the standard form of an MpsFile (b2p_upload_mps)."""
        self.m, self.n = int(mps.std_m), int(mps.n)
        self._check(lib().b2p_upload_mps(self._h, mps._h))

    def solve(self, x0=None, y0=None, **params):
        p = default_params(**params)
        r = Result()
        x = np.zeros(self.n)
        y = np.zeros(self.m)
        x0 = None if x0 is None else np.ascontiguousarray(x0, np.float64)
        y0 = None if y0 is None else np.ascontiguousarray(y0, np.float64)
        self._check(lib().b2p_solve(self._h, C.byref(p), _ptr(x0), _ptr(y0), C.byref(r), _ptr(x), _ptr(y)))
        return _result_dict(r), x, y

    # ---- batch
    def batch_upload(self, mats, inst_mat, b, c, lb, ub, is_eq):
        """mats: list of (m, n, rowptr, colidx, vals); per-instance vectors concatenated."""
        mm = np.array([q[0] for q in mats], np.int32)
        nn = np.array([q[1] for q in mats], np.int32)
        nnz = np.array([int(q[2][-1]) for q in mats], np.int64)
        off = np.zeros(len(mats) + 1, np.int64)
        off[1:] = np.cumsum(nnz)
        rowptr = np.concatenate([np.asarray(q[2], np.int32) for q in mats])
        colidx = np.concatenate([np.asarray(q[3], np.int32) for q in mats])
        vals = np.concatenate([np.asarray(q[4], np.float64) for q in mats])
        self.batch_m = mm[np.asarray(inst_mat)]
        self.batch_n = nn[np.asarray(inst_mat)]
        self._check(lib().b2p_batch_upload(self._h, len(mats), mm, nn, off, rowptr, colidx, vals, len(inst_mat),
                                           np.ascontiguousarray(inst_mat, np.int32),
                                           np.ascontiguousarray(b, np.float64), np.ascontiguousarray(c, np.float64),
                                           np.ascontiguousarray(lb, np.float64),
                                           np.ascontiguousarray(ub, np.float64),
                                           np.ascontiguousarray(is_eq, np.uint8)))

    def batch_solve(self, x0=None, y0=None, omega0=None, outputs=True, **params):
        """Solve every uploaded instance (b2p_batch_solve).  outputs=False skips the
        host copies of x and y (the answers stay on the device, e.g. as training labels)."""
        p = default_params(engine="halpern", **params)
        cnt = len(self.batch_m)
        st = np.zeros(cnt, np.int32)
        it = np.zeros(cnt, np.int64)
        kk = np.zeros(cnt)
        omo = np.zeros(cnt)
        x = np.zeros(int(self.batch_n.sum())) if outputs else None
        y = np.zeros(int(self.batch_m.sum())) if outputs else None
        r = Result()
        x0 = None if x0 is None else np.ascontiguousarray(x0, np.float64)
        y0 = None if y0 is None else np.ascontiguousarray(y0, np.float64)
        om = None if omega0 is None else np.ascontiguousarray(omega0, np.float64)
        self._check(lib().b2p_batch_solve(self._h, C.byref(p), _ptr(x0), _ptr(y0), _ptr(om), _ptr(st), _ptr(it),
                                          _ptr(kk), _ptr(omo), _ptr(x), _ptr(y), C.byref(r)))
        return _result_dict(r), {"status": st, "iterations": it, "rel_kkt": kk, "omega": omo}, x, y

    def batch_objectives(self):
        """Per-instance primal objective c.x, dual objective d(y) and FP64 bound on the
        relative objective error of the last batched solve (b2p_batch_objectives)."""
        cnt = len(self.batch_m)
        p, d, e = np.zeros(cnt), np.zeros(cnt), np.zeros(cnt)
        self._check(lib().b2p_batch_objectives(self._h, _ptr(p), _ptr(d), _ptr(e)))
        return {"pobj": p, "dobj": d, "obj_err": e}

    def batch_trace(self):
        """(t_ms, active) after every persistent-graph replay of the last batched solve."""
        n = C.c_int()
        self._check(lib().b2p_batch_trace(self._h, 0, C.byref(n), None, None))
        t = np.zeros(n.value)
        a = np.zeros(n.value, np.int32)
        self._check(lib().b2p_batch_trace(self._h, n.value, C.byref(n), _ptr(t), _ptr(a)))
        return t, a

    def batch_solve_learned(self, features, fallback=True, outputs=True, **params):
        """Learned warm start for every instance of the uploaded batch (see
        b2p_batch_solve_learned): MLP inference, warm-started solve, cold fallback."""
        params.setdefault("precision", "fp32")
        p = default_params(engine="halpern", **params)
        cnt = len(self.batch_m)
        F = np.ascontiguousarray(features, np.float32)
        st = np.zeros(cnt, np.int32)
        it = np.zeros(cnt, np.int64)
        kk = np.zeros(cnt)
        used = np.zeros(cnt, np.uint8)
        x = np.zeros(int(self.batch_n.sum())) if outputs else None
        y = np.zeros(int(self.batch_m.sum())) if outputs else None
        r = Result()
        self._check(lib().b2p_batch_solve_learned(self._h, C.byref(p), F, 1 if fallback else 0, _ptr(st), _ptr(it),
                                                  _ptr(kk), _ptr(used), _ptr(x), _ptr(y), C.byref(r)))
        summ = _result_dict(r)
        summ["fallbacks"] = r.refinement_rounds_done
        return summ, {"status": st, "iterations": it, "rel_kkt": kk, "warm_used": used}, x, y

    # ---- MLP
    def mlp_create(self, in_dim, hidden, out_dim, seed=0):
        self._check(lib().b2p_mlp_create(self._h, in_dim, hidden, out_dim, seed))
        self.mlp_out = out_dim
        self.mlp_dims = (in_dim, hidden, out_dim)

    def mlp_train_epoch(self, X, Y, batch=256, lr=1e-3):
        loss = C.c_float()
        X = np.ascontiguousarray(X, np.float32)
        Y = np.ascontiguousarray(Y, np.float32)
        self._check(lib().b2p_mlp_train_epoch(self._h, X, Y, X.shape[0], batch, lr, C.byref(loss)))
        return loss.value

    def mlp_dataset_from_batch(self, features):
        F = np.ascontiguousarray(features, np.float32)
        self._check(lib().b2p_mlp_dataset_from_batch(self._h, F, F.shape[0]))

    def mlp_train(self, epochs, batch=256, lr_start=1e-3, lr_end=1e-5, seed=0):
        loss = C.c_float()
        self._check(lib().b2p_mlp_train(self._h, epochs, batch, lr_start, lr_end, seed, C.byref(loss)))
        return loss.value

    def mlp_get_normalization(self):
        i, _, o = self.mlp_dims
        a, b, c, d = (np.zeros(i, np.float32), np.zeros(i, np.float32), np.zeros(o, np.float32),
                      np.zeros(o, np.float32))
        self._check(lib().b2p_mlp_get_normalization(self._h, a, b, c, d))
        return a, b, c, d

    def mlp_set_normalization(self, in_mean, in_std, out_mean, out_std):
        arr = [np.ascontiguousarray(v, np.float32) for v in (in_mean, in_std, out_mean, out_std)]
        self._check(lib().b2p_mlp_set_normalization(self._h, *arr))

    def mlp_infer(self, X):
        X = np.ascontiguousarray(X, np.float32)
        out = np.zeros((X.shape[0], self.mlp_out), np.float32)
        self._check(lib().b2p_mlp_infer(self._h, X, X.shape[0], out))
        return out

    def mlp_param_count(self):
        i, h, o = self.mlp_dims
        return h * i + h + h * h + h + o * h + o

    def mlp_get_params(self):
        out = np.zeros(self.mlp_param_count(), np.float32)
        self._check(lib().b2p_mlp_get_params(self._h, out))
        return out

    def mlp_set_params(self, flat):
        flat = np.ascontiguousarray(flat, np.float32)
        assert flat.size == self.mlp_param_count()
        self._check(lib().b2p_mlp_set_params(self._h, flat))

    def mlp_gradient(self, X, Y):
        X = np.ascontiguousarray(X, np.float32)
        Y = np.ascontiguousarray(Y, np.float32)
        g = np.zeros(self.mlp_param_count(), np.float32)
        loss = C.c_float()
        self._check(lib().b2p_mlp_gradient(self._h, X, Y, X.shape[0], C.byref(loss), g))
        return loss.value, g

    def gemm_bf16(self, A, B, trans_a=False, trans_b=False):
        """A, B given as uint16 bf16 bit patterns (row-major)."""
        M = A.shape[1] if trans_a else A.shape[0]
        K = A.shape[0] if trans_a else A.shape[1]
        N = B.shape[0] if trans_b else B.shape[1]
        out = np.zeros((M, N), np.float32)
        self._check(lib().b2p_gemm_bf16(self._h, M, N, K, np.ascontiguousarray(A, np.uint16), int(trans_a),
                                        np.ascontiguousarray(B, np.uint16), int(trans_b), out))
        return out
