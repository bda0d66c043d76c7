"""ORACLE -- test infrastructure only.

ctypes access to
  * oracle/_ref/liboracle.so       -- pdhg_oracle.c, the C restatement of the reference PDHG loop
  * oracle/_ref/libbharatopt_ref.so -- the reference's own sources compiled in place + ref_shim.cpp
Neither is ever loaded by the product path.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
# the reference source tree (its MPS fixtures are read by the CPU tests when it is present)
REF_TREE = Path(os.environ.get("B2P_REFERENCE_TREE", "/root/reference"))

_F64P = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_I32P = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_U8P = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")

REF_STATUS = ["OPTIMAL", "MAX_ITERATIONS", "NUMERICAL_FAILURE", "INFEASIBLE_DETECTED", "UNBOUNDED_DETECTED",
              "INTERRUPTED"]


class OracleRefResult(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_long), ("constraint_violation", C.c_double),
                ("bound_violation", C.c_double), ("max_primal_delta", C.c_double), ("max_dual_delta", C.c_double),
                ("used_average", C.c_int)]


class RefLP(C.Structure):
    _fields_ = [("m", C.c_int), ("n", C.c_int), ("rowptr", C.c_void_p), ("colidx", C.c_void_p),
                ("vals", C.c_void_p), ("sense", C.c_void_p), ("rhs", C.c_void_p), ("range_upper", C.c_void_p),
                ("obj", C.c_void_p), ("lb", C.c_void_p), ("ub", C.c_void_p), ("maximize", C.c_int),
                ("obj_offset", C.c_double)]


class RefFOResult(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_long), ("objective", C.c_double),
                ("constraint_violation", C.c_double), ("bound_violation", C.c_double),
                ("solve_time_ms", C.c_double), ("n_primal", C.c_long), ("n_dual", C.c_long)]


class RefVerifyResult(C.Structure):
    _fields_ = [("verified", C.c_int), ("objective_recomputed", C.c_double),
                ("max_constraint_violation", C.c_double), ("max_lower_bound_violation", C.c_double),
                ("max_upper_bound_violation", C.c_double), ("violated_constraints", C.c_long),
                ("violated_bounds", C.c_long)]


class OracleLib:
    """The C restatement (always built from repo sources)."""

    def __init__(self, path: Path | None = None):
        p = path or REF_DIR / "liboracle.so"
        if not Path(p).exists():
            raise RuntimeError(f"oracle not built: {p} (run `make -C oracle port`)")
        self.L = C.CDLL(str(p))
        self.L.oracle_ref_pdhg.restype = C.c_int
        self.L.oracle_ref_pdhg.argtypes = [C.c_int, C.c_int, _I32P, _I32P, _F64P, _F64P, _F64P, _F64P, _F64P, _U8P,
                                           C.c_long, C.c_long, C.c_double, C.c_int, C.c_double, C.c_double,
                                           _F64P, _F64P, _F64P, _F64P, C.POINTER(OracleRefResult)]
        self.L.oracle_spmv.argtypes = [C.c_int, _I32P, _I32P, _F64P, _F64P, _F64P]
        self.L.oracle_spmv_t.argtypes = [C.c_int, C.c_int, _I32P, _I32P, _F64P, _F64P, _F64P]

    def ref_pdhg(self, lp, max_iterations=50000, check_frequency=100, feas_tol=1e-7, adaptive=True,
                 primal_step=0.01, dual_step=0.01):
        n, m = lp.n, lp.m
        xf, xl, xs = np.zeros(n), np.zeros(n), np.zeros(n)
        yl = np.zeros(m)
        r = OracleRefResult()
        self.L.oracle_ref_pdhg(m, n, np.ascontiguousarray(lp.rowptr, np.int32),
                               np.ascontiguousarray(lp.colidx, np.int32), np.ascontiguousarray(lp.vals, np.float64),
                               np.ascontiguousarray(lp.b, np.float64), np.ascontiguousarray(lp.c, np.float64),
                               np.ascontiguousarray(lp.lb, np.float64), np.ascontiguousarray(lp.ub, np.float64),
                               np.ascontiguousarray(lp.is_eq, np.uint8), max_iterations, check_frequency, feas_tol,
                               int(adaptive), primal_step, dual_step, xf, xl, yl, xs, C.byref(r))
        return {"status": REF_STATUS[r.status], "iterations": r.iterations,
                "constraint_violation": r.constraint_violation, "bound_violation": r.bound_violation,
                "max_primal_delta": r.max_primal_delta, "max_dual_delta": r.max_dual_delta,
                "used_average": r.used_average, "x_final": xf, "x_last": xl, "y_last": yl, "x_sum": xs}

    def spmv(self, lp, x):
        y = np.zeros(lp.m)
        self.L.oracle_spmv(lp.m, lp.rowptr, lp.colidx, lp.vals, np.ascontiguousarray(x, np.float64), y)
        return y

    def spmv_t(self, lp, y):
        w = np.zeros(lp.n)
        self.L.oracle_spmv_t(lp.m, lp.n, lp.rowptr, lp.colidx, lp.vals, np.ascontiguousarray(y, np.float64), w)
        return w


class RefLib:
    """The reference's own code (compiled in place from its sources)."""

    def __init__(self, path: Path | None = None):
        p = path or REF_DIR / "libbharatopt_ref.so"
        if not Path(p).exists():
            raise RuntimeError(f"reference not built: {p} (run `make -C oracle ref`)")
        L = C.CDLL(str(p))
        L.ref_fo_solve.restype = C.c_int
        L.ref_fo_solve.argtypes = [C.POINTER(RefLP), C.c_long, C.c_long, C.c_double, C.c_int, C.c_double, C.c_double,
                                   C.POINTER(RefFOResult), _F64P, C.c_long, _F64P, C.c_long]
        L.ref_sf_create.restype = C.c_void_p
        L.ref_sf_create.argtypes = [C.POINTER(RefLP)]
        L.ref_sf_dims.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 4
        L.ref_sf_copy.argtypes = [C.c_void_p, _I32P, _I32P, _F64P, _F64P, _F64P, _F64P, _F64P, _U8P]
        L.ref_sf_recover.restype = C.c_double
        L.ref_sf_recover.argtypes = [C.c_void_p, _F64P, C.c_long, _F64P]
        L.ref_sf_free.argtypes = [C.c_void_p]
        L.ref_spmv.argtypes = [C.c_int, C.c_int, _I32P, _I32P, _F64P, _F64P, _F64P]
        L.ref_spmv_t.argtypes = [C.c_int, C.c_int, _I32P, _I32P, _F64P, _F64P, _F64P]
        L.ref_verify.argtypes = [C.POINTER(RefLP), _F64P, C.c_double, C.c_double, C.c_int,
                                 C.POINTER(RefVerifyResult)]
        L.ref_mps_parse.restype = C.c_void_p
        L.ref_mps_parse.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
        L.ref_mps_dims.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 4 + [C.POINTER(C.c_double)]
        L.ref_mps_copy.argtypes = [C.c_void_p, _I32P, _I32P, _F64P, _I32P, _F64P, _F64P, _F64P, _F64P, _F64P, _I32P]
        L.ref_mps_free.argtypes = [C.c_void_p]
        self.L = L

    @staticmethod
    def _reflp(lp, keep):
        """Row-form lpgen.LP -> RefLP (arrays kept alive in `keep`)."""
        arrs = dict(rowptr=np.ascontiguousarray(lp.rowptr, np.int32), colidx=np.ascontiguousarray(lp.colidx, np.int32),
                    vals=np.ascontiguousarray(lp.vals, np.float64), sense=np.ascontiguousarray(lp.sense, np.int32),
                    rhs=np.ascontiguousarray(lp.rhs, np.float64), obj=np.ascontiguousarray(lp.obj, np.float64),
                    lb=np.ascontiguousarray(lp.lb, np.float64), ub=np.ascontiguousarray(lp.ub, np.float64))
        keep.append(arrs)
        r = RefLP()
        r.m, r.n = lp.m, lp.n
        for k, a in arrs.items():
            setattr(r, k, a.ctypes.data)
        r.range_upper = None
        r.maximize = int(lp.maximize)
        r.obj_offset = 0.0
        return r

    def fo_solve(self, lp, max_iterations=50000, check_frequency=100, feas_tol=1e-7, adaptive=True,
                 primal_step=0.01, dual_step=0.01):
        keep = []
        r = self._reflp(lp, keep)
        out = RefFOResult()
        x = np.zeros(lp.n)
        y = np.zeros(max(lp.m, 1))
        self.L.ref_fo_solve(C.byref(r), max_iterations, check_frequency, feas_tol, int(adaptive), primal_step,
                            dual_step, C.byref(out), x, lp.n, y, y.size)
        return {"status": REF_STATUS[out.status], "iterations": out.iterations, "objective": out.objective,
                "constraint_violation": out.constraint_violation, "bound_violation": out.bound_violation,
                "solve_time_ms": out.solve_time_ms, "x": x[:out.n_primal], "y": y[:out.n_dual]}

    def standard_form(self, lp):
        """Presolve + standard form exactly as CPUFirstOrderSolver::solve builds it."""
        keep = []
        r = self._reflp(lp, keep)
        h = self.L.ref_sf_create(C.byref(r))
        st, m, n, nnz = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        self.L.ref_sf_dims(h, C.byref(st), C.byref(m), C.byref(n), C.byref(nnz))
        out = {"status": st.value, "m": m.value, "n": n.value, "handle": h, "orig_n": lp.n}
        if st.value == 0:
            rp = np.zeros(m.value + 1, np.int32)
            ci = np.zeros(nnz.value, np.int32)
            va = np.zeros(nnz.value)
            b = np.zeros(m.value)
            c = np.zeros(n.value)
            lo = np.zeros(n.value)
            hi = np.zeros(n.value)
            eq = np.zeros(m.value, np.uint8)
            self.L.ref_sf_copy(h, rp, ci, va, b, c, lo, hi, eq)
            out.update(rowptr=rp, colidx=ci, vals=va, b=b, c=c, lb=lo, ub=hi, is_eq=eq)
        return out

    def recover(self, sf, x_red):
        x = np.zeros(self._orig_n(sf))
        obj = self.L.ref_sf_recover(sf["handle"], np.ascontiguousarray(x_red, np.float64), len(x_red), x)
        return x, obj

    def _orig_n(self, sf):
        return sf["orig_n"]

    def free(self, sf):
        self.L.ref_sf_free(sf["handle"])

    def spmv(self, m, n, rowptr, colidx, vals, x):
        y = np.zeros(m)
        st = self.L.ref_spmv(m, n, rowptr, colidx, vals, np.ascontiguousarray(x, np.float64), y)
        if st:
            raise ValueError("reference CSRMatrix rejected the matrix")
        return y

    def spmv_t(self, m, n, rowptr, colidx, vals, y):
        w = np.zeros(n)
        st = self.L.ref_spmv_t(m, n, rowptr, colidx, vals, np.ascontiguousarray(y, np.float64), w)
        if st:
            raise ValueError("reference CSRMatrix rejected the matrix")
        return w

    def verify(self, lp, x, feas_tol=1e-7, reported_obj=None):
        keep = []
        r = self._reflp(lp, keep)
        out = RefVerifyResult()
        self.L.ref_verify(C.byref(r), np.ascontiguousarray(x, np.float64), feas_tol,
                          0.0 if reported_obj is None else reported_obj, int(reported_obj is not None),
                          C.byref(out))
        return {k: getattr(out, k) for k, _ in RefVerifyResult._fields_}

    def parse_mps(self, path):
        """The reference MpsParser's LPModel of an MPS file, as arrays (rows in CSR with each
        row's terms in the model's order; sense 0 <=, 1 =, 2 >=, 3 ranged)."""
        err = C.create_string_buffer(512)
        h = self.L.ref_mps_parse(str(path).encode(), err, 512)
        if not h:
            raise ValueError(err.value.decode())
        m, n, nnz, mx, off = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_double()
        self.L.ref_mps_dims(h, C.byref(m), C.byref(n), C.byref(nnz), C.byref(mx), C.byref(off))
        out = dict(rowptr=np.zeros(m.value + 1, np.int32), colidx=np.zeros(nnz.value, np.int32),
                   vals=np.zeros(nnz.value), sense=np.zeros(m.value, np.int32), rhs=np.zeros(m.value),
                   range_upper=np.zeros(m.value), obj=np.zeros(n.value), lb=np.zeros(n.value), ub=np.zeros(n.value),
                   vtype=np.zeros(n.value, np.int32))
        self.L.ref_mps_copy(h, *[out[k] for k in ("rowptr", "colidx", "vals", "sense", "rhs", "range_upper", "obj",
                                                   "lb", "ub", "vtype")])
        self.L.ref_mps_free(h)
        out.update(m=m.value, n=n.value, maximize=mx.value, obj_offset=off.value)
        return out

