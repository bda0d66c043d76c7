"""MPS ingest (b2p_mps_read / b2p_upload_mps): the reader against the reference's
MpsParser (src/mps_parser.cpp:140-531), the standard form it produces, and
solves of MPS files on the GPU.

CPU: every MPS fixture of the reference tree is parsed by both readers and the
models must agree field for field (row kinds, right-hand sides, ranges, costs,
bounds, variable kinds, coefficients); files the reference rejects must be
rejected too.  Synthetic files written here pin the standard form (G rows
negated, ranged rows as two <= rows) and the error messages.
GPU: synthetic LPs written as MPS, read and uploaded by the library, solved by
the Halpern engine; objectives against scipy-HiGHS on the same LP.
"""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.optimize import linprog

from oracle_lib import REF_DIR, REF_TREE

import pdlp_oracle


def write_mps(path, name, rows, cols, obj, rhs=None, ranges=None, bounds=None, maximize=False, obj_rhs=None,
              integer=()):
    """Free-format MPS.  rows: [(name, 'L'|'G'|'E')]; cols: {col: {row: value}} in order;
    obj: {col: cost}; rhs / ranges: {row: value}; bounds: [(type, col, value)]."""
    out = [f"NAME {name}"]
    if maximize:
        out += ["OBJSENSE", "    MAX"]
    out += ["ROWS", " N obj"] + [f" {t} {r}" for r, t in rows]
    out.append("COLUMNS")
    in_int = False
    for c, ent in cols.items():
        if (c in integer) != in_int:
            out.append(f"    M{len(out)} 'MARKER' '{'INTORG' if not in_int else 'INTEND'}'")
            in_int = not in_int
        if c in obj:
            out.append(f"    {c} obj {float(obj[c])!r}")
        for r, v in ent.items():
            out.append(f"    {c} {r} {float(v)!r}")
    if in_int:
        out.append(f"    M{len(out)} 'MARKER' 'INTEND'")
    out.append("RHS")
    for r, v in (rhs or {}).items():
        out.append(f"    RHS {r} {float(v)!r}")
    if obj_rhs is not None:
        out.append(f"    RHS obj {float(obj_rhs)!r}")
    if ranges:
        out.append("RANGES")
        for r, v in ranges.items():
            out.append(f"    RNG {r} {float(v)!r}")
    if bounds:
        out.append("BOUNDS")
        for t, c, v in bounds:
            out.append(f" {t} BND {c}" + ("" if v is None else f" {float(v)!r}"))
    out.append("ENDATA")
    path.write_text("\n".join(out) + "\n")


def ref_fixtures():
    root = REF_TREE / "benchmarks"
    return sorted(root.rglob("*.mps")) if root.exists() else []


@pytest.mark.skipif(not ref_fixtures(), reason="reference tree (its MPS fixtures) not present")
def test_reader_matches_reference_parser_on_every_fixture(b2p):
    if not (REF_DIR / "libbharatopt_ref.so").exists():
        pytest.skip("compiled reference not present")
    from oracle_lib import RefLib
    ref = RefLib()
    checked = 0
    for f in ref_fixtures():
        try:
            r = ref.parse_mps(f)
        except ValueError:
            with pytest.raises(b2p.B2PError):
                b2p.MpsFile(f)
            continue
        mf = b2p.MpsFile(f)
        d = mf.model()
        assert (r["m"], r["n"], r["maximize"], r["obj_offset"]) == (mf.m, mf.n, int(mf.maximize), mf.obj_offset), f
        for k_ref, k in (("obj", "obj"), ("lb", "lb"), ("ub", "ub"), ("rhs", "rhs")):
            assert np.array_equal(r[k_ref], d[k]), (f, k)
        assert np.array_equal(r["vtype"], d["col_type"].astype(np.int32)), f
        sense = np.array([{"L": 0, "E": 1, "G": 2}[t] for t in d["row_type"]], np.int32)
        sense[d["ranged"] == 1] = 3
        assert np.array_equal(r["sense"], sense), f
        rng = r["sense"] == 3
        assert np.array_equal(r["range_upper"][rng], d["range_upper"][rng]), f
        for i in range(r["m"]):
            a, b = slice(r["rowptr"][i], r["rowptr"][i + 1]), slice(d["rowptr"][i], d["rowptr"][i + 1])
            assert sorted(zip(r["colidx"][a], r["vals"][a])) == list(zip(d["colidx"][b], d["vals"][b])), (f, i)
        checked += 1
    assert checked >= 40


def test_standard_form_of_ranged_and_ge_rows(b2p, tmp_path):
    p = tmp_path / "ranged.mps"
    write_mps(p, "ranged", rows=[("r1", "L"), ("r2", "G"), ("r3", "E"), ("r4", "E"), ("r5", "L")],
              cols={"x": {"r1": 1.0, "r2": 2.0, "r3": 1.0, "r5": 1.0}, "y": {"r1": 3.0, "r4": 1.0, "r5": -1.0}},
              obj={"x": 1.0, "y": -2.0}, rhs={"r1": 10.0, "r2": 4.0, "r3": 5.0, "r4": 7.0, "r5": 3.0},
              ranges={"r1": 4.0, "r3": -2.0, "r5": 0.0}, bounds=[("MI", "x", None), ("UP", "y", 9.0)],
              maximize=True, obj_rhs=2.5)
    mf = b2p.MpsFile(p)
    assert mf.maximize and mf.obj_offset == -2.5
    d = mf.model()
    assert d["row_type"] == "LGEEL" and list(d["ranged"]) == [1, 0, 1, 0, 1]
    # L with R = 4: [6, 10]; E with R = -2: [3, 5]; L with R = 0: [3, 3]
    assert list(d["rhs"]) == [6.0, 4.0, 3.0, 7.0, 3.0] and d["range_upper"][0] == 10.0 and d["range_upper"][2] == 5.0
    s = mf.standard_form()
    # r1 -> x+3y <= 10, -x-3y <= -6; r2 -> -2x <= -4; r3 -> x <= 5, -x <= -3; r4 -> y = 7; r5 -> x - y = 3
    assert s.m == 7 and list(s.b) == [10.0, -6.0, -4.0, 5.0, -3.0, 7.0, 3.0]
    assert list(s.is_eq) == [0, 0, 0, 0, 0, 1, 1]
    A = sp.csr_matrix((s.vals, s.colidx, s.rowptr), shape=(s.m, s.n)).toarray()
    assert np.array_equal(A, [[1, 3], [-1, -3], [-2, 0], [1, 0], [-1, 0], [0, 1], [1, -1]])
    assert list(s.c) == [-1.0, 2.0] and s.lb[0] == -np.inf and s.ub[1] == 9.0


@pytest.mark.parametrize("body, message", [
    ("NAME t\nROWS\n N obj\n L r\nCOLUMNS\n x r 1\n", "missing ENDATA"),
    ("NAME t\nROWS\n N obj\n Q r\nENDATA\n", "invalid row type"),
    ("NAME t\nROWS\n N obj\n L r\nCOLUMNS\n x r abc\nENDATA\n", "invalid coefficient"),
    ("NAME t\nROWS\n N obj\n L r\nCOLUMNS\n x r 1\nBOUNDS\n ZZ B x 1\nENDATA\n", "unknown bound type"),
    ("NAME t\nROWS\n N obj\n L r\nCOLUMNS\n M1 'MARKER' 'INTORG'\n x r 1\nENDATA\n", "unclosed integer marker"),
])
def test_reader_errors(b2p, tmp_path, body, message):
    p = tmp_path / "bad.mps"
    p.write_text(body)
    with pytest.raises(b2p.B2PError) as e:
        b2p.MpsFile(p)
    assert e.value.code == b2p.INVALID_ARGUMENT and message in str(e.value)


def _synthetic(lpgen, tmp_path, seed, maximize):
    """A random-sparse LP written as MPS with ranged, >= and = rows, a free and a
    negative-lower-bound column and an objective offset."""
    std = lpgen.random_sparse(m=80, n=240, nnz_per_col=3, seed=seed).standard()
    rng = np.random.default_rng(seed)
    A = sp.csr_matrix((std.vals, std.colidx, std.rowptr), shape=(std.m, std.n))
    x0 = rng.uniform(0.5, 1.5, std.n)
    act = A @ x0
    rows, rhs, ranges = [], {}, {}
    for i in range(std.m):
        kind = ["L", "G", "E", "R"][i % 4]
        name = f"r{i}"
        if kind == "L":
            rows.append((name, "L")); rhs[name] = act[i] + 1.0
        elif kind == "G":
            rows.append((name, "G")); rhs[name] = act[i] - 1.0
        elif kind == "E":
            rows.append((name, "E")); rhs[name] = act[i]
        else:
            rows.append((name, "L")); rhs[name] = act[i] + 0.5; ranges[name] = 2.0
    Ac = A.tocsc()
    cols = {f"x{j}": {f"r{Ac.indices[p]}": float(Ac.data[p]) for p in range(Ac.indptr[j], Ac.indptr[j + 1])}
            for j in range(std.n)}
    obj = {f"x{j}": float(rng.uniform(-1, 1)) for j in range(std.n)}
    bounds = [("UP", f"x{j}", 5.0) for j in range(std.n)]
    bounds += [("LO", "x3", -2.0), ("FR", "x7", None)]
    bounds = [b for b in bounds if not (b[1] == "x7" and b[0] == "UP")]
    path = tmp_path / f"syn{seed}.mps"
    write_mps(path, f"syn{seed}", rows, cols, obj, rhs=rhs, ranges=ranges, bounds=bounds, maximize=maximize,
              obj_rhs=1.25)
    return path


def _highs(std):
    A = sp.csr_matrix((std.vals, std.colidx, std.rowptr), shape=(std.m, std.n))
    eq = std.is_eq.astype(bool)
    r = linprog(std.c, A_ub=A[~eq], b_ub=std.b[~eq], A_eq=A[eq] if eq.any() else None,
                b_eq=std.b[eq] if eq.any() else None,
                bounds=[(None if np.isinf(l) else l, None if np.isinf(u) else u) for l, u in zip(std.lb, std.ub)],
                method="highs")
    assert r.status == 0, r.message
    return float(r.fun)


@pytest.mark.gpu
@pytest.mark.parametrize("seed, maximize, precision", [(31, False, "fp64"), (32, True, "fp32")])
def test_mps_ingest_solve_matches_highs(ctx, b2p, lpgen, tmp_path, seed, maximize, precision):
    mf = b2p.MpsFile(_synthetic(lpgen, tmp_path, seed, maximize))
    std = mf.standard_form()
    z = _highs(std)
    ctx.upload_mps(mf)
    res, x, y = ctx.solve(engine="halpern", precision=precision, eps=1e-8, eps_objective=1e-8, max_iterations=400000)
    assert res["status"] == "OPTIMAL", res
    k = pdlp_oracle.kkt(std, x, y)
    assert k["rel_kkt"] <= 1.05e-8, k
    assert abs(k["pobj"] - z) <= 1e-7 * max(1.0, abs(z)), (k["pobj"], z)


@pytest.mark.gpu
def test_mps_ingest_certificates(ctx, b2p, tmp_path):
    """An infeasible and an unbounded MPS model, read and uploaded: the engine's
    certificates (the reference's edge_infeasible / edge_unbounded cases in spirit)."""
    p = tmp_path / "inf.mps"
    write_mps(p, "inf", rows=[("a", "L"), ("b", "G")], cols={"x": {"a": 1.0, "b": 1.0}, "y": {"a": 1.0, "b": 1.0}},
              obj={"x": 1.0, "y": 1.0}, rhs={"a": 1.0, "b": 3.0})
    ctx.upload_mps(b2p.MpsFile(p))
    res, _, _ = ctx.solve(engine="halpern", precision="fp64", eps=1e-6, max_iterations=200000)
    assert res["status"] == "INFEASIBLE_DETECTED", res
    p = tmp_path / "unb.mps"
    write_mps(p, "unb", rows=[("a", "L")], cols={"x": {"a": 1.0}, "y": {"a": -1.0}}, obj={"x": -1.0, "y": -1.0},
              rhs={"a": 4.0})
    ctx.upload_mps(b2p.MpsFile(p))
    res, _, _ = ctx.solve(engine="halpern", precision="fp64", eps=1e-6, max_iterations=200000)
    assert res["status"] == "UNBOUNDED_DETECTED", res
