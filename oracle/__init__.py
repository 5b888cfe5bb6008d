"""CPU oracle for the per-batch operators — TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
the checker / CPU baseline; the product never imports it.

``liboracle.so`` (oracle.c) holds the C restatements (stable ORDER BY,
nested-loop join, the timed query baselines); ``expr_eval`` evaluates
expression trees with numpy. Parity status: the reference ships no golden
vectors or known-answer tests; the oracle is pinned against the reference's
own GPU kernels run on the same inputs (``oracle/_ref``, built by
``oracle/Makefile`` from the reference sources) by ``tests/test_ref_pin_gpu.py``.

CSV scan (``csv_scan``, ``convert_batch``): pinned against the reference's own
reader, csv-parser plus std::stoi / std::stof / strptime
(``oracle/_ref/libcsvref.so`` from ``csv_ref_harness.cpp``), live in
``tests/test_csv_cpu.py`` and through the golden fixtures it wrote
(``tests/golden/csv_ref.npz``).

CSV writer (``csv_format``): snprintf / gmtime_r + strftime, the C library
routines behind the reference writer's std::to_chars and strftime, checked
against std::to_chars itself in ``tests/test_csv_cpu.py``.

GROUP BY (``group_by``): parity unpinned. The reference ignores GROUP BY and
the DuckDB it defers to is not available here, so this numpy restatement of
SQL semantics is checked only against a plain-Python restatement of the same
semantics (``tests/test_group_cpu.py``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SRC = os.path.join(HERE, "oracle.c")


def reference_sources() -> str | None:
    """The reference's source tree for the parity-pin builds, or None where it
    is absent (the GPU box uses the prebuilt oracle/_ref libraries). Taken from
    YQ_REFERENCE_SOURCES, else the read-only mount the build container
    provides; this recipe is the one place that names that mount."""
    for cand in (os.environ.get("YQ_REFERENCE_SOURCES"), "/root/reference"):
        if cand and os.path.isdir(os.path.join(cand, "src", "kernels")):
            return cand
    return None


def build() -> str:
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.check_call(["gcc", "-O3", "-march=x86-64-v2", "-shared", "-fPIC", "-pthread", "-o", LIB, SRC,
                               "-lm"])
    return LIB


class OrcCol(C.Structure):
    _fields_ = [("data", C.c_void_p), ("nulls", C.c_void_p), ("type", C.c_int), ("width", C.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        vp, u32, i32, u64 = C.c_void_p, C.c_uint32, C.c_int, C.c_uint64
        L.orc_sort_perm.argtypes = [i32, vp, vp, i32, u32, i32, i32, vp, i32, vp, vp, i32]
        L.orc_sort_perm.restype = i32
        L.orc_join_pairs.argtypes = [C.POINTER(OrcCol), C.POINTER(OrcCol), vp, i32, u32, u32, vp, vp, u64]
        L.orc_join_pairs.restype = u64
        L.orc_sales_query.argtypes = [vp, vp, vp, vp, i32, vp, u32, i32, C.POINTER(C.c_double),
                                      C.POINTER(C.c_int64), C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.orc_sales_query.restype = None
        L.orc_star_query.argtypes = [vp, vp, vp, vp, u32, vp, i32, i32, C.POINTER(C.c_double), C.POINTER(C.c_int64)]
        L.orc_star_query.restype = None
        L.orc_cross_lt.argtypes = [vp, u32, vp, u32, vp, vp, u64]
        L.orc_cross_lt.restype = u64
        L.orc_gather.argtypes = [vp, vp, i32, vp, u32]
        L.orc_gather.restype = None
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# yq_type codes (0..3 equal the reference's DataType)
INT32, FLOAT32, DATETIME, TEXT, INT64, FLOAT64, BOOL = range(7)


def type_of(a: np.ndarray) -> int:
    if a.ndim == 2:
        return TEXT
    return {np.dtype(np.int32): INT32, np.dtype(np.float32): FLOAT32, np.dtype(np.int64): INT64,
            np.dtype(np.float64): FLOAT64, np.dtype(np.uint8): BOOL}[a.dtype]


def sort_perm(key: np.ndarray, desc=False, nulls=None, nulls_first=False, segments=None, in_perm=None,
              threads=1, type_=None) -> np.ndarray:
    """Stable ORDER BY permutation of one key (row ids), per segment."""
    key = np.ascontiguousarray(key)
    n = key.shape[0]
    t = type_ if type_ is not None else type_of(key)
    width = key.shape[1] if key.ndim == 2 else key.dtype.itemsize
    out = np.empty(n, dtype=np.uint32)
    seg = None if segments is None else np.ascontiguousarray(np.asarray(segments, dtype=np.uint32))
    nl = None if nulls is None else np.ascontiguousarray(nulls.astype(np.uint8))
    ip = None if in_perm is None else np.ascontiguousarray(in_perm.astype(np.uint32))
    rc = lib().orc_sort_perm(t, _ptr(key), _ptr(nl), width, n, int(desc), int(nulls_first), _ptr(seg),
                             0 if seg is None else len(seg) - 1, _ptr(ip), _ptr(out), threads)
    assert rc == 0
    return out


def sort_perm_multi(keys: list, descs: list, nulls=None, nulls_first=None, threads=1) -> np.ndarray:
    """ORDER BY k0, k1, ...: stable sorts from the least significant key."""
    perm = None
    for i in range(len(keys) - 1, -1, -1):
        perm = sort_perm(keys[i], descs[i], None if nulls is None else nulls[i],
                         False if nulls_first is None else nulls_first[i], in_perm=perm, threads=threads)
    return perm


def join_pairs(lcols: list, rcols: list, conds: list, lnulls=None, rnulls=None, cap=None):
    """Inner join pairs (l, r) in (l, r) order; conds = [(lcol, rcol, cmp)]."""
    def mk(cols, nulls):
        arr = (OrcCol * len(cols))()
        keep = []
        for i, c in enumerate(cols):
            c = np.ascontiguousarray(c)
            keep.append(c)
            nl = None if nulls is None or nulls[i] is None else np.ascontiguousarray(nulls[i].astype(np.uint8))
            keep.append(nl)
            arr[i] = OrcCol(c.ctypes.data, None if nl is None else nl.ctypes.data, type_of(c),
                            c.shape[1] if c.ndim == 2 else c.dtype.itemsize)
        return arr, keep

    la, lk = mk(lcols, lnulls)
    ra, rk = mk(rcols, rnulls)
    L, R = lcols[0].shape[0], rcols[0].shape[0]
    cd = np.asarray([x for c in conds for x in c], dtype=np.int32)
    cap = cap if cap is not None else L * R
    ol = np.empty(max(1, cap), dtype=np.uint32)
    orr = np.empty(max(1, cap), dtype=np.uint32)
    n = lib().orc_join_pairs(la, ra, _ptr(cd), len(conds), L, R, _ptr(ol), _ptr(orr), cap)
    n = min(n, cap)
    return ol[:n], orr[:n]


def sales_query(t: dict, excluded: bytes, n: int | None = None, threads=1):
    n = len(t["price"]) if n is None else n
    ex = np.zeros(t["category"].shape[1], dtype=np.uint8)
    ex[: len(excluded)] = np.frombuffer(excluded, dtype=np.uint8)
    s, c, mn, mx = C.c_double(), C.c_int64(), C.c_float(), C.c_float()
    lib().orc_sales_query(_ptr(t["price"]), _ptr(t["qty"]), _ptr(t["discount"]), _ptr(t["category"]),
                          t["category"].shape[1], _ptr(ex), n, threads, C.byref(s), C.byref(c), C.byref(mn),
                          C.byref(mx))
    return s.value, c.value, mn.value, mx.value


def star_query(fact: dict, dim: dict, year: int, n: int | None = None, threads=1):
    n = len(fact["datekey"]) if n is None else n
    ok = np.zeros(len(dim["datekey"]), dtype=np.uint8)
    ok[dim["datekey"][dim["year"] == year]] = 1
    s, c = C.c_double(), C.c_int64()
    lib().orc_star_query(_ptr(fact["datekey"]), _ptr(fact["quantity"]), _ptr(fact["discount"]),
                         _ptr(fact["extendedprice"]), n, _ptr(ok), len(ok), threads, C.byref(s), C.byref(c))
    return s.value, c.value


def cross_lt(x: np.ndarray, y: np.ndarray, cap=None):
    cap = cap if cap is not None else len(x) * len(y)
    ox = np.empty(max(1, cap), dtype=np.int32)
    oy = np.empty(max(1, cap), dtype=np.int32)
    n = lib().orc_cross_lt(_ptr(x), len(x), _ptr(y), len(y), _ptr(ox), _ptr(oy), cap)
    return ox[: min(n, cap)], oy[: min(n, cap)], n


# ------------------------------------------------------------------ CSV scan
REF_CSV_LIB = os.path.join(HERE, "_ref", "libcsvref.so")
CSV_WIDTH = {0: 4, 1: 4, 2: 8}
CSV_DTYPE = {0: np.int32, 1: np.float32, 2: np.int64}


def _csv_outputs(types, width, cap):
    datas, nulls = [], []
    for t in types:
        if t < 0:
            datas.append(np.zeros(1, np.uint8))
            nulls.append(np.zeros(1, np.uint8))
            continue
        w = width if t == 3 else CSV_WIDTH[t]
        datas.append(np.zeros(cap * w + 1, np.uint8))
        nulls.append(np.zeros(cap + 1, np.uint8))
    return datas, nulls


def _csv_result(rows, bad, fr, ff, fk, types, width, datas, nulls):
    cols = []
    for t, d, n in zip(types, datas, nulls):
        if t < 0:
            cols.append(None)
            continue
        w = width if t == 3 else CSV_WIDTH[t]
        raw = d[: rows * w]
        vals = raw.reshape(rows, w).copy() if t == 3 else raw.view(CSV_DTYPE[t]).copy()
        cols.append((vals, n[:rows].copy()))
    return {"rows": rows, "bad": bad, "first_row": fr, "first_field": ff, "first_kind": fk, "cols": cols}


def csv_scan(body: bytes, types: list, width: int = 16) -> dict:
    """The oracle's CSV scan of `body` (text after the header line): rows kept,
    conversion failures, and per field (values, null bytes) or None when skipped."""
    L = lib()
    L.orc_csv_scan.restype = C.c_int64
    n = len(types)
    cap = body.count(b"\n") + body.count(b"\r") + 2
    datas, nulls = _csv_outputs(types, width, cap)
    dp = (C.c_void_p * n)(*[d.ctypes.data for d in datas])
    npp = (C.c_void_p * n)(*[x.ctypes.data for x in nulls])
    ty = (C.c_int * n)(*types)
    wd = (C.c_int * n)(*[width if t == 3 else 0 for t in types])
    bad, fr, ff, fk = C.c_uint64(), C.c_int64(), C.c_int(), C.c_int()
    rows = L.orc_csv_scan(C.c_char_p(body), C.c_uint64(len(body)), n, ty, wd, dp, npp, C.c_uint64(cap),
                          C.byref(bad), C.byref(fr), C.byref(ff), C.byref(fk))
    assert rows >= 0
    return _csv_result(rows, bad.value, fr.value, ff.value, fk.value, types, width, datas, nulls)


def ref_csv_available() -> bool:
    return os.path.exists(REF_CSV_LIB)


def ref_csv_scan(header: bytes, body: bytes, types: list, width: int = 16, guess: bool = False) -> dict:
    """The reference's own reader (csv-parser + std::stoi/stof + strptime), from
    oracle/_ref/libcsvref.so, on header + body written to a temporary file."""
    import tempfile
    L = C.CDLL(REF_CSV_LIB)
    n = len(types)
    cap = body.count(b"\n") + body.count(b"\r") + 2
    datas, nulls = _csv_outputs(types, width, cap)
    dp = (C.c_void_p * n)(*[d.ctypes.data for d in datas])
    npp = (C.c_void_p * n)(*[x.ctypes.data for x in nulls])
    ty = (C.c_int * n)(*types)
    wd = (C.c_int * n)(*[width if t == 3 else 0 for t in types])
    rows, bad, fr, ff, fk = C.c_uint64(), C.c_uint64(), C.c_int64(), C.c_int(), C.c_int()
    with tempfile.NamedTemporaryFile("wb", suffix=".csv", delete=False) as fh:
        fh.write(header + body)
        path = fh.name
    try:
        rc = L.ref_csv_scan(C.c_char_p(path.encode()), C.c_int(1 if guess else 0), n, ty, wd, dp, npp,
                            C.c_uint64(cap), C.byref(rows), C.byref(bad), C.byref(fr), C.byref(ff), C.byref(fk))
    finally:
        os.unlink(path)
    if rc != 0:
        raise RuntimeError(f"reference CSV reader returned {rc}")
    return _csv_result(rows.value, bad.value, fr.value, ff.value, fk.value, types, width, datas, nulls)


def convert_batch(kind: int, strings: list) -> tuple:
    """glibc conversions as the reference calls them: kind 0 std::stoi, 1 std::stof
    (float bits), 2 strptime+timegm. Returns (values int64, status int32)."""
    L = lib()
    buf = b"".join(strings)
    offs = np.zeros(len(strings) + 1, np.uint64)
    offs[1:] = np.cumsum([len(s) for s in strings])
    out = np.zeros(len(strings), np.int64)
    st = np.zeros(len(strings), np.int32)
    L.orc_convert_batch(C.c_int(kind), C.c_char_p(buf), offs.ctypes.data_as(C.c_void_p), C.c_uint64(len(strings)),
                        out.ctypes.data_as(C.c_void_p), st.ctypes.data_as(C.c_void_p))
    return out, st


def csv_format(cols: list, rows: int) -> bytes:
    """The reference writer's rows (CsvWriter::batchToCsv without the header)
    for columns given as (type, width, values ndarray, nulls ndarray or None);
    type 0 INT32, 1 FLOAT32, 2 DATETIME, 3 TEXT (values uint8 [rows, width]), 4 INT64."""
    L = lib()
    L.orc_csv_format.restype = C.c_uint64
    n = len(cols)
    keep = [np.ascontiguousarray(v) for _, _, v, _ in cols]
    nul = [None if x is None else np.ascontiguousarray(x, dtype=np.uint8) for _, _, _, x in cols]
    ty = (C.c_int * n)(*[c[0] for c in cols])
    wd = (C.c_int * n)(*[c[1] for c in cols])
    dp = (C.c_void_p * n)(*[k.ctypes.data for k in keep])
    npp = (C.c_void_p * n)(*[None if x is None else x.ctypes.data for x in nul])
    need = L.orc_csv_format(n, ty, wd, dp, npp, C.c_uint64(rows), None, C.c_uint64(0))
    buf = C.create_string_buffer(int(need) + 1)
    L.orc_csv_format(n, ty, wd, dp, npp, C.c_uint64(rows), buf, C.c_uint64(need))
    return buf.raw[: int(need)]


# ------------------------------------------------------------------ GROUP BY
def _ordered_f64(x: np.ndarray) -> np.ndarray:
    """Order-preserving int64 of doubles (NaN above +inf, -0.0 below +0.0)."""
    d = np.asarray(x, dtype=np.float64).copy()
    u = d.view(np.uint64).copy()
    u[np.isnan(d)] = np.uint64(0x7ff8000000000000)
    neg = (u >> np.uint64(63)) == 1
    u = np.where(neg, ~u, u | np.uint64(1 << 63))
    return (u ^ np.uint64(1 << 63)).view(np.int64)


def _unordered_f64(k: np.ndarray) -> np.ndarray:
    u = k.view(np.uint64) ^ np.uint64(1 << 63)
    pos = (u >> np.uint64(63)) == 1
    u = np.where(pos, u & ~np.uint64(1 << 63), ~u)
    return u.view(np.float64)


def group_by(key, key_nulls, key_type, aggs):
    """SQL GROUP BY (the device operator's semantics, numpy): groups in
    ascending key order (stable: a group's key is its first row's), the NULL
    group last, -0.0 equal to +0.0 and NaNs one group above +inf. aggs: list of
    (kind, values|None, nulls|None, type) with kind 0 COUNT(*), 1 COUNT, 2 SUM,
    3 AVG, 4 MIN, 5 MAX. Returns (key values, key nulls, [(values, nulls)])."""
    n = len(key)
    kn = np.zeros(n, bool) if key_nulls is None else np.asarray(key_nulls).astype(bool)
    # NULL keys are all equal: the NULL group keeps row order
    if key_type == 3:  # text: byte strings
        k = np.ascontiguousarray(key)
        sk = np.where(kn, b"", k.view(f"S{k.shape[1]}").ravel())
        order = np.lexsort((np.arange(n), sk, kn))
        sorted_k = sk[order]
        eq = sorted_k[1:] == sorted_k[:-1]
    elif key_type in (1, 5):
        kf = np.asarray(key, dtype=np.float64)
        canon = np.where(kf == 0, 0.0, kf)
        nanm = np.isnan(canon)
        sortable = np.where(kn, 0.0, np.where(nanm, np.inf, canon))
        order = np.lexsort((np.arange(n), np.where(kn, False, nanm), sortable, kn))
        c, nm = canon[order], nanm[order]
        eq = (c[1:] == c[:-1]) | (nm[1:] & nm[:-1])
    else:
        kv = np.where(kn, 0, np.asarray(key).astype(np.int64))
        order = np.lexsort((np.arange(n), kv, kn))
        s = kv[order]
        eq = s[1:] == s[:-1]
    skn = kn[order]
    same = eq & (skn[1:] == skn[:-1])
    same = np.where(skn[1:] & skn[:-1], True, same)
    head = np.concatenate([[True], ~same]) if n else np.zeros(0, bool)
    starts = np.flatnonzero(head)
    out_key = np.asarray(key)[order[starts]]
    out_kn = kn[order[starts]]
    res = []
    for kind, vals, nulls, typ in aggs:
        if kind == 0:
            res.append((np.diff(np.concatenate([starts, [n]])).astype(np.int64), None))
            continue
        vn = np.zeros(n, bool) if nulls is None else np.asarray(nulls).astype(bool)
        ok = ~vn[order]
        cnt = np.add.reduceat(ok.astype(np.int64), starts) if n else np.zeros(0, np.int64)
        if kind == 1:
            res.append((cnt, None))
            continue
        v = np.asarray(vals)[order]
        isf = typ in (1, 5)
        if kind in (2, 3):
            if isf:
                s = np.add.reduceat(np.where(ok, v.astype(np.float64), 0.0), starts)
            else:
                s = np.add.reduceat(np.where(ok, v.astype(np.int64), 0), starts)
            if kind == 3:
                with np.errstate(invalid="ignore", divide="ignore"):
                    s = s.astype(np.float64) / cnt
            res.append((np.where(cnt > 0, s, 0), cnt == 0))
            continue
        enc = _ordered_f64(v) if isf else v.astype(np.int64)
        fill = np.iinfo(np.int64).max if kind == 4 else np.iinfo(np.int64).min
        enc = np.where(ok, enc, fill)
        red = (np.minimum if kind == 4 else np.maximum).reduceat(enc, starts)
        if isf:
            outv = _unordered_f64(red).astype(np.float32 if typ == 1 else np.float64)
        else:
            outv = red.astype({0: np.int32, 4: np.int64, 2: np.int64}[typ])
        res.append((np.where(cnt > 0, outv, 0).astype(outv.dtype), cnt == 0))
    return out_key, out_kn, res
