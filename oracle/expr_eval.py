"""numpy evaluation of expression trees — TEST INFRASTRUCTURE ONLY (oracle).

Independent restatement of the semantics the fused kernels implement, node by
node after the reference's expression classes:

- BoundRef / BoundValue (bound_ref.hpp:16-43, bound_value.hpp:14-60)
- Cast (cast.hpp:23-90): numeric casts; float -> int rounds half to even and
  yields NULL when out of range (DuckDB); the reference truncates (static_cast).
- BoundFunc (bound_func.hpp:45-167, binary_operators_kernel.hpp:23-53):
  typed + - * / %; integer / and % by zero give NULL (DuckDB; the reference
  gives 0); int32 arithmetic wraps.
- Comparison (filters/comparison.hpp:51-215): typed; text compares unsigned
  bytes of the NUL-padded slot (strcmp_device, string_kernel.hpp:48-57).
- Conjunction (filters/conjunction.hpp:76-113): SQL three-valued AND / OR.
- Aggregates (aggregate.hpp:55-284): NULL inputs skipped; SUM/AVG of floats
  in FP64; COUNT(*) counts selected rows.

A value is a pair (values ndarray, valid bool ndarray).
"""
from __future__ import annotations

import numpy as np

from yallasql_b200 import _abi as A
from yallasql_b200.expr import (Aggregate, And, Arith, Cast, ColumnRef, Compare, Constant, IsNull, Not, Or,
                                parse_datetime)

NP = {A.INT32: np.int32, A.FLOAT32: np.float32, A.INT64: np.int64, A.DATETIME: np.int64, A.FLOAT64: np.float64,
      A.BOOL: np.bool_}


def _text_slot(v, width):
    b = v.encode() if isinstance(v, str) else bytes(v)
    out = np.zeros(width, dtype=np.uint8)
    out[: len(b)] = np.frombuffer(b[:width], dtype=np.uint8)
    return out


def _text_cmp(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Row-wise sign of memcmp over zero-padded slots (a, b: [n, w] or [w])."""
    w = max(a.shape[-1], b.shape[-1])
    pa = np.zeros(a.shape[:-1] + (w,), np.uint8); pa[..., : a.shape[-1]] = a
    pb = np.zeros(b.shape[:-1] + (w,), np.uint8); pb[..., : b.shape[-1]] = b
    pa, pb = np.broadcast_arrays(pa.astype(np.int16), pb.astype(np.int16))
    diff = pa - pb
    nz = diff != 0
    first = np.where(nz.any(axis=-1), nz.argmax(axis=-1), 0)
    d = np.take_along_axis(diff, first[..., None], axis=-1)[..., 0]
    return np.sign(d).astype(np.int8)


def _cmp(op, a, b):
    return {A.LT: a < b, A.LE: a <= b, A.GT: a > b, A.GE: a >= b, A.EQ: a == b, A.NE: a != b}[op]


def _cast(v, valid, frm, to):
    if frm == to or {frm, to} <= {A.INT64, A.DATETIME}:
        return v.astype(NP[to]), valid
    if to in (A.INT32, A.INT64, A.DATETIME) and frm in (A.FLOAT32, A.FLOAT64):
        x = v.astype(np.float64)
        lo, hi = (-2.0 ** 31, 2.0 ** 31) if to == A.INT32 else (-2.0 ** 63, 2.0 ** 63)
        ok = np.isfinite(x) & (x >= lo) & (x < hi)
        r = np.rint(np.where(ok, x, 0.0))
        if to == A.INT32:
            ok &= r <= 2 ** 31 - 1
        return r.astype(NP[to]), valid & ok
    if to == A.INT32 and frm in (A.INT64, A.DATETIME):
        ok = (v >= -2 ** 31) & (v <= 2 ** 31 - 1)
        return np.where(ok, v, 0).astype(np.int32), valid & ok
    if to == A.BOOL:
        return v != 0, valid
    return v.astype(NP[to]), valid


def _arith(op, t, a, b):
    with np.errstate(all="ignore"):
        if t in (A.FLOAT32, A.FLOAT64):
            f = {A.ADD: np.add, A.SUB: np.subtract, A.MUL: np.multiply, A.DIV: np.divide, A.MOD: np.fmod}[op]
            return f(a, b).astype(NP[t]), None
        a = a.astype(NP[t]); b = b.astype(NP[t])
        if op == A.ADD:
            return a + b, None
        if op == A.SUB:
            return a - b, None
        if op == A.MUL:
            return a * b, None
        zero = b == 0
        bs = np.where(zero, 1, b)
        if op == A.DIV:  # truncates toward zero (C semantics)
            a64, b64 = a.astype(np.int64), bs.astype(np.int64)
            q = np.abs(a64) // np.abs(b64) * np.sign(a64) * np.sign(b64)
            return np.where(b64 == -1, -a64, q).astype(NP[t]), ~zero
        r = np.where(bs == -1, 0, np.fmod(a, bs))
        return r.astype(NP[t]), ~zero


def evaluate(e, cols: dict, n: int):
    """cols: index -> (values ndarray, nulls ndarray|None, type)."""
    if isinstance(e, ColumnRef):
        v, nl, t = cols[e.index]
        valid = np.ones(n, bool) if nl is None else ~(nl.astype(bool))
        if t != e.type and t != A.TEXT:
            return _cast(v, valid, t, e.type)
        return v, valid
    if isinstance(e, Constant):
        if e.value is None:
            return np.zeros(n, NP.get(e.type, np.int64)), np.zeros(n, bool)
        if e.type == A.TEXT:
            return e.value, np.ones(n, bool)
        if e.type == A.DATETIME and isinstance(e.value, str):
            return np.full(n, parse_datetime(e.value), np.int64), np.ones(n, bool)
        return np.full(n, e.value, NP[e.type]), np.ones(n, bool)
    if isinstance(e, Cast):
        v, ok = evaluate(e.child, cols, n)
        return _cast(v, ok, e.child.type, e.to)
    if isinstance(e, Arith):
        a, va = evaluate(e.lhs, cols, n)
        b, vb = evaluate(e.rhs, cols, n)
        r, ok = _arith(e.op, e.lhs.type, a, b)
        valid = va & vb
        if ok is not None:
            valid &= ok
        return r, valid
    if isinstance(e, Compare):
        lhs, rhs = e.lhs, e.rhs
        if lhs.type == A.TEXT or rhs.type == A.TEXT:
            a, va = evaluate(lhs, cols, n)
            b, vb = evaluate(rhs, cols, n)
            w = cols[lhs.index][0].shape[1] if isinstance(lhs, ColumnRef) else 16
            if isinstance(a, (str, bytes)):
                a = _text_slot(a, w)
            if isinstance(b, (str, bytes)):
                b = _text_slot(b, max(w, len(b) + 1))
            s = _text_cmp(a, b)
            return _cmp(e.op, s, 0), va & vb
        a, va = evaluate(lhs, cols, n)
        b, vb = evaluate(rhs, cols, n)
        return _cmp(e.op, a, b), va & vb
    if isinstance(e, (And, Or)):
        vals = [evaluate(c, cols, n) for c in e.children]
        t = [v.astype(bool) & ok for v, ok in vals]
        f = [~v.astype(bool) & ok for v, ok in vals]
        if isinstance(e, And):
            tt = np.logical_and.reduce(t)
            ff = np.logical_or.reduce(f)
        else:
            tt = np.logical_or.reduce(t)
            ff = np.logical_and.reduce(f)
        return tt, tt | ff
    if isinstance(e, Not):
        v, ok = evaluate(e.child, cols, n)
        return ~v.astype(bool), ok
    if isinstance(e, IsNull):
        _, ok = evaluate(e.child, cols, n)
        r = ok if e.negate else ~ok
        return r, np.ones(n, bool)
    raise TypeError(e)


def selection(pred, cols, n) -> np.ndarray:
    if pred is None:
        return np.ones(n, bool)
    v, ok = evaluate(pred, cols, n)
    return v.astype(bool) & ok


def aggregate(pred, aggs: list[Aggregate], cols, n) -> list:
    sel = selection(pred, cols, n)
    out = []
    for a in aggs:
        if a.kind == A.AGG_COUNT_STAR:
            out.append(int(sel.sum()))
            continue
        v, ok = evaluate(a.arg, cols, n)
        m = sel & ok
        x = v[m]
        if a.kind == A.AGG_COUNT:
            out.append(int(m.sum()))
        elif x.size == 0:
            out.append(None)
        elif a.kind == A.AGG_SUM:
            out.append(float(x.astype(np.float64).sum()) if a.input_type in (A.FLOAT32, A.FLOAT64)
                       else int(x.astype(np.int64).sum()))
        elif a.kind == A.AGG_AVG:
            out.append(float(x.astype(np.float64).sum() / x.size) if a.input_type in (A.FLOAT32, A.FLOAT64)
                       else float(int(x.astype(np.int64).sum()) / x.size))
        elif a.kind == A.AGG_MIN:
            out.append(float(x.min()) if a.input_type in (A.FLOAT32, A.FLOAT64) else int(x.min()))
        else:
            out.append(float(x.max()) if a.input_type in (A.FLOAT32, A.FLOAT64) else int(x.max()))
    return out


def project(pred, select: list, cols, n):
    """WHERE + SELECT: list of (values, valid) for the surviving rows in input order."""
    sel = selection(pred, cols, n)
    res = []
    for s in select:
        if isinstance(s, int):
            v, nl, t = cols[s]
            valid = np.ones(n, bool) if nl is None else ~nl.astype(bool)
            res.append((v[sel], valid[sel]))
        else:
            v, ok = evaluate(s, cols, n)
            res.append((v[sel], ok[sel]))
    return res
