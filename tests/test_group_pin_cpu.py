"""GROUP BY oracle pinned against pandas.

The reference ignores GROUP BY (AggregateOperator folds every row into one
result, include/engine/operators/aggregate_operator.hpp:84-104) and defers SQL
semantics to DuckDB, which is not available here. pandas' groupby (an
implementation this repository did not write) stands in for it on the cases
where the two agree with SQL: `sort=True, dropna=False` gives one row per
distinct key in ascending order with the NULL group last; `size` is COUNT(*),
`count` COUNT(col); `sum(min_count=1)`, `mean`, `min`, `max` skip NULLs and are
NULL over no non-NULL input. Keys here hold no NaN or -0.0 (pandas folds NaN
into NULL; SQL keeps it a value), which `test_group_cpu.py` covers against a
plain restatement instead.
"""
import numpy as np
import pandas as pd
import pytest

import oracle

KINDS = ["size", "count", "sum", "mean", "min", "max"]  # oracle kinds 0..5


def pandas_group_by(key, key_nulls, vals, vnulls, key_kind):
    if key_kind == "text":
        k = pd.array([None if n else bytes(row).rstrip(b"\0").decode() for row, n in zip(key, key_nulls)],
                     dtype="string")
    elif key_kind == "float":
        k = pd.array(np.where(key_nulls, np.nan, key.astype(np.float64)), dtype="Float64")
        k[key_nulls] = pd.NA
    else:
        k = pd.array(key.astype(np.int64), dtype="Int64")
        k[key_nulls] = pd.NA
    cols = {}
    for name, (v, vn) in vals.items():
        if v.dtype.kind == "f":
            a = pd.array(v.astype(np.float64), dtype="Float64")
        else:
            a = pd.array(v.astype(np.int64), dtype="Int64")
        a[vn] = pd.NA
        cols[name] = a
    df = pd.DataFrame({"k": k, **cols})
    g = df.groupby("k", sort=True, dropna=False)
    return g


def oracle_type(a):
    return {np.dtype(np.int32): 0, np.dtype(np.float32): 1, np.dtype(np.int64): 4, np.dtype(np.float64): 5}[a.dtype]


@pytest.mark.parametrize("key_kind", ["int", "float", "text", "bigint"])
def test_group_by_oracle_matches_pandas(key_kind):
    rng = np.random.default_rng({"int": 1, "float": 2, "text": 3, "bigint": 4}[key_kind])
    for trial in range(6):
        n = int(rng.integers(1, 3000))
        ndist = int(rng.integers(1, 60))
        if key_kind == "int":
            key, ktype = rng.integers(-20, 20, n).astype(np.int32), 0
        elif key_kind == "bigint":
            key, ktype = (rng.integers(0, ndist, n) * (1 << 35) - (1 << 40)).astype(np.int64), 4
        elif key_kind == "float":
            key, ktype = (rng.integers(-ndist, ndist, n) * 0.75 + 0.125).astype(np.float32), 1
        else:
            words = [f"w{i:03d}" for i in range(ndist)]
            key = np.zeros((n, 16), np.uint8)
            for i, j in enumerate(rng.integers(0, ndist, n)):
                b = words[j].encode()
                key[i, :len(b)] = np.frombuffer(b, np.uint8)
            ktype = 3
        knull = rng.random(n) < 0.08
        fv = np.round(rng.normal(0, 100, n), 2).astype(np.float32)
        iv = rng.integers(-1000, 1000, n).astype(np.int32)
        fnull, inull = rng.random(n) < 0.15, rng.random(n) < 0.15
        if trial == 0:  # a group whose values are all NULL
            fnull[:] = True
        aggs = [(0, None, None, 0)] + [(kind, v, vn, oracle_type(v)) for v, vn in ((fv, fnull), (iv, inull))
                                       for kind in range(1, 6)]
        ok, okn, res = oracle.group_by(key, knull, ktype, aggs)
        g = pandas_group_by(key, knull, {"f": (fv, fnull), "i": (iv, inull)}, None, "text" if ktype == 3 else
                            ("float" if ktype == 1 else "int"))
        size = g.size()
        assert len(ok) == len(size)
        # keys: same order, NULL group last
        pk = list(size.index)
        for gi, want in enumerate(pk):
            if pd.isna(want):
                assert okn[gi]
            elif ktype == 3:
                assert not okn[gi] and bytes(ok[gi]).rstrip(b"\0").decode() == want
            else:
                assert not okn[gi] and ok[gi] == want
        np.testing.assert_array_equal(res[0][0], size.to_numpy(np.int64))
        idx = 1
        for col in ("f", "i"):
            s = g[col]
            want = {1: s.count(), 2: s.sum(min_count=1), 3: s.mean(), 4: s.min(), 5: s.max()}
            for kind in range(1, 6):
                vals, nulls = res[idx]
                w = want[kind]
                idx += 1
                if kind == 1:
                    np.testing.assert_array_equal(vals, w.to_numpy(np.int64))
                    continue
                wn = w.isna().to_numpy()
                np.testing.assert_array_equal(nulls.astype(bool), wn)
                wv = w.to_numpy(np.float64, na_value=0.0)
                gv = np.where(wn, 0.0, vals.astype(np.float64))
                if kind in (2, 3) and col == "f":
                    np.testing.assert_allclose(gv, wv, rtol=1e-9, atol=1e-9)
                else:
                    np.testing.assert_array_equal(gv, wv)
