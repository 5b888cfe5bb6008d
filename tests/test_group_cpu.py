"""The GROUP BY oracle (numpy) against a plain Python restatement of the same
SQL semantics on small inputs: groups, their order, NULL handling, float
equality (-0.0 = +0.0, NaN one group) and every aggregate."""
import math
import struct

import numpy as np

import oracle


def f64_order_key(x):
    if math.isnan(x):
        return (2, 0.0)
    return (1, x, 0 if math.copysign(1.0, x) < 0 else 1)


def python_group_by(keys, knull, vals, vnull):
    groups = {}
    order = []
    for i, (k, kn) in enumerate(zip(keys, knull)):
        if kn:
            g = ("null",)
        elif isinstance(k, float) and math.isnan(k):
            g = ("nan",)
        else:
            g = ("v", 0.0 if k == 0 else k)
        if g not in groups:
            groups[g] = []
            order.append(g)
        groups[g].append(i)

    def sort_key(g):
        if g[0] == "null":
            return (2, 0)
        if g[0] == "nan":
            return (1, math.inf, 1)
        return (1, g[1], 0)
    out = []
    for g in sorted(order, key=sort_key):
        rows = groups[g]
        present = [vals[i] for i in rows if not vnull[i]]
        s = sum(present) if present else None
        mn = min(present, key=f64_order_key) if present else None
        mx = max(present, key=f64_order_key) if present else None
        out.append((keys[rows[0]], knull[rows[0]], len(rows), len(present), s,
                    None if not present else s / len(present), mn, mx))
    return out


def test_group_by_oracle_matches_python():
    rng = np.random.default_rng(40)
    for trial in range(30):
        n = int(rng.integers(1, 300))
        keys = rng.choice(np.array([0.0, -0.0, 1.5, -2.0, np.nan, np.inf, 7.0]), n)
        knull = rng.random(n) < 0.1
        vals = np.round(rng.normal(0, 10, n), 3)
        vals[rng.random(n) < 0.05] = -0.0
        vnull = rng.random(n) < 0.2
        ok, okn, res = oracle.group_by(keys, knull, 5, [(0, None, None, 5), (1, vals, vnull, 5), (2, vals, vnull, 5),
                                                        (3, vals, vnull, 5), (4, vals, vnull, 5), (5, vals, vnull, 5)])
        want = python_group_by(list(keys), list(knull), list(vals), list(vnull))
        assert len(ok) == len(want)
        for gi, w in enumerate(want):
            assert struct.pack("<d", ok[gi]) == struct.pack("<d", w[0]) and bool(okn[gi]) == bool(w[1])
            assert res[0][0][gi] == w[2] and res[1][0][gi] == w[3]
            if w[4] is None:
                assert res[2][1][gi] and res[3][1][gi] and res[4][1][gi] and res[5][1][gi]
            else:
                assert abs(res[2][0][gi] - w[4]) <= 1e-9 * max(1.0, abs(w[4]))
                assert abs(res[3][0][gi] - w[5]) <= 1e-9 * max(1.0, abs(w[5]))
                assert struct.pack("<d", res[4][0][gi]) == struct.pack("<d", w[6])
                assert struct.pack("<d", res[5][0][gi]) == struct.pack("<d", w[7])


def test_group_by_wrapper_rejects_more_aggregates_than_the_limit():
    """yq_group_by takes at most YQ_MAX_AGGREGATES (8) aggregates a call; the
    Python wrapper says so before touching the device."""
    import pytest
    from yallasql_b200 import _abi as A
    from yallasql_b200 import ops
    with pytest.raises(ValueError, match="at most 8"):
        ops.group_by(None, 0, [(A.AGG_COUNT_STAR, 0)] * 9)
