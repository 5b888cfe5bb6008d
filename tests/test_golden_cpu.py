"""The oracle against golden outputs of the reference's own kernels
(tests/golden/*.npz, written by tests/golden/make_golden.py from the
reference's src/kernels built into oracle/_ref). CPU only."""
import os

import numpy as np
import pytest

import oracle
from oracle import expr_eval
from yallasql_b200 import _abi as A
from yallasql_b200.expr import Arith, Cast, ColumnRef

from helpers import oracle_cols

G = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    p = os.path.join(G, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} not generated")
    return np.load(p)


def test_reductions_match_reference():
    z = load("reduce.npz")
    f, i, nulls, out = z["f"], z["i"], z["nulls"], z["out"]
    n = len(f)
    cols = {0: (f, nulls, A.FLOAT32), 1: (i, nulls, A.INT32)}
    want = expr_eval.aggregate(None, [expr_eval.Aggregate(A.AGG_SUM, ColumnRef(0, A.FLOAT32)),
                                      expr_eval.Aggregate(A.AGG_MIN, ColumnRef(0, A.FLOAT32)),
                                      expr_eval.Aggregate(A.AGG_MAX, ColumnRef(0, A.FLOAT32)),
                                      expr_eval.Aggregate(A.AGG_SUM, ColumnRef(1, A.INT32)),
                                      expr_eval.Aggregate(A.AGG_MIN, ColumnRef(1, A.INT32)),
                                      expr_eval.Aggregate(A.AGG_MAX, ColumnRef(1, A.INT32)),
                                      expr_eval.Aggregate(A.AGG_COUNT, ColumnRef(1, A.INT32))], cols, n)
    assert abs(out[0] - want[0]) <= 1e-9 * abs(want[0])  # FP64 sums in different orders
    assert [float(x) for x in out[1:]] == [float(x) for x in want[1:]]


@pytest.mark.parametrize("name,desc", [("merge_asc.npz", False), ("merge_desc.npz", True)])
def test_merge_order_and_ties_match_reference(name, desc):
    z = load(name)
    a, b, k = z["a"], z["b"], int(z["k"])
    both = np.concatenate([a, b])
    order = oracle.sort_perm(both, desc=desc)[:k]
    np.testing.assert_array_equal(z["merged"], both[order])
    np.testing.assert_array_equal(z["from_a"], (order < len(a)).astype(np.uint8))  # ties take run A
    assert int(z["last"]) == int((order < len(a)).sum())


def test_join_pairs_match_reference():
    z = load("join_eq.npz")
    wl, wr = oracle.join_pairs([z["left"]], [z["right"]], [(0, 0, A.EQ)])
    assert sorted(zip(wl.tolist(), wr.tolist())) == [tuple(p) for p in z["pairs"].tolist()]


def test_mul_cast_matches_reference():
    z = load("mul_cast.npz")
    e = Arith(A.MUL, ColumnRef(0, A.FLOAT32), Cast(ColumnRef(1, A.INT32), A.FLOAT32))
    want = expr_eval.evaluate(e, oracle_cols([z["price"], z["discount"]]), len(z["price"]))[0]
    np.testing.assert_array_equal(z["out"], want)
