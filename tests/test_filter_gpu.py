"""Parity of the fused WHERE+aggregate and WHERE+projection kernels with the
oracle. Exact for integers, counts, MIN/MAX, text and row order; float
SUM/AVG within 1e-6 relative of the oracle's FP64 result."""
import numpy as np
import pytest

from oracle import expr_eval
from yallasql_b200 import _abi as A
from yallasql_b200 import datagen, ops
from yallasql_b200.expr import (Aggregate, And, Arith, Cast, ColumnRef, Compare, Constant, IsNull, Not, Or,
                                between)

from helpers import dev_batch, host, oracle_cols, rel_close

pytestmark = pytest.mark.gpu
FLOAT_TOL = 1e-6


def sales_query_exprs():
    """SUM(price*discount), COUNT(*), MIN(price), MAX(price) WHERE discount BETWEEN 1 AND 3
    AND qty < 25 AND category <> 'category_007' over (price, qty, discount, category)."""
    price, qty, disc, cat = (ColumnRef(0, A.FLOAT32), ColumnRef(1, A.INT32), ColumnRef(2, A.INT32),
                             ColumnRef(3, A.TEXT))
    pred = And(between(disc, Constant(1, A.INT32), Constant(3, A.INT32)),
               Compare(A.LT, qty, Constant(25, A.INT32)),
               Compare(A.NE, cat, Constant(datagen.EXCLUDED_CATEGORY, A.TEXT)))
    aggs = [Aggregate(A.AGG_SUM, Arith(A.MUL, price, Cast(disc, A.FLOAT32))), Aggregate(A.AGG_COUNT_STAR),
            Aggregate(A.AGG_MIN, price), Aggregate(A.AGG_MAX, price)]
    return pred, aggs


def check_aggs(got, want):
    assert len(got) == len(want)
    for g, w in zip(got, want):
        if isinstance(w, float) or isinstance(g, float):
            assert rel_close(g, w, FLOAT_TOL), (got, want)
        else:
            assert g == w, (got, want)


# 3,000,017 rows: enough steps per block for the staged (shared-memory ring)
# kernel; the smaller batches take the unstaged one.
@pytest.mark.parametrize("rows", [1_000_000, 0, 1, 5, 1023, 1024, 1025, 77_777, 3_000_017])
def test_sales_query_matches_oracle(cuda, orc, rows):
    t = datagen.sales_table(max(rows, 1), seed=0)
    cols = [t["price"][:rows], t["qty"][:rows], t["discount"][:rows], t["category"][:rows]]
    pred, aggs = sales_query_exprs()
    got = ops.filter_aggregate(dev_batch(cols), pred, aggs)
    want = expr_eval.aggregate(pred, aggs, oracle_cols(cols), rows)
    check_aggs(got, want)
    if rows > 0:
        s, c, mn, mx = orc.sales_query({k: v[:rows] for k, v in t.items()}, datagen.EXCLUDED_CATEGORY.encode())
        assert got[1] == c
        if c:
            assert got[2] == pytest.approx(mn, abs=0) and got[3] == pytest.approx(mx, abs=0)
            assert rel_close(got[0], s, FLOAT_TOL)


def test_sales_query_deterministic_and_batch_accumulation(cuda):
    t = datagen.sales_table(300_000, seed=5)
    cols = [t["price"], t["qty"], t["discount"], t["category"]]
    pred, aggs = sales_query_exprs()
    whole = ops.filter_aggregate(dev_batch(cols), pred, aggs)
    again = ops.filter_aggregate(dev_batch(cols), pred, aggs)
    assert whole == again  # bitwise: fixed partial order
    plan = ops.AggPlan([A.FLOAT32, A.INT32, A.INT32, A.TEXT], pred, aggs)
    st = ops.AggState(aggs)
    for lo in range(0, 300_000, 65_536):  # uneven 4 MB-style batches into one accumulator
        plan.run(dev_batch([c[lo:lo + 65_536] for c in cols]), st)
    check_aggs(st.read(), whole)


def _random_typed(rng, n, nulls_p=0.1):
    i32 = rng.integers(-1000, 1000, n).astype(np.int32)
    f32 = rng.normal(0, 100, n).astype(np.float32)
    i64 = rng.integers(-(1 << 40), 1 << 40, n).astype(np.int64)
    f64 = rng.normal(0, 1e6, n)
    words = ["", "a", "ab", "abc", "b", "zz", "hello world", "x" * 15]
    txt = datagen.text_slots([words[j] for j in rng.integers(0, len(words), n)])
    nl = [rng.random(n) < nulls_p for _ in range(5)]
    return [(i32, A.INT32, nl[0]), (f32, A.FLOAT32, nl[1]), (i64, A.INT64, nl[2]), (f64, A.FLOAT64, nl[3]),
            (txt, A.TEXT, nl[4])]


@pytest.mark.parametrize("rows", [1, 33, 4096, 50_001])
def test_all_aggregate_kinds_with_nulls(cuda, rows):
    rng = np.random.default_rng(rows)
    cols = _random_typed(rng, rows)
    c = [ColumnRef(i, t) for i, (_, t, _) in enumerate(cols)]
    pred = Or(Compare(A.GT, c[0], Constant(-500, A.INT32)), Compare(A.EQ, c[4], Constant("abc", A.TEXT)))
    aggs = []
    for kind in (A.AGG_COUNT, A.AGG_SUM, A.AGG_AVG, A.AGG_MIN, A.AGG_MAX):
        for col in c[:4]:
            aggs.append(Aggregate(kind, col))
    aggs.append(Aggregate(A.AGG_COUNT_STAR))
    for lo in range(0, len(aggs), 8):
        part = aggs[lo:lo + 8]
        got = ops.filter_aggregate(dev_batch(cols), pred, part)
        want = expr_eval.aggregate(pred, part, oracle_cols(cols), rows)
        check_aggs(got, want)


@pytest.mark.parametrize("rows", [0, 1, 7, 1024, 1025, 200_003])
def test_where_projection_matches_oracle(cuda, rows):
    rng = np.random.default_rng(100 + rows)
    cols = _random_typed(rng, max(rows, 1))
    cols = [(a[:rows], t, n[:rows]) for a, t, n in cols]
    c = [ColumnRef(i, t) for i, (_, t, _) in enumerate(cols)]
    pred = And(Compare(A.GE, c[0], Constant(-200, A.INT32)), Not(Compare(A.LT, c[1], Constant(0.0, A.FLOAT32))),
               Compare(A.NE, c[4], Constant("zz", A.TEXT)))
    select = [0, 4, 2, Arith(A.ADD, c[0], Constant(7, A.INT32)),
              Arith(A.MUL, Cast(c[0], A.FLOAT32), c[1]), Arith(A.DIV, c[2], Cast(c[0], A.INT64)),
              Compare(A.LE, c[3], Constant(0.5, A.FLOAT64))]
    out = ops.filter_project(dev_batch(cols), pred, select)
    want = expr_eval.project(pred, select, oracle_cols(cols), rows)
    assert out.rows == len(want[0][0])
    for col, (wv, wvalid) in zip(out.columns, want):
        v, nl = host(col)
        valid = ~nl
        np.testing.assert_array_equal(valid, wvalid)
        if v.dtype == np.uint8 and v.ndim == 1:
            v = v.astype(bool)
        np.testing.assert_array_equal(v[valid], np.asarray(wv)[wvalid].astype(v.dtype))


# Batches long enough that one claimed chunk spans several 1,024-row steps,
# with a last chunk that ends early (its missing steps sit between the
# predicate pass and the output pass of the ring).
@pytest.mark.parametrize("jit", [True, False])
@pytest.mark.parametrize("rows", [2_500_001, 5_000_000, 9_437_185])
def test_sales_projection_multi_step_chunks(cuda, rows, jit):
    t = datagen.sales_table(rows, seed=11)
    cols = [t["price"], t["qty"], t["discount"], t["category"]]
    price, disc = ColumnRef(0, A.FLOAT32), ColumnRef(2, A.INT32)
    pred, _ = sales_query_exprs()
    select = [3, 0, Arith(A.MUL, price, Cast(disc, A.FLOAT32)), 1]
    lib = ops.lib()
    prev = lib.yq_jit_enable(1 if jit else 0)
    try:
        out = ops.filter_project(dev_batch(cols), pred, select)
    finally:
        lib.yq_jit_enable(prev)
    keep = ((t["discount"] >= 1) & (t["discount"] <= 3) & (t["qty"] < 25) &
            np.any(t["category"] != datagen.text_slots([datagen.EXCLUDED_CATEGORY])[0], axis=1))
    assert out.rows == int(keep.sum())
    np.testing.assert_array_equal(host(out.columns[0])[0], t["category"][keep])
    np.testing.assert_array_equal(host(out.columns[1])[0], t["price"][keep])
    np.testing.assert_array_equal(host(out.columns[2])[0],
                                  (t["price"] * t["discount"].astype(np.float32))[keep])
    np.testing.assert_array_equal(host(out.columns[3])[0], t["qty"][keep])


def test_projection_capacity_reported(cuda):
    rng = np.random.default_rng(3)
    x = rng.integers(0, 100, 10_000).astype(np.int32)
    plan = ops.ProjectPlan([A.INT32], [4], Compare(A.LT, ColumnRef(0, A.INT32), Constant(50, A.INT32)), [0])
    with pytest.raises(A.YQError) as e:
        plan.run(dev_batch([x]), capacity=100)
    assert e.value.status == A.ERR_CAPACITY


def test_three_valued_logic_truth_table(cuda):
    # a, b in {TRUE, FALSE, NULL}^2 via comparisons on nullable int columns
    vals = np.array([1, 0, 0, 1, 0, 0, 1, 0, 0], np.int32)
    na = np.array([0, 0, 1, 0, 0, 1, 0, 0, 1], bool)
    vb = np.array([1, 1, 1, 0, 0, 0, 0, 0, 0], np.int32)
    nb = np.array([0, 0, 0, 0, 0, 0, 1, 1, 1], bool)
    cols = [(vals, A.INT32, na), (vb, A.INT32, nb)]
    a = Compare(A.EQ, ColumnRef(0, A.INT32), Constant(1, A.INT32))
    b = Compare(A.EQ, ColumnRef(1, A.INT32), Constant(1, A.INT32))
    select = [And(a, b), Or(a, b), Not(a), IsNull(ColumnRef(0, A.INT32)), IsNull(ColumnRef(1, A.INT32), negate=True)]
    out = ops.filter_project(dev_batch(cols), None, select)
    want = expr_eval.project(None, select, oracle_cols(cols), 9)
    for col, (wv, wvalid) in zip(out.columns, want):
        v, nl = host(col)
        np.testing.assert_array_equal(~nl, wvalid)
        np.testing.assert_array_equal(v.astype(bool)[wvalid], np.asarray(wv).astype(bool)[wvalid])
