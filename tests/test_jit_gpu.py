"""Program-specialised row kernels (runtime compiled) against the interpreting
kernels: same programs, same inputs, same results (float SUM/AVG at 1e-12
relative, since a different grid sums partials in another order; everything
else exact), and the compiler really ran on this box."""
import ctypes as C

import numpy as np
import pytest
import torch

from yallasql_b200 import _abi as A
from yallasql_b200 import datagen, ops
from yallasql_b200.expr import (Aggregate, And, Arith, Cast, ColumnRef, Compare, Constant, IsNull, Not, Or,
                                between)

from helpers import dev_col

pytestmark = pytest.mark.gpu


def stats():
    c, f, h, ms = C.c_int32(), C.c_int32(), C.c_int32(), C.c_double()
    log = C.create_string_buffer(4096)
    ops.lib().yq_jit_stats(C.byref(c), C.byref(f), C.byref(h), C.byref(ms), log, 4096)
    return c.value, f.value, h.value, ms.value, log.value.decode(errors="replace")


def both(fn):
    lib = ops.lib()
    prev = lib.yq_jit_enable(0)
    try:
        a = fn()
        lib.yq_jit_enable(1)
        b = fn()
    finally:
        lib.yq_jit_enable(prev)
    return a, b


def same_aggs(a, b):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        if isinstance(x, float) and isinstance(y, float):
            assert abs(x - y) <= 1e-12 * max(1.0, abs(x))
        else:
            assert x == y


def sales(rows, seed=0, nulls=False):
    t = datagen.sales_table(rows, seed=seed)
    rng = np.random.default_rng(seed)
    nl = (rng.random(rows) < 0.1) if nulls else None
    b = ops.DeviceBatch([dev_col(t["price"], A.FLOAT32, nl), dev_col(t["qty"], A.INT32),
                         dev_col(t["discount"], A.INT32), dev_col(t["category"], A.TEXT)])
    return b


PRICE, QTY, DISC, CAT = ColumnRef(0, A.FLOAT32), ColumnRef(1, A.INT32), ColumnRef(2, A.INT32), ColumnRef(3, A.TEXT)
PROGRAMS = {
    "sales": (And(between(DISC, Constant(1, A.INT32), Constant(3, A.INT32)), Compare(A.LT, QTY, Constant(25, A.INT32)),
                  Compare(A.NE, CAT, Constant(datagen.EXCLUDED_CATEGORY, A.TEXT))),
              [Aggregate(A.AGG_SUM, Arith(A.MUL, PRICE, Cast(DISC, A.FLOAT32))), Aggregate(A.AGG_COUNT_STAR),
               Aggregate(A.AGG_MIN, PRICE), Aggregate(A.AGG_MAX, PRICE)]),
    "divmod_casts": (Or(Compare(A.GT, Arith(A.MOD, QTY, DISC), Constant(2, A.INT32)),
                        Not(Compare(A.LE, Cast(PRICE, A.INT32), Constant(500, A.INT32)))),
                     [Aggregate(A.AGG_SUM, Arith(A.DIV, QTY, DISC)), Aggregate(A.AGG_AVG, Cast(PRICE, A.FLOAT64)),
                      Aggregate(A.AGG_MAX, Cast(PRICE, A.INT64)), Aggregate(A.AGG_COUNT, Arith(A.DIV, QTY, DISC))]),
    "text_order_nulls": (And(Compare(A.GE, CAT, Constant("category_010", A.TEXT)), Not(IsNull(PRICE))),
                         [Aggregate(A.AGG_MIN, PRICE), Aggregate(A.AGG_COUNT, PRICE), Aggregate(A.AGG_SUM, QTY)]),
}


@pytest.mark.parametrize("name", list(PROGRAMS))
@pytest.mark.parametrize("rows", [1, 1023, 300_001])
def test_filter_aggregate_same_results(cuda, name, rows):
    pred, aggs = PROGRAMS[name]
    b = sales(rows, seed=rows % 7, nulls=(name == "text_order_nulls"))
    a, j = both(lambda: ops.filter_aggregate(b, pred, aggs))
    same_aggs(a, j)
    c, f, _, _, log = stats()
    assert f == 0, log
    assert c > 0


@pytest.mark.parametrize("name", list(PROGRAMS))
def test_filter_project_same_rows(cuda, name):
    pred, _ = PROGRAMS[name]
    b = sales(200_003, seed=3, nulls=(name == "text_order_nulls"))
    sel = [3, Arith(A.MUL, PRICE, Cast(DISC, A.FLOAT32)), Arith(A.MOD, QTY, Constant(7, A.INT32))]
    a, j = both(lambda: ops.filter_project(b, pred, sel))
    for x, y in zip(a.columns, j.columns):
        assert torch.equal(x.data, y.data)
        if x.nulls is not None:
            assert torch.equal(x.nulls, y.nulls)


def test_segmented_and_join_same_results(cuda):
    pred, aggs = PROGRAMS["sales"]
    b = sales(500_000, seed=5)
    offs = [0, 7, 1500, 1500, 200_000, 500_000]
    plan = ops.AggPlan([A.FLOAT32, A.INT32, A.INT32, A.TEXT], pred, aggs)

    def seg():
        st = ops.AggStates(aggs, len(offs) - 1)
        plan.run_segments(b, offs, st)
        return st.read()
    a, j = both(seg)
    for x, y in zip(a, j):
        same_aggs(x, y)
    fact, dim = datagen.star_tables(400_000, seed=2)
    fb = ops.DeviceBatch([dev_col(fact["datekey"]), dev_col(fact["quantity"]), dev_col(fact["discount"]),
                          dev_col(fact["extendedprice"])])
    db = ops.DeviceBatch([dev_col(dim["datekey"]), dev_col(dim["year"]), dev_col(dim["month"])])
    jp = ops.JoinAggPlan([A.INT32] * 3 + [A.FLOAT32], [A.INT32] * 3,
                         And(between(ColumnRef(2, A.INT32), Constant(1, A.INT32), Constant(3, A.INT32)),
                             Compare(A.LT, ColumnRef(1, A.INT32), Constant(25, A.INT32))), 0,
                         Compare(A.EQ, ColumnRef(1, A.INT32), Constant(1993, A.INT32)), 0,
                         [Aggregate(A.AGG_SUM, Arith(A.MUL, ColumnRef(3, A.FLOAT32),
                                                     Cast(ColumnRef(2, A.INT32), A.FLOAT32))),
                          Aggregate(A.AGG_COUNT_STAR)])

    def join():
        st = ops.AggState(jp.aggs)
        jp.run(fb, db, st)
        return st.read()
    a, j = both(join)
    same_aggs(a, j)
    assert stats()[1] == 0
