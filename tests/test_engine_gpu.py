"""The C++ operator layer end to end from host columns: scan (pinned,
double-buffered H2D) -> operators -> host result, against the oracle."""
import numpy as np
import pytest
import torch

import oracle
from oracle import expr_eval
from yallasql_b200 import _abi as A
from yallasql_b200 import datagen
from yallasql_b200.expr import Aggregate, Arith, Cast, ColumnRef, Compare, Constant
from yallasql_b200.plan import Plan

from helpers import oracle_cols, rel_close
from test_filter_gpu import sales_query_exprs

pytestmark = pytest.mark.gpu


def sales_cols(rows, seed=0):
    t = datagen.sales_table(rows, seed=seed)
    return t, [t["price"], t["qty"], t["discount"], t["category"]]


@pytest.mark.parametrize("batch_rows", [0, 4096, 100_000])
def test_filter_aggregate_query(cuda, batch_rows):
    t, cols = sales_cols(500_000)
    pred, aggs = sales_query_exprs()
    p = Plan()
    root = p.aggregate(p.filter(p.scan(cols, batch_rows=batch_rows), pred), aggs)
    res = p.execute(root)
    got = [v[0] if (n is None or not n[0]) else None for v, n in res]
    want = expr_eval.aggregate(pred, aggs, oracle_cols(cols), len(cols[0]))
    assert int(got[1]) == want[1]
    assert float(got[2]) == want[2] and float(got[3]) == want[3]
    assert rel_close(float(got[0]), want[0], 1e-6)
    st = p.stats()
    assert st.batches >= 1 and st.h2d_bytes == sum(c.nbytes for c in cols)


def test_empty_aggregate_returns_one_row(cuda):
    _, cols = sales_cols(1000)
    p = Plan()
    never = Compare(A.LT, ColumnRef(1, A.INT32), Constant(-1, A.INT32))
    aggs = [Aggregate(A.AGG_COUNT_STAR), Aggregate(A.AGG_SUM, ColumnRef(0, A.FLOAT32)),
            Aggregate(A.AGG_MIN, ColumnRef(1, A.INT32))]
    res = p.execute(p.aggregate(p.filter(p.scan(cols), never), aggs))
    assert res[0][0][0] == 0 and res[1][1][0] and res[2][1][0]


def test_filter_project_query_pinned_and_pageable(cuda):
    t, cols = sales_cols(300_000, seed=4)
    pred, _ = sales_query_exprs()
    select = [3, 0, Arith(A.MUL, ColumnRef(0, A.FLOAT32), Cast(ColumnRef(2, A.INT32), A.FLOAT32))]
    want = expr_eval.project(pred, select, oracle_cols(cols), len(cols[0]))
    for pinned in (False, True):
        p = Plan()
        if pinned:
            src = [torch.from_numpy(c).pin_memory() for c in cols]
            scan = p.scan(src, types=[A.FLOAT32, A.INT32, A.INT32, A.TEXT], batch_rows=50_000)
        else:
            scan = p.scan(cols, batch_rows=50_000)
        res = p.execute(p.project(p.filter(scan, pred), select))
        for (v, _), (wv, _) in zip(res, want):
            np.testing.assert_array_equal(v, np.asarray(wv).astype(v.dtype))


@pytest.mark.parametrize("budget", [0, 1 << 20])
def test_order_by_query_with_spills(cuda, budget):
    t = datagen.order_table(200_000, seed=1, dist="zipf")
    cols = [t["key"], t["id"], t["txt"], t["d"]]
    p = Plan(gpu_budget=budget)
    root = p.order(p.scan(cols, types=[A.FLOAT32, A.INT64, A.TEXT, A.DATETIME], batch_rows=7000), 0, descending=True)
    res = p.execute(root)
    perm = oracle.sort_perm(t["key"], desc=True)
    for (v, _), name in zip(res, ["key", "id", "txt", "d"]):
        np.testing.assert_array_equal(v, t[name][perm])
    if budget:
        assert p.stats().spilled_batches > 0


@pytest.mark.parametrize("host_budget", [1 << 20, 1])
def test_order_by_query_spills_to_files(cuda, tmp_path, host_budget):
    """Device budget 1 MB and a host budget: spilled batches move on to files
    in the cache directory (the reference's FS tier) with their null bytes,
    come back for the merge, and the files are gone afterwards. The key and
    a payload column carry nulls."""
    rng = np.random.default_rng(12)
    t = datagen.order_table(150_000, seed=3, dist="zipf")
    knull = rng.random(len(t["key"])) < 0.03
    inull = rng.random(len(t["key"])) < 0.1
    cols = [t["key"], t["id"], t["txt"], t["d"]]
    p = Plan(gpu_budget=1 << 20, host_budget=host_budget, cache_dir=str(tmp_path))
    root = p.order(p.scan(cols, types=[A.FLOAT32, A.INT64, A.TEXT, A.DATETIME], nulls=[knull, inull, None, None],
                          batch_rows=6000), 0, descending=True)
    res = p.execute(root)
    st = p.stats()
    assert st.spilled_batches > 0 and st.disk_batches > 0
    assert list(tmp_path.iterdir()) == []
    perm = oracle.sort_perm(t["key"], desc=True, nulls=knull)
    np.testing.assert_array_equal(res[0][1].astype(bool), knull[perm])
    np.testing.assert_array_equal(res[1][1].astype(bool), inull[perm])
    np.testing.assert_array_equal(np.where(knull[perm], 0, res[0][0]), np.where(knull[perm], 0, t["key"][perm]))
    for (v, _), name in zip(res[1:], ["id", "txt", "d"]):
        np.testing.assert_array_equal(v, t[name][perm])


def test_spill_needs_a_directory(cuda):
    from yallasql_b200.plan import lib as plan_lib
    p = Plan()
    assert plan_lib().yq_plan_set_spill(p.h, 1 << 20, None) == A.ERR_INVALID_ARG
    assert plan_lib().yq_plan_set_spill(p.h, 0, None) == 0


def test_or_join_query(cuda):
    """JoinOperator with an OR of ANDs (the reference throws on OR in a join
    condition): fact.datekey = dim.datekey OR fact.quantity > dim.year - 1945,
    over several batches on both sides, against the union of the groups'
    oracle pairs."""
    fact, dim = datagen.star_tables(6_000, seed=4)
    dyear = (dim["year"] - 1945).astype(np.int32)
    p = Plan()
    f = p.scan([fact["datekey"], fact["quantity"]], batch_rows=2048)
    d = p.scan([dim["datekey"], dyear], batch_rows=700)
    res = p.execute(p.join(f, d, [(0, 0, A.EQ), (1, 1, A.GT)], disjunct=[0, 1]))
    got = sorted(zip(*[r[0].tolist() for r in res]))
    pairs = set()
    for conds in ([(0, 0, A.EQ)], [(1, 1, A.GT)]):
        wl, wr = oracle.join_pairs([fact["datekey"], fact["quantity"]], [dim["datekey"], dyear], conds)
        pairs.update(zip(wl.tolist(), wr.tolist()))
    want = sorted((int(fact["datekey"][l]), int(fact["quantity"][l]), int(dim["datekey"][r]), int(dyear[r]))
                  for l, r in pairs)
    assert got == want


def test_join_and_cross_product_queries(cuda):
    fact, dim = datagen.star_tables(50_000, seed=2)
    p = Plan()
    f = p.scan([fact["datekey"], fact["quantity"]], batch_rows=16_384)
    d = p.filter(p.scan([dim["datekey"], dim["year"]]), Compare(A.EQ, ColumnRef(1, A.INT32), Constant(1993, A.INT32)))
    res = p.execute(p.join(f, d, [(0, 0, A.EQ)]))
    got = sorted(zip(res[0][0].tolist(), res[1][0].tolist(), res[2][0].tolist(), res[3][0].tolist()))
    keep = dim["year"] == 1993
    wl, wr = oracle.join_pairs([fact["datekey"]], [dim["datekey"][keep]], [(0, 0, A.EQ)])
    want = sorted(zip(fact["datekey"][wl].tolist(), fact["quantity"][wl].tolist(),
                      dim["datekey"][keep][wr].tolist(), dim["year"][keep][wr].tolist()))
    assert got == want
    x, y = datagen.cross_tables(300, seed=2)
    p2 = Plan()
    res2 = p2.execute(p2.cross(p2.scan([x]), p2.scan([y])))
    assert len(res2[0][0]) == 300 * 300
    np.testing.assert_array_equal(res2[0][0], np.repeat(x, 300))
    np.testing.assert_array_equal(res2[1][0], np.tile(y, 300))


@pytest.mark.parametrize("batch_rows", [0, 7_000])
def test_group_by_node(cuda, batch_rows):
    """GROUP BY as an operator-tree node over scanned batches (the reference's
    AggregateOperator ignores the groups): scan -> WHERE -> GROUP BY discount
    with COUNT(*), SUM(price), AVG(qty), MIN(price), MAX(price), against the
    oracle's GROUP BY of the filtered rows."""
    rng = np.random.default_rng(31)
    t, cols = sales_cols(300_001, seed=5)
    pnull = rng.random(len(t["price"])) < 0.05
    p = Plan()
    scan = p.scan(cols, nulls=[pnull, None, None, None], batch_rows=batch_rows)
    where = p.filter(scan, Compare(A.LT, ColumnRef(1, A.INT32), Constant(40, A.INT32)))
    aggs = [(A.AGG_COUNT_STAR, 0), (A.AGG_SUM, 0), (A.AGG_AVG, 1), (A.AGG_MIN, 0), (A.AGG_MAX, 0)]
    res = p.execute(p.group_by(where, 2, aggs))
    keep = t["qty"] < 40
    price, pn, qty, disc = t["price"][keep], pnull[keep], t["qty"][keep], t["discount"][keep]
    okey, okn, ores = oracle.group_by(disc, None, A.INT32, [(0, None, None, 0), (2, price, pn, 1), (3, qty, None, 0),
                                                            (4, price, pn, 1), (5, price, pn, 1)])
    np.testing.assert_array_equal(res[0][0], okey)
    for j, (w, wn) in enumerate(ores):
        got, gn = res[1 + j]
        if wn is None:
            np.testing.assert_array_equal(got, w)
            continue
        np.testing.assert_array_equal(gn, wn)
        if got.dtype == np.float64 and j in (1, 2):
            np.testing.assert_allclose(np.where(wn, 0, got), np.where(wn, 0, w), rtol=1e-9)
        else:
            np.testing.assert_array_equal(np.where(wn, 0, got), np.where(wn, 0, w))


@pytest.mark.parametrize("batch_rows", [0, 50_000])
def test_order_by_several_keys_node(cuda, batch_rows):
    """ORDER BY discount DESC, qty ASC, price DESC as one node (the reference
    sorts by its first key only): stable, every column moved."""
    t, cols = sales_cols(400_003, seed=6)
    p = Plan()
    root = p.order_multi(p.scan(cols, batch_rows=batch_rows), [2, 1, 0], [True, False, True])
    res = p.execute(root)
    perm = oracle.sort_perm_multi([t["discount"], t["qty"], t["price"]], [True, False, True])
    for (got, _), want in zip(res, cols):
        np.testing.assert_array_equal(got, want[perm])


def test_order_by_long_text_key_node(cuda):
    """One text key longer than the merge path's 32 bytes: the node sorts the
    whole input by its chunked text key instead of merging runs."""
    rng = np.random.default_rng(7)
    n = 60_000
    words = ["k" * int(rng.integers(20, 60)) + "".join(rng.choice(list("xyz"), 5)) for _ in range(n)]
    txt = datagen.text_slots(words, 96)
    ids = np.arange(n, dtype=np.int64)
    p = Plan()
    res = p.execute(p.order(p.scan([txt, ids], batch_rows=8_192), 0, descending=False))
    perm = oracle.sort_perm(txt)
    np.testing.assert_array_equal(res[1][0], ids[perm])
    np.testing.assert_array_equal(res[0][0], txt[perm])
