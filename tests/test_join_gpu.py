"""Join parity: pair multisets (here: identical ordered lists, since both
sides emit (left asc, right asc)) against the nested-loop oracle, the
predicate cross product against its oracle, and the fused star-join
aggregate against the C oracle of the config query."""
import numpy as np
import pytest

import oracle
from oracle import expr_eval
from yallasql_b200 import _abi as A
from yallasql_b200 import datagen, ops
from yallasql_b200.expr import Aggregate, And, Arith, Cast, ColumnRef, Compare, Constant, between

from helpers import dev_batch, dev_col, rel_close

pytestmark = pytest.mark.gpu


def pairs_np(l, r):
    return l.cpu().numpy().view(np.uint32), r.cpu().numpy().view(np.uint32)


def random_side(rng, n, nulls_p=0.0):
    k = rng.integers(0, 50, n).astype(np.int32)
    v = rng.integers(-100, 100, n).astype(np.int64)
    f = rng.normal(0, 5, n).astype(np.float32)
    t = datagen.text_slots([["a", "b", "c", "dd"][j] for j in rng.integers(0, 4, n)])
    nk = (rng.random(n) < nulls_p) if nulls_p else None
    return [k, v, f, t], [nk, None, None, None]


@pytest.mark.parametrize("L,R", [(1, 1), (33, 17), (1025, 300), (5000, 2048), (3000, 9000)])
@pytest.mark.parametrize("conds", [
    [(0, 0, A.EQ)],                      # equality: hashed right side (nested loop when R > 8192)
    [(0, 0, A.EQ), (1, 1, A.LT)],        # equality + residual inequality
    [(1, 1, A.LT)],                      # inequality only: nested loop
    [(3, 3, A.EQ)],                      # text equality: nested loop
    [(2, 2, A.GE), (0, 0, A.NE)],
])
def test_join_pairs_match_oracle(cuda, L, R, conds):
    rng = np.random.default_rng(L * 31 + R)
    lc, ln = random_side(rng, L, 0.05)
    rc, rn = random_side(rng, R, 0.05)
    lb = ops.DeviceBatch([dev_col(c, None, n) for c, n in zip(lc, ln)])
    rb = ops.DeviceBatch([dev_col(c, None, n) for c, n in zip(rc, rn)])
    gl, gr = pairs_np(*ops.join_pairs(lb, rb, conds))
    wl, wr = oracle.join_pairs(lc, rc, conds, ln, rn)
    np.testing.assert_array_equal(gl, wl)
    np.testing.assert_array_equal(gr, wr)


def union_pairs(lc, rc, conds, disjunct, ln, rn):
    """Oracle of an OR of ANDs: the union of each group's conjunction pairs,
    in (left, right) order."""
    got = set()
    for g in range(max(disjunct) + 1):
        wl, wr = oracle.join_pairs(lc, rc, [c for c, d in zip(conds, disjunct) if d == g], ln, rn)
        got.update(zip(wl.tolist(), wr.tolist()))
    pairs = sorted(got)
    return (np.array([p[0] for p in pairs], dtype=np.uint32), np.array([p[1] for p in pairs], dtype=np.uint32))


@pytest.mark.parametrize("L,R", [(1, 1), (33, 17), (1025, 300), (3000, 9000)])
@pytest.mark.parametrize("conds,disjunct", [
    ([(0, 0, A.EQ), (1, 1, A.LT)], [0, 1]),                          # a.k = b.k OR a.v < b.v
    ([(0, 0, A.EQ), (2, 2, A.GT), (3, 3, A.EQ)], [0, 0, 1]),         # (k = k AND f > f) OR t = t
    ([(3, 3, A.NE), (1, 1, A.EQ), (0, 0, A.LE), (2, 2, A.LT)], [1, 0, 1, 2]),
])
def test_or_join_pairs_match_union_of_conjunctions(cuda, L, R, conds, disjunct):
    """Join conditions as an OR of ANDs, NULL keys included (a comparison
    with a NULL side does not hold in any group)."""
    rng = np.random.default_rng(L * 7 + R)
    lc, ln = random_side(rng, L, 0.05)
    rc, rn = random_side(rng, R, 0.05)
    lb = ops.DeviceBatch([dev_col(c, None, n) for c, n in zip(lc, ln)])
    rb = ops.DeviceBatch([dev_col(c, None, n) for c, n in zip(rc, rn)])
    gl, gr = pairs_np(*ops.join_pairs(lb, rb, conds, disjunct=disjunct))
    wl, wr = union_pairs(lc, rc, conds, disjunct, ln, rn)
    np.testing.assert_array_equal(gl, wl)
    np.testing.assert_array_equal(gr, wr)
    # the projecting form writes the same pairs' columns
    out = ops.join_project(lb, rb, conds, [(0, 1), (1, 1)], disjunct=disjunct)
    np.testing.assert_array_equal(out.columns[0].data.cpu().numpy(), lc[1][wl])
    np.testing.assert_array_equal(out.columns[1].data.cpu().numpy(), rc[1][wr])


def test_or_join_one_group_is_the_conjunction(cuda):
    rng = np.random.default_rng(5)
    lc, ln = random_side(rng, 2000, 0.05)
    rc, rn = random_side(rng, 700, 0.05)
    lb = ops.DeviceBatch([dev_col(c, None, n) for c, n in zip(lc, ln)])
    rb = ops.DeviceBatch([dev_col(c, None, n) for c, n in zip(rc, rn)])
    conds = [(0, 0, A.EQ), (1, 1, A.LT)]
    a = pairs_np(*ops.join_pairs(lb, rb, conds, disjunct=[0, 0]))
    b = pairs_np(*ops.join_pairs(lb, rb, conds))
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])


def test_or_join_rejects_unused_group(cuda):
    rng = np.random.default_rng(6)
    lc, ln = random_side(rng, 10)
    lb = ops.DeviceBatch([dev_col(c) for c in lc])
    with pytest.raises(A.YQError) as e:
        ops.join_pairs(lb, lb, [(0, 0, A.EQ), (1, 1, A.LT)], disjunct=[0, 2])
    assert e.value.status == A.ERR_INVALID_ARG


_NP_CMP = {A.LT: np.less, A.LE: np.less_equal, A.GT: np.greater, A.GE: np.greater_equal, A.EQ: np.equal,
           A.NE: np.not_equal}


@pytest.mark.parametrize("kind", ["i32", "i64", "f32", "f64", "date"])
@pytest.mark.parametrize("cmp", [A.LT, A.LE, A.GT, A.GE, A.EQ, A.NE])
def test_single_inequality_nested_loop_types(cuda, kind, cmp):
    """One comparison of two null-free columns of the same type (the typed
    nested-loop kernel): right side longer than one shared-memory chunk,
    floats with NaN and signed zeros. IEEE comparisons are the SQL results
    (NaN satisfies only <>, -0.0 equals +0.0)."""
    rng = np.random.default_rng(len(kind) * 7 + cmp)
    L, R = 131, 9_001

    def side(n):
        if kind == "i32":
            return rng.integers(-30, 30, n).astype(np.int32), A.INT32
        if kind in ("i64", "date"):
            return rng.integers(-(1 << 35), 1 << 35, n).astype(np.int64) // (1 << 30), \
                (A.INT64 if kind == "i64" else A.DATETIME)
        dt = np.float32 if kind == "f32" else np.float64
        v = rng.choice(np.array([0.0, -0.0, 1.5, -2.5, np.nan, 3.0], dt), n)
        return v, (A.FLOAT32 if kind == "f32" else A.FLOAT64)

    (x, tx), (y, ty) = side(L), side(R)
    gl, gr = pairs_np(*ops.join_pairs(ops.DeviceBatch([dev_col(x, tx)]), ops.DeviceBatch([dev_col(y, ty)]),
                                      [(0, 0, cmp)]))
    with np.errstate(invalid="ignore"):
        m = _NP_CMP[cmp](x[:, None], y[None, :])
    wl, wr = np.nonzero(m)  # row-major: left ascending, then right ascending
    np.testing.assert_array_equal(gl, wl.astype(np.uint32))
    np.testing.assert_array_equal(gr, wr.astype(np.uint32))


@pytest.mark.parametrize("kind", ["i32", "f32", "i64", "f64"])
@pytest.mark.parametrize("cmp", [A.LT, A.GE, A.EQ, A.NE])
def test_typed_nested_loop_projection_counted(cuda, kind, cmp):
    """Right side long enough that each left row's matches are counted up
    front (the right key sorted once, two binary searches per left row), then
    written in left-major, right-ascending order; outputs are the condition's
    right column (written from the staged value) or another right column."""
    rng = np.random.default_rng(len(kind) * 11 + cmp)
    L, R = 257, 12_345
    if kind in ("i32", "i64"):
        dt = np.int32 if kind == "i32" else np.int64
        x, y = rng.integers(-40, 40, L).astype(dt), rng.integers(-40, 40, R).astype(dt)
    else:
        dt = np.float32 if kind == "f32" else np.float64
        pool = np.array([0.0, -0.0, 1.5, -2.5, np.nan, 3.0, -7.25], dt)
        x, y = rng.choice(pool, L), rng.choice(pool, R)
    z = rng.integers(0, 1 << 30, R).astype(np.int32)
    lb = ops.DeviceBatch([dev_col(x)])
    rb = ops.DeviceBatch([dev_col(y), dev_col(z)])
    with np.errstate(invalid="ignore"):
        m = _NP_CMP[cmp](x[:, None], y[None, :])
    wl, wr = np.nonzero(m)
    out = ops.join_project(lb, rb, [(0, 0, cmp)], [(0, 0), (1, 0)])
    np.testing.assert_array_equal(out.columns[0].data.cpu().numpy().view(x.dtype).view(np.uint8),
                                  x[wl].view(np.uint8))
    np.testing.assert_array_equal(out.columns[1].data.cpu().numpy().view(y.dtype).view(np.uint8),
                                  y[wr].view(np.uint8))
    out2 = ops.join_project(lb, rb, [(0, 0, cmp)], [(1, 1), (0, 0)])
    np.testing.assert_array_equal(out2.columns[0].data.cpu().numpy(), z[wr])
    if len(wl) > 1:
        with pytest.raises(A.YQError) as e:
            ops.join_project(lb, rb, [(0, 0, cmp)], [(0, 0), (1, 0)], capacity=len(wl) // 2)
        assert e.value.status == A.ERR_CAPACITY


def test_join_project_writes_pair_columns(cuda):
    rng = np.random.default_rng(5)
    lc, _ = random_side(rng, 4000)
    rc, _ = random_side(rng, 700)
    lb, rb = dev_batch(lc), dev_batch(rc)
    out = ops.join_project(lb, rb, [(0, 0, A.EQ)], [(0, 1), (1, 3), (1, 2), (0, 0)])
    wl, wr = oracle.join_pairs(lc, rc, [(0, 0, A.EQ)])
    np.testing.assert_array_equal(out.columns[0].data.cpu().numpy(), lc[1][wl])
    np.testing.assert_array_equal(out.columns[1].data.cpu().numpy(), rc[3][wr])
    np.testing.assert_array_equal(out.columns[2].data.cpu().numpy(), rc[2][wr])
    np.testing.assert_array_equal(out.columns[3].data.cpu().numpy(), lc[0][wl])


@pytest.mark.parametrize("n", [1, 100, 2000])
def test_cross_product_with_predicate(cuda, n):
    x, y = datagen.cross_tables(n, seed=2)
    out = ops.join_project(dev_batch([x]), dev_batch([y]), [(0, 0, A.LT)], [(0, 0), (1, 0)])
    wx, wy, cnt = oracle.cross_lt(x, y)
    assert out.rows == cnt
    np.testing.assert_array_equal(out.columns[0].data.cpu().numpy(), wx)
    np.testing.assert_array_equal(out.columns[1].data.cpu().numpy(), wy)


def test_plain_cross_product_left_major(cuda):
    rng = np.random.default_rng(9)
    a = rng.integers(0, 100, 37).astype(np.int32)
    t = datagen.text_slots(["x", "yy", "zzz"])
    b = np.array([1.5, -2.0, 3.25], np.float32)
    out = ops.cross_product(dev_batch([a]), dev_batch([t, b]))
    assert out.rows == 37 * 3
    np.testing.assert_array_equal(out.columns[0].data.cpu().numpy(), np.repeat(a, 3))
    np.testing.assert_array_equal(out.columns[1].data.cpu().numpy(), np.tile(t, (37, 1)))
    np.testing.assert_array_equal(out.columns[2].data.cpu().numpy(), np.tile(b, 37))


def test_join_capacity_reported(cuda):
    a = np.zeros(1000, np.int32)
    lb, rb = dev_batch([a]), dev_batch([a[:100]])
    with pytest.raises(A.YQError) as e:
        ops.join_pairs(lb, rb, [(0, 0, A.EQ)], capacity=5000)
    assert e.value.status == A.ERR_CAPACITY


def star_exprs(year=1993):
    qty, disc, price = ColumnRef(1, A.INT32), ColumnRef(2, A.INT32), ColumnRef(3, A.FLOAT32)
    fact_pred = And(between(disc, Constant(1, A.INT32), Constant(3, A.INT32)),
                    Compare(A.LT, qty, Constant(25, A.INT32)))
    dim_pred = Compare(A.EQ, ColumnRef(1, A.INT32), Constant(year, A.INT32))
    aggs = [Aggregate(A.AGG_SUM, Arith(A.MUL, price, Cast(disc, A.FLOAT32))), Aggregate(A.AGG_COUNT_STAR)]
    return fact_pred, dim_pred, aggs


@pytest.mark.parametrize("rows", [1, 4097, 2_000_000])
def test_star_join_aggregate(cuda, rows):
    fact, dim = datagen.star_tables(rows, seed=2)
    fb = dev_batch([fact["datekey"], fact["quantity"], fact["discount"], fact["extendedprice"]])
    db = dev_batch([dim["datekey"], dim["year"], dim["month"]])
    fp, dp, aggs = star_exprs()
    plan = ops.JoinAggPlan([A.INT32, A.INT32, A.INT32, A.FLOAT32], [A.INT32] * 3, fp, 0, dp, 0, aggs)
    st = ops.AggState(aggs)
    plan.run(fb, db, st)
    got = st.read()
    s, c = oracle.star_query(fact, dim, 1993)
    assert got[1] == c
    assert rel_close(got[0], s if c else None, 1e-6) or (c == 0 and got[0] is None)


def test_star_join_rejects_repeated_dimension_keys(cuda):
    fact, dim = datagen.star_tables(1000, seed=2)
    dk = dim["datekey"].copy()
    dk[1] = dk[0]
    fb = dev_batch([fact["datekey"], fact["quantity"], fact["discount"], fact["extendedprice"]])
    db = dev_batch([dk, dim["year"], dim["month"]])
    fp, _, aggs = star_exprs()
    plan = ops.JoinAggPlan([A.INT32, A.INT32, A.INT32, A.FLOAT32], [A.INT32] * 3, fp, 0, None, 0, aggs)
    with pytest.raises(A.YQError) as e:
        plan.run(fb, db, ops.AggState(aggs))
    assert e.value.status == A.ERR_UNSUPPORTED


@pytest.mark.parametrize("rows", [1, 4097, 3_000_000])
def test_star_join_prepared_dimension(cuda, rows):
    """The dimension side built once (yq_join_dim_table_build) and probed by
    several aggregates with no host synchronisation: the same result as the
    one-call join and the oracle, on every repetition."""
    fact, dim = datagen.star_tables(rows, seed=3)
    fb = dev_batch([fact["datekey"], fact["quantity"], fact["discount"], fact["extendedprice"]])
    db = dev_batch([dim["datekey"], dim["year"], dim["month"]])
    fp, dp, aggs = star_exprs(1994)
    plan = ops.JoinAggPlan([A.INT32, A.INT32, A.INT32, A.FLOAT32], [A.INT32] * 3, fp, 0, dp, 0, aggs)
    prep = plan.prepare(db)
    assert prep.kept == int((dim["year"] == 1994).sum())
    s, c = oracle.star_query(fact, dim, 1994)
    one = ops.AggState(aggs)
    plan.run(fb, db, one)
    want = one.read()
    for _ in range(3):
        st = ops.AggState(aggs)
        plan.run_prepared(fb, prep, st)
        got = st.read()
        assert got[1] == c == want[1]
        assert rel_close(got[0], want[0], 1e-9) or (c == 0 and got[0] is None)
        assert rel_close(got[0], s if c else None, 1e-6) or (c == 0 and got[0] is None)
