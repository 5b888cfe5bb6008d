"""GROUP BY on the B200 (yq_group_by) against the numpy oracle: every key
type (with NULL keys, -0.0/+0.0 and NaN for floats), every aggregate over
every numeric input type with NULL inputs, few and many groups, and the
capacity error. Integers, counts, MIN/MAX and keys bit-exact; float SUM/AVG
(FP64) within 1e-9 relative."""
import numpy as np
import pytest
import torch

import oracle
from yallasql_b200 import _abi as A
from yallasql_b200 import datagen, ops

pytestmark = pytest.mark.gpu

ORC_TYPE = {A.INT32: 0, A.FLOAT32: 1, A.DATETIME: 2, A.TEXT: 3, A.INT64: 4, A.FLOAT64: 5}


def dcol(v, t, nulls=None):
    d = torch.from_numpy(np.ascontiguousarray(v)).cuda()
    return ops.DeviceColumn(d, t, None if nulls is None else torch.from_numpy(nulls.astype(np.uint8)).cuda())


def check(batch_np, key, aggs):
    """batch_np: list of (values, type, nulls|None)."""
    b = ops.DeviceBatch([dcol(v, t, n) for v, t, n in batch_np])
    got = ops.group_by(b, key, aggs)
    kv, kt, kn = batch_np[key]
    ok, okn, res = oracle.group_by(kv, kn, ORC_TYPE[kt], [
        (k, None if k == A.AGG_COUNT_STAR else batch_np[c][0], None if k == A.AGG_COUNT_STAR else batch_np[c][2],
         ORC_TYPE[batch_np[c][1]] if k != A.AGG_COUNT_STAR else 4) for k, c in aggs])
    g = got.columns[0]
    assert g.rows == len(ok)
    gkn = g.nulls.cpu().numpy().astype(bool)
    assert np.array_equal(gkn, okn)
    gk = g.data.cpu().numpy()
    assert gk[~gkn].tobytes() == np.ascontiguousarray(ok[~okn]).tobytes()
    for j, ((kind, col), (want, wnull)) in enumerate(zip(aggs, res)):
        c = got.columns[1 + j]
        v = c.data.cpu().numpy()
        if wnull is not None:
            gn = c.nulls.cpu().numpy().astype(bool)
            assert np.array_equal(gn, wnull)
            v, want = v[~wnull], np.asarray(want)[~wnull]
        if kind in (A.AGG_SUM, A.AGG_AVG) and c.type == A.FLOAT64:
            np.testing.assert_allclose(v, want, rtol=1e-9, atol=1e-9)
        else:
            assert v.tobytes() == np.ascontiguousarray(np.asarray(want).astype(v.dtype)).tobytes()


ALL_AGGS = lambda cols: [(A.AGG_COUNT_STAR, 0)] + [(k, c) for c in cols for k in
                                                   (A.AGG_COUNT, A.AGG_SUM, A.AGG_AVG, A.AGG_MIN, A.AGG_MAX)]


@pytest.mark.parametrize("ktype", [A.INT32, A.INT64, A.DATETIME, A.FLOAT32, A.FLOAT64, A.TEXT])
def test_key_types_and_aggregates(cuda, ktype):
    rng = np.random.default_rng(ktype + 50)
    n = 20_000
    if ktype == A.INT32:
        k = rng.integers(-40, 40, n).astype(np.int32)
    elif ktype in (A.INT64, A.DATETIME):
        k = (rng.integers(-50, 50, n) * (1 << 33)).astype(np.int64)
    elif ktype in (A.FLOAT32, A.FLOAT64):
        dt = np.float32 if ktype == A.FLOAT32 else np.float64
        k = rng.choice(np.array([0.0, -0.0, 1.5, -2.25, np.nan, np.inf, -np.inf, 3.0], dt), n)
    else:
        k = datagen.text_slots([f"g{int(x):03d}" for x in rng.integers(0, 60, n)], 12)
    kn = rng.random(n) < 0.05
    i32 = rng.integers(-1000, 1000, n).astype(np.int32)
    f32 = rng.normal(0, 100, n).astype(np.float32)
    i64 = rng.integers(-(1 << 40), 1 << 40, n).astype(np.int64)
    f64 = rng.normal(0, 1e6, n)
    cols = [(k, ktype, kn), (i32, A.INT32, rng.random(n) < 0.1), (f32, A.FLOAT32, rng.random(n) < 0.1),
            (i64, A.INT64, None), (f64, A.FLOAT64, rng.random(n) < 0.3)]
    for c in (1, 2, 3, 4):  # one input column a call: COUNT(*) + five aggregates (the limit is 8)
        check(cols, 0, ALL_AGGS([c]))


def test_all_null_inputs_and_single_group(cuda):
    n = 1000
    k = np.zeros(n, np.int32)
    v = np.arange(n, dtype=np.float32)
    check([(k, A.INT32, None), (v, A.FLOAT32, np.ones(n, bool))], 0, ALL_AGGS([1]))
    d = np.arange(n, dtype=np.int64) * 86400
    check([(k, A.INT32, None), (d, A.DATETIME, None)], 0, [(A.AGG_MIN, 1), (A.AGG_MAX, 1), (A.AGG_COUNT, 1)])


@pytest.mark.parametrize("rows,key", [(4_000_000, "discount"), (4_000_000, "qty"), (2_000_000, "id")])
def test_sales_table_group_by(cuda, rows, key):
    t = datagen.sales_table(rows, seed=6)
    kcol = {"discount": (t["discount"], A.INT32), "qty": (t["qty"], A.INT32),
            "id": ((t["id"] % 700_000).astype(np.int64), A.INT64)}[key]
    cols = [(kcol[0], kcol[1], None), (t["price"], A.FLOAT32, None), (t["qty"], A.INT32, None)]
    check(cols, 0, [(A.AGG_COUNT_STAR, 0), (A.AGG_SUM, 1), (A.AGG_AVG, 2), (A.AGG_MIN, 1), (A.AGG_MAX, 1),
                    (A.AGG_SUM, 2)])


def test_capacity_error(cuda):
    k = np.arange(100, dtype=np.int32) % 10
    b = ops.DeviceBatch([dcol(k, A.INT32)])
    with pytest.raises(A.YQError) as e:
        ops.group_by(b, 0, [(A.AGG_COUNT_STAR, 0)], capacity=5)
    assert e.value.status == A.ERR_CAPACITY
    got = ops.group_by(b, 0, [(A.AGG_COUNT_STAR, 0)], capacity=10)
    assert got.columns[0].data.cpu().tolist() == list(range(10))
    assert got.columns[1].data.cpu().tolist() == [10] * 10


@pytest.mark.parametrize("layout", ["one_group", "tile_edges", "short_groups"])
def test_tiles_inside_one_group(cuda, layout):
    """Tiles of 2,048 sorted positions that lie inside one group fold it with
    a block reduction: one group over ~500 tiles; groups whose boundaries
    fall exactly on tile edges; groups shorter than a tile. NULL inputs."""
    rng = np.random.default_rng(len(layout))
    n = 1_000_000
    if layout == "one_group":
        k = np.full(n, 7, np.int32)
    elif layout == "tile_edges":
        k = (np.arange(n) // (2048 * 3)).astype(np.int32)  # every group ends on a tile edge
        k = rng.permutation(k)
    else:
        k = rng.integers(0, 3000, n).astype(np.int32)
    v = rng.normal(0, 100, n).astype(np.float32)
    vn = rng.random(n) < 0.05
    q = rng.integers(-1000, 1000, n).astype(np.int64)
    check([(k, A.INT32, None), (v, A.FLOAT32, vn), (q, A.INT64, None)], 0,
          ALL_AGGS([1]) + [(A.AGG_SUM, 2), (A.AGG_MIN, 2)])  # eight aggregates, the most a call takes
