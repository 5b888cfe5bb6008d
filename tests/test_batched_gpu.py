"""Batched form parity: many tasks in a handful of launches (segmented
filter+aggregate, segmented ORDER BY, CUDA-graph replay) give every task the
same result as running it alone, and the oracle's."""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle
from yallasql_b200 import _abi as A
from yallasql_b200 import batched, datagen, ops

pytestmark = pytest.mark.gpu

REL = 1e-6  # float SUM/AVG tolerance (summation order); everything else exact


def check_agg(got, want):
    assert got[1] == want[1]            # COUNT(*)
    if want[1] == 0:
        assert got[0] is None and got[2] is None and got[3] is None
        return
    assert got[2] == want[2] and got[3] == want[3]  # MIN, MAX (float32 values, exact)
    assert abs(got[0] - want[0]) <= REL * max(1.0, abs(want[0]))


@pytest.mark.parametrize("graph", [False, True])
def test_batched_equals_plain_and_oracle(cuda, graph):
    rows = batched.task_rows(24, seed=3, lo=50, hi=40_000)
    ts = batched.TaskSet(rows, seed=3, on_device=False)
    hf, hs = ts.host
    plain = batched.PlainRunner(ts)
    plain.run()
    pres = plain.results()
    pipe = batched.BatchedPipeline(ts, graph=graph)
    for _ in range(2):  # replays reuse every buffer
        pipe.run()
        torch.cuda.synchronize()
        assert pipe.error_word() == 0
        bres = pipe.results()
        for g, (a, b) in enumerate(zip(ts.foffs[:-1], ts.foffs[1:])):
            sl = {k: hf[k][a:b] for k in ("price", "qty", "discount", "category")}
            want = oracle.sales_query(sl, datagen.EXCLUDED_CATEGORY.encode())
            want = [want[0], want[1], want[2], want[3]]
            check_agg(bres[g], want)
            check_agg(pres[g], want)
            assert bres[g][1:] == pres[g][1:]
        names = ["id", "price", "qty", "discount", "category", "updated_at"]
        for g, (a, b) in enumerate(zip(ts.soffs[:-1], ts.soffs[1:])):
            perm = oracle.sort_perm(hs["price"][a:b], desc=True)
            for ci, name in enumerate(names):
                got = ts.sout.columns[ci].data[a:b].cpu().numpy()
                np.testing.assert_array_equal(got, hs[name][a:b][perm])
                np.testing.assert_array_equal(ts.souts[g].columns[ci].data.cpu().numpy(), got)


def test_segments_edge_tasks(cuda):
    """Empty tasks, single rows, unaligned starts and tasks spanning step windows."""
    sizes = [0, 1, 17, 1023, 1024, 1025, 0, 3000, 5, 2048]
    offs = [0] + list(np.cumsum(sizes).astype(int))
    t = datagen.sales_table(offs[-1], seed=9)
    b = ops.DeviceBatch([ops.DeviceColumn(torch.from_numpy(np.ascontiguousarray(t[k])).cuda(), ty) for k, ty in
                         zip(["price", "qty", "discount", "category"], [A.FLOAT32, A.INT32, A.INT32, A.TEXT])])
    pred, aggs = batched.sales_query()
    plan = ops.AggPlan([A.FLOAT32, A.INT32, A.INT32, A.TEXT], pred, aggs)
    st = ops.AggStates(aggs, len(sizes))
    plan.run_segments(b, offs, st)
    res = st.read()
    for g, (a, e) in enumerate(zip(offs[:-1], offs[1:])):
        sl = {k: t[k][a:e] for k in ("price", "qty", "discount", "category")}
        w = oracle.sales_query(sl, datagen.EXCLUDED_CATEGORY.encode())
        check_agg(res[g], [w[0], w[1], w[2], w[3]])
    # ORDER BY segments with the same sizes
    key = np.random.default_rng(4).normal(0, 5, offs[-1]).astype(np.float32)
    pay = np.arange(offs[-1], dtype=np.int64)
    sb = ops.DeviceBatch([ops.DeviceColumn(torch.from_numpy(key).cuda(), A.FLOAT32),
                          ops.DeviceColumn(torch.from_numpy(pay).cuda(), A.INT64)])
    out = ops.DeviceBatch([ops.DeviceColumn.empty(A.FLOAT32, offs[-1]), ops.DeviceColumn.empty(A.INT64, offs[-1])])
    ops.order_by_segments(sb, 0, False, offs, out)
    perm = oracle.sort_perm(key, segments=offs)
    np.testing.assert_array_equal(out.columns[1].data.cpu().numpy(), pay[perm])


def test_sort_autotune_choice_is_used(cuda):
    rng = np.random.default_rng(5)
    key = rng.uniform(-1e6, 1e6, 300_000).astype(np.float32)
    col = ops.DeviceColumn(torch.from_numpy(key).cuda(), A.FLOAT32)
    offs = [0, 100_000, 300_000]
    best = ops.sort_autotune(col, offs, descending=True)
    assert best.digit_bits in (4, 6, 8) and best.items_per_thread in (8, 12, 16)
    assert best.block_threads in (128, 256, 512)
    perm = ops.sort_segments(col, offs, True, config=ops.sort_config(digit_bits=0))
    np.testing.assert_array_equal(perm.cpu().numpy().astype(np.int64), oracle.sort_perm(key, desc=True, segments=offs))


@pytest.mark.parametrize("variant", [(8, 8, 512), (8, 12, 512), (6, 16, 128), (4, 16, 128), (8, 12, 256),
                                     (6, 16, 256)])
@pytest.mark.parametrize("kind", ["f32", "i64", "f32_nulls"])
def test_every_block_size_variant(cuda, variant, kind):
    """Each instantiated (digit bits, items per thread, block threads) sort
    variant, asked for explicitly, gives the stable segmented sort; a variant
    that is not instantiated for the key width falls back to 8-bit digits."""
    d, items, block = variant
    rng = np.random.default_rng(d * 100 + items + block)
    n = 250_003
    nulls = None
    if kind == "f32":
        key = rng.integers(-5000, 5000, n).astype(np.float32)
    elif kind == "i64":
        key = rng.integers(-(1 << 40), 1 << 40, n).astype(np.int64)
    else:
        key = rng.normal(0, 1, n).astype(np.float32)
        nulls = rng.random(n) < 0.1
    col = ops.DeviceColumn(torch.from_numpy(key).cuda(), A.FLOAT32 if key.dtype == np.float32 else A.INT64,
                           None if nulls is None else torch.from_numpy(nulls.astype(np.uint8)).cuda())
    offs = [0, 7, 100_000, 100_000, 250_003]
    cfg = ops.sort_config(digit_bits=d, items_per_thread=items, block_threads=block)
    perm = ops.sort_segments(col, offs, True, config=cfg)
    want = oracle.sort_perm(key, desc=True, nulls=nulls, segments=offs)
    np.testing.assert_array_equal(perm.cpu().numpy().astype(np.int64), want)


def test_block_threads_validated(cuda):
    key = np.arange(1000, dtype=np.float32)
    col = ops.DeviceColumn(torch.from_numpy(key).cuda(), A.FLOAT32)
    with pytest.raises(A.YQError) as e:
        ops.sort_segments(col, [0, 1000], False, config=ops.sort_config(block_threads=96))
    assert e.value.status == A.ERR_INVALID_ARG
