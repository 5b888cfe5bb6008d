"""Parity at the benchmark configurations' full sizes.

The throughput figures are measured on a 64M-row ORDER BY table (three key
distributions), a 60M-row star join and a 20K x 20K cross product; these
tests run the same calls on the same inputs and compare every output with the
oracle, so nothing the benchmark times is left unchecked at its own size.

- ORDER BY: `bench.OrderByJob` in its out-of-core mode (the reference's plan,
  src/engine/operators/order_operator.cpp:117-220: 4 MB batches sorted into
  550 runs of 116,480 rows, merged pairwise by merge path, ties to the earlier
  run as in src/kernels/merge_batchs.cu:61), `ORDER BY key DESC` and
  `ORDER BY d ASC`, every column compared with the oracle's stable sort
  followed by a gather.
- Star join: the 60M-row fact table joined with the date dimension,
  SUM(extendedprice * discount) and COUNT(*) against `oracle.star_query`.
- Cross product: 20K x 20K with `a.x < b.y`, every output pair compared with
  `oracle.cross_lt` (left-major, right ascending).
"""
import os

import numpy as np
import pytest

import oracle
from yallasql_b200 import _abi as A
from yallasql_b200 import datagen, ops

from helpers import dev_batch, rel_close

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1
ORDER_ROWS = 64_000_000


@pytest.mark.parametrize("dist", ["uniform", "zipf", "equal"])
def test_order_by_64M_outofcore_equals_oracle(cuda, dist):
    import bench
    import torch
    t = datagen.order_table(ORDER_ROWS, seed=1, dist=dist)
    job = bench.OrderByJob(t, "outofcore")
    assert len(job.batch_rows) == 550 and job.batch_rows[0] == 116_480
    a, b = job.step()
    torch.cuda.synchronize()
    for out, name, desc, ty in ((a, "key", True, None), (b, "d", False, oracle.DATETIME)):
        perm = oracle.sort_perm(t[name], desc=desc, threads=THREADS, type_=ty)
        for col, n in zip(out.columns, ("key", "id", "txt", "d")):
            got = col.data.cpu().numpy()
            want = np.take(t[n], perm, axis=0)
            assert np.array_equal(got, want), f"ORDER BY {name}: column {n} differs from the oracle ({dist})"
        del perm
    del job


def test_star_join_aggregate_60M(cuda):
    from test_join_gpu import star_exprs
    fact, dim = datagen.star_tables(60_000_000, seed=2)
    fb = dev_batch([fact["datekey"], fact["quantity"], fact["discount"], fact["extendedprice"]])
    db = dev_batch([dim["datekey"], dim["year"], dim["month"]])
    fp, dp, aggs = star_exprs()
    plan = ops.JoinAggPlan([A.INT32, A.INT32, A.INT32, A.FLOAT32], [A.INT32] * 3, fp, 0, dp, 0, aggs)
    st = ops.AggState(aggs)
    plan.run(fb, db, st)
    got = st.read()
    s, c = oracle.star_query(fact, dim, 1993, threads=THREADS)
    assert c > 1_000_000
    assert got[1] == c
    assert rel_close(got[0], s, 1e-6), (got[0], s)


def test_cross_product_lt_20K_by_20K(cuda):
    x, y = datagen.cross_tables(20_000, seed=2)
    out = ops.join_project(dev_batch([x]), dev_batch([y]), [(0, 0, A.LT)], [(0, 0), (1, 0)])
    wx, wy, cnt = oracle.cross_lt(x, y)
    assert cnt > 190_000_000
    assert out.rows == cnt
    gx = out.columns[0].data.cpu().numpy()
    assert np.array_equal(gx, wx), "cross product left column differs from the oracle"
    del gx, wx
    gy = out.columns[1].data.cpu().numpy()
    assert np.array_equal(gy, wy), "cross product right column differs from the oracle"
