"""Out-of-core ORDER BY parity: runs (4 MB-batch segments) sorted, then
merged pairwise by the merge-path kernel, must equal one stable sort of the
whole table (ties take the earlier run, order_operator.cpp:117-220 /
merge_batchs.cu:61)."""
import numpy as np
import pytest

import oracle
from yallasql_b200 import _abi as A
from yallasql_b200 import datagen, ops

from helpers import dev_col

pytestmark = pytest.mark.gpu


def table_batch(t):
    return ops.DeviceBatch([dev_col(t["key"]), dev_col(t["id"]), dev_col(t["txt"]), dev_col(t["d"], A.DATETIME)])


def out_like(b):
    return ops.DeviceBatch([ops.DeviceColumn.empty(c.type, c.rows, c.width if c.type == A.TEXT else None,
                                                   nulls=c.nulls is not None) for c in b.columns])


def run_outofcore(b, key, desc, offsets):
    perm = ops.sort_segments(b.columns[key], offsets, desc)
    runs = ops.gather(b, perm)
    out = out_like(b)
    ops.merge_runs(runs, key, desc, offsets, out)
    return out


@pytest.mark.parametrize("dist", ["uniform", "zipf", "equal"])
@pytest.mark.parametrize("batch", [116_480, 5_000, 777])
def test_outofcore_order_by_equals_stable_sort(cuda, dist, batch):
    rows = 300_000
    t = datagen.order_table(rows, seed=1, dist=dist)
    b = table_batch(t)
    counts = [batch] * (rows // batch) + ([rows % batch] if rows % batch else [])
    offs = list(np.concatenate([[0], np.cumsum(counts)]).astype(int))
    for key, name, desc, ty in ((0, "key", True, None), (3, "d", False, oracle.DATETIME)):
        out = run_outofcore(b, key, desc, offs)
        perm = oracle.sort_perm(t[name], desc=desc, type_=ty)
        for col, n in zip(out.columns, ["key", "id", "txt", "d"]):
            np.testing.assert_array_equal(col.data.cpu().numpy(), t[n][perm])


@pytest.mark.parametrize("dist", ["uniform", "zipf", "equal"])
@pytest.mark.parametrize("batch", [116_480, 3_001, 300_000])
def test_order_by_runs_key_id_path(cuda, dist, batch):
    """Runs sorted, (key, row id) merged, payload gathered once: same table as one stable sort."""
    rows = 250_000
    t = datagen.order_table(rows, seed=2, dist=dist)
    b = table_batch(t)
    counts = [batch] * (rows // batch) + ([rows % batch] if rows % batch else [])
    offs = list(np.concatenate([[0], np.cumsum(counts)]).astype(int))
    for key, name, desc, ty in ((0, "key", True, None), (3, "d", False, oracle.DATETIME)):
        job = ops.OrderByRuns(b, key, offs)
        out = out_like(b)
        for _ in range(2):  # buffers are reused across calls
            job.run(b, desc, out)
            perm = oracle.sort_perm(t[name], desc=desc, type_=ty)
            for col, n in zip(out.columns, ["key", "id", "txt", "d"]):
                np.testing.assert_array_equal(col.data.cpu().numpy(), t[n][perm])


@pytest.mark.parametrize("dist", ["uniform", "zipf", "equal"])
@pytest.mark.parametrize("two_level", [True, False])
def test_order_by_runs_two_level_gather(cuda, dist, two_level):
    """A table above the two-level threshold (2.1M rows x 36 bytes): the
    columns go through the sorted-run copy, or not when the workspace only
    holds the one-level minimum; both equal one stable sort."""
    rows = 2_100_003
    t = datagen.order_table(rows, seed=4, dist=dist)
    b = table_batch(t)
    batch = 116_480
    counts = [batch] * (rows // batch) + ([rows % batch] if rows % batch else [])
    offs = list(np.concatenate([[0], np.cumsum(counts)]).astype(int))
    assert (ops.order_by_batch_workspace_bytes(b, 0, offs) > ops.order_by_workspace_bytes(b.columns[0], offs))
    for key, name, desc, ty in ((0, "key", True, None), (3, "d", False, oracle.DATETIME)):
        job = ops.OrderByRuns(b, key, offs, two_level=two_level)
        out = out_like(b)
        job.run(b, desc, out)
        perm = oracle.sort_perm(t[name], desc=desc, type_=ty)
        for col, n in zip(out.columns, ["key", "id", "txt", "d"]):
            np.testing.assert_array_equal(col.data.cpu().numpy(), t[n][perm])


@pytest.mark.parametrize("nruns", [1, 2, 3, 8, 13])
@pytest.mark.parametrize("kind", ["i32", "i64", "text16", "f32_nulls"])
def test_merge_pass_types(cuda, nruns, kind):
    rng = np.random.default_rng(nruns * 7 + len(kind))
    sizes = rng.integers(0, 9000, nruns)
    sizes[0] = max(sizes[0], 1)
    n = int(sizes.sum())
    offs = [0] + list(np.cumsum(sizes).astype(int))
    nulls = None
    if kind == "i32":
        k = rng.integers(-20, 20, n).astype(np.int32)
    elif kind == "i64":
        k = rng.integers(-(1 << 40), 1 << 40, n).astype(np.int64)
    elif kind == "text16":
        k = datagen.text_slots([["", "a", "ab", "b", "zz", "hello"][j] for j in rng.integers(0, 6, n)])
    else:
        k = rng.normal(0, 10, n).astype(np.float32)
        nulls = rng.random(n) < 0.2
    payload = np.arange(n, dtype=np.int64)
    b = ops.DeviceBatch([dev_col(k, None, nulls), dev_col(payload)])
    for desc in (False, True):
        out = run_outofcore(b, 0, desc, offs)
        perm = oracle.sort_perm(k, desc=desc, nulls=nulls)
        np.testing.assert_array_equal(out.columns[1].data.cpu().numpy(), payload[perm])


@pytest.mark.parametrize("nruns", [1, 2, 5, 16])
@pytest.mark.parametrize("kind", ["f32", "i32", "i64", "date", "f64", "text16", "text32", "f32_nulls", "bool",
                                  "equal", "f32_special", "bool_bytes"])
@pytest.mark.parametrize("desc,nulls_first", [(False, False), (True, False), (True, True)])
def test_order_by_entry_matches_stable_sort(cuda, nruns, kind, desc, nulls_first):
    """yq_order_by over runs of random sizes (empty runs included): every column
    equals the rows of one stable sort of the whole table."""
    rng = np.random.default_rng(nruns * 31 + len(kind) + 7 * desc + nulls_first)
    sizes = rng.integers(0, 6000, nruns)
    if nruns > 2:
        sizes[1] = 0
    n = int(sizes.sum())
    offs = [0] + list(np.cumsum(sizes).astype(int))
    nulls = None
    ty = None
    if kind == "f32":
        k, t = rng.uniform(-1e6, 1e6, n).astype(np.float32), A.FLOAT32
    elif kind == "i32":
        k, t = rng.integers(-50, 50, n).astype(np.int32), A.INT32
    elif kind == "i64":
        k, t = rng.integers(-(1 << 40), 1 << 40, n).astype(np.int64), A.INT64
    elif kind == "date":
        k, t, ty = rng.integers(1420070400, 1640995199, n).astype(np.int64), A.DATETIME, oracle.DATETIME
    elif kind == "f64":
        k, t = rng.normal(0, 1e3, n).astype(np.float64), A.FLOAT64
    elif kind == "text16":
        k, t = datagen.text_slots([["", "a", "ab", "b", "zz", "hello", "category_007"][j]
                                   for j in rng.integers(0, 7, n)]), A.TEXT
    elif kind == "text32":
        k = np.zeros((n, 32), np.uint8)
        k[:, :20] = rng.integers(97, 100, (n, 20))
        t = A.TEXT
    elif kind == "f32_nulls":
        k, t = rng.normal(0, 10, n).astype(np.float32), A.FLOAT32
        nulls = rng.random(n) < 0.2
    elif kind == "bool":
        k, t = (rng.random(n) < 0.5).astype(np.uint8), A.BOOL
    elif kind == "f32_special":
        # -0.0 ties +0.0 and NaNs sort last: the key column must still come out bit for bit
        k = rng.choice(np.array([0.0, -0.0, 1.5, -2.5], np.float32), n)
        bits = k.view(np.uint32)
        bits[rng.random(n) < 0.05] = 0x7fc00000
        bits[rng.random(n) < 0.05] = 0x7f800001
        bits[rng.random(n) < 0.05] = 0xffc00000
        t = A.FLOAT32
    elif kind == "bool_bytes":
        k, t = rng.integers(0, 4, n).astype(np.uint8), A.BOOL
    else:
        k, t = np.full(n, 3.5, np.float32), A.FLOAT32
    payload = np.arange(n, dtype=np.int64)
    txt = datagen.text_slots([f"r{i % 97}" for i in range(n)])
    b = ops.DeviceBatch([dev_col(k, t, nulls), dev_col(payload), dev_col(txt, A.TEXT)])
    out = ops.order_by(b, 0, desc, offs, nulls_first=nulls_first)
    perm = oracle.sort_perm(k, desc=desc, nulls=nulls, nulls_first=nulls_first, type_=ty)
    np.testing.assert_array_equal(out.columns[1].data.cpu().numpy(), payload[perm])
    got = out.columns[0].data.cpu().numpy()
    np.testing.assert_array_equal(got.view(np.uint8), k[perm].view(np.uint8))  # bit for bit
    np.testing.assert_array_equal(out.columns[2].data.cpu().numpy(), txt[perm])
    if nulls is not None:
        np.testing.assert_array_equal(out.columns[0].nulls.cpu().numpy().astype(bool), nulls[perm])


@pytest.mark.parametrize("merge_items", [4, 8, 16])
@pytest.mark.parametrize("kind", ["f32", "i64", "text32", "f32_nulls"])
def test_order_by_every_merge_tile(cuda, merge_items, kind):
    """yq_order_by_tiled: every merge-path tile (4, 8 or 16 outputs per thread)
    gives the stable sort; 16 is refused for keys wider than two words."""
    rng = np.random.default_rng(merge_items * 13 + len(kind))
    sizes = rng.integers(1, 40_000, 9)
    n = int(sizes.sum())
    offs = [0] + list(np.cumsum(sizes).astype(int))
    nulls = None
    if kind == "f32":
        k, t = rng.integers(-300, 300, n).astype(np.float32), A.FLOAT32
    elif kind == "i64":
        k, t = rng.integers(-(1 << 40), 1 << 40, n).astype(np.int64), A.INT64
    elif kind == "text32":
        k = np.zeros((n, 32), np.uint8)
        k[:, :20] = rng.integers(97, 100, (n, 20))
        t = A.TEXT
    else:
        k, t = rng.normal(0, 10, n).astype(np.float32), A.FLOAT32
        nulls = rng.random(n) < 0.2
    payload = np.arange(n, dtype=np.int64)
    b = ops.DeviceBatch([dev_col(k, t, nulls), dev_col(payload)])
    if kind == "text32" and merge_items == 16:
        with pytest.raises(A.YQError) as e:
            ops.order_by(b, 0, True, offs, merge_items=merge_items)
        assert e.value.status == A.ERR_UNSUPPORTED
        return
    out = ops.order_by(b, 0, True, offs, merge_items=merge_items)
    perm = oracle.sort_perm(k, desc=True, nulls=nulls)
    np.testing.assert_array_equal(out.columns[1].data.cpu().numpy(), payload[perm])


def test_order_by_autotune_then_order_by(cuda):
    """The tuner returns a sort variant and a merge tile; later yq_order_by
    calls on that shape use them and still give the stable sort."""
    rows = 600_000
    t = datagen.order_table(rows, seed=9, dist="zipf")
    b = table_batch(t)
    offs = list(range(0, rows, 116_480)) + [rows]
    best, items = ops.order_by_autotune(b, 0, True, offs)
    assert best.digit_bits in (4, 6, 8) and best.block_threads in (128, 256, 512) and items in (4, 8, 16)
    out = ops.order_by(b, 0, True, offs)
    perm = oracle.sort_perm(t["key"], desc=True)
    for col, n in zip(out.columns, ["key", "id", "txt", "d"]):
        np.testing.assert_array_equal(col.data.cpu().numpy(), t[n][perm])
