"""CSV scan on the B200 (yq_csv_index + yq_csv_parse through ops.csv_scan)
against the oracle's restatement of the reference's reader, bit-exact: record
splitting, rows dropped for a wrong field count, NULL cells and sentinels,
int/float/date/text values (float bits, NaN payloads, text slots) and the
cells the reference's std::stoi / std::stof would reject."""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle
from oracle import expr_eval
from tests import csv_cases
from yallasql_b200 import _abi as A
from yallasql_b200 import datagen, ops
from yallasql_b200.expr import Aggregate, And, Arith, Cast, ColumnRef, Compare, Constant, between

pytestmark = pytest.mark.gpu


def gpu_scan(body: bytes, types, width=16, offset=0):
    proj = [f for f, t in enumerate(types) if t >= 0]
    full = [t if t >= 0 else A.TEXT for t in types]
    host = torch.zeros(len(body) + offset + 16, dtype=torch.uint8)
    if body:
        host[offset:offset + len(body)] = torch.frombuffer(bytearray(body), dtype=torch.uint8)
    text = host.cuda()[offset:offset + len(body)]
    err = None
    try:
        batch = ops.csv_scan(text, full, proj, width)
    except ops.CsvScanError as e:
        batch, err = e.batch, e.error
    torch.cuda.synchronize()
    cols, k = [], 0
    for t in types:
        if t < 0:
            cols.append(None)
            continue
        c = batch.columns[k]
        k += 1
        cols.append((c.data.cpu().numpy(), c.nulls.cpu().numpy()))
    rows = batch.columns[0].rows if batch.columns else 0
    meta = (err.bad_cells, err.first_row, err.first_field, err.kind) if err else (0, -1, -1, 0)
    return {"rows": rows, "bad": meta[0], "first_row": meta[1], "first_field": meta[2], "first_kind": meta[3],
            "cols": cols}


def same(g, o):
    assert (g["rows"], g["bad"], g["first_row"], g["first_field"], g["first_kind"]) == \
        (o["rows"], o["bad"], o["first_row"], o["first_field"], o["first_kind"])
    for x, y in zip(g["cols"], o["cols"]):
        if x is None:
            continue
        assert np.array_equal(x[1], y[1]), "null bytes"
        assert x[0].tobytes() == y[0].tobytes(), "values"


def test_edge_cases(cuda):
    for types, header, body in csv_cases.edge_cases():
        same(gpu_scan(body, types), oracle.csv_scan(body, types))


def test_random_tables(cuda):
    rng = np.random.default_rng(21)
    for _ in range(120):
        types, header, body = csv_cases.random_csv(rng)
        same(gpu_scan(body, types), oracle.csv_scan(body, types))


def test_many_tiles_with_quotes(cuda):
    """Quote-heavy text of many 16 KiB tiles: record index look-back across
    tiles that start inside quoted fields, escaped quotes and CR/LF runs."""
    rng = np.random.default_rng(24)
    done = 0
    while done < 3:
        types, header, body = csv_cases.random_csv(rng, max_rows=12000)
        if len(body) < 200_000:
            continue
        same(gpu_scan(body, types), oracle.csv_scan(body, types))
        done += 1


def test_unaligned_text_and_wide_slots(cuda):
    rng = np.random.default_rng(22)
    for off in (1, 3, 7, 13):
        types, header, body = csv_cases.random_csv(rng, max_rows=200)
        same(gpu_scan(body, types, width=256, offset=off), oracle.csv_scan(body, types, width=256))


def test_records_longer_than_the_staging_span(cuda):
    # 128 records of ~1 KB exceed a parse block's shared-memory span: the walk reads global memory
    rng = np.random.default_rng(23)
    lines = [f"{i},{'x' * int(rng.integers(300, 1500))},{rng.uniform(0, 9):.3f}" for i in range(700)]
    body = ("\n".join(lines) + "\n").encode()
    types = [0, 3, 1]
    same(gpu_scan(body, types, width=256), oracle.csv_scan(body, types, width=256))


def test_index_capacity_and_count(cuda, yq):
    body = b"1\n2\n\n3\r\n4"
    t = torch.frombuffer(bytearray(body), dtype=torch.uint8).cuda()
    n = C.c_uint64(0)
    starts = torch.zeros(8, dtype=torch.int32, device="cuda")
    st = yq.yq_csv_index(t.data_ptr(), len(body), starts.data_ptr(), 2, C.byref(n), None, 0, None)
    assert st == A.ERR_CAPACITY and n.value == 4
    assert yq.yq_csv_index(t.data_ptr(), len(body), starts.data_ptr(), 8, C.byref(n), None, 0, None) == A.OK
    torch.cuda.synchronize()
    assert starts[:4].tolist() == [0, 2, 5, 8]


def test_sales_csv_then_the_filter_aggregate_query(cuda):
    """The 1M-row filter+aggregate table as CSV text: scanned columns equal the
    oracle's, and the benchmark query over them equals the oracle's result."""
    header, body = datagen.sales_csv(1_000_000, seed=0)
    schema = ops.csv_schema(header.decode().strip(), bytes(body[:200]).decode().split("\n")[0])
    types = [c.type for c in schema]
    assert types == [A.INT32, A.FLOAT32, A.INT32, A.INT32, A.TEXT, A.DATETIME]
    b = body.tobytes()
    g = gpu_scan(b, types)
    o = oracle.csv_scan(b, types)
    same(g, o)
    assert g["rows"] == 1_000_000 and np.array_equal(g["cols"][0][0], np.arange(1_000_000, dtype=np.int32))
    # WHERE discount BETWEEN 1 AND 3 AND qty < 25 AND category <> '<one>' over the scanned batch
    text = torch.frombuffer(bytearray(b), dtype=torch.uint8).cuda()
    batch = ops.csv_scan(text, types, [1, 2, 3, 4], text_width=datagen.TEXT_WIDTH)
    price, qty, disc = ColumnRef(0, A.FLOAT32), ColumnRef(1, A.INT32), ColumnRef(2, A.INT32)
    pred = And(between(disc, Constant(1, A.INT32), Constant(3, A.INT32)), Compare(A.LT, qty, Constant(25, A.INT32)),
               Compare(A.NE, ColumnRef(3, A.TEXT), Constant(datagen.EXCLUDED_CATEGORY, A.TEXT)))
    aggs = [Aggregate(A.AGG_SUM, Arith(A.MUL, price, Cast(disc, A.FLOAT32))), Aggregate(A.AGG_COUNT_STAR),
            Aggregate(A.AGG_MIN, price), Aggregate(A.AGG_MAX, price)]
    got = ops.filter_aggregate(batch, pred, aggs)
    cols = {0: (o["cols"][1][0], None, A.FLOAT32), 1: (o["cols"][2][0], None, A.INT32),
            2: (o["cols"][3][0], None, A.INT32), 3: (o["cols"][4][0], None, A.TEXT)}
    want = expr_eval.aggregate(pred, aggs, cols, 1_000_000)
    assert got[1:] == want[1:]
    assert abs(got[0] - want[0]) <= 1e-6 * abs(want[0])


def test_large_csv_properties(cuda):
    """8M rows (~420 MB of text, thousands of tiles and parse blocks): every id
    in order, no NULLs, values in their generators' ranges, and every 997th row
    equal to the oracle's parse of that line."""
    rows = 8_000_000
    header, body = datagen.sales_csv(rows, seed=5)
    types = [A.INT32, A.FLOAT32, A.INT32, A.INT32, A.TEXT, A.DATETIME]
    text = torch.from_numpy(body).cuda()
    batch = ops.csv_scan(text, types, text_width=16)
    assert batch.rows == rows
    ids = batch.columns[0].data.cpu().numpy()
    assert np.array_equal(ids, np.arange(rows, dtype=np.int32))
    for c in batch.columns:
        assert int(c.nulls.sum()) == 0
    qty = batch.columns[2].data.cpu().numpy()
    assert qty.min() >= 1 and qty.max() <= 50
    d = batch.columns[5].data.cpu().numpy()
    assert d.min() >= datagen.DATE_LO and d.max() < datagen.DATE_HI + 86400
    ends = np.flatnonzero(body == ord("\n"))
    starts = np.concatenate([[0], ends[:-1] + 1])
    pick = np.arange(0, rows, 997)
    sample = b"".join(body[starts[i]:ends[i] + 1].tobytes() for i in pick)
    o = oracle.csv_scan(sample, types)
    for k in range(6):
        gv = batch.columns[k].data[torch.from_numpy(pick).cuda()].cpu().numpy()
        assert gv.tobytes() == o["cols"][k][0].tobytes()


# ------------------------------------------------------------------ writer
def random_batch(rng, rows):
    """Columns of every writer type with NULLs, special floats, negative and
    far dates, and text slots of every fill (empty, partial, full without NUL)."""
    W = 12
    f = rng.integers(0, 2**32, rows, dtype=np.uint64).astype(np.uint32).view(np.float32).copy()
    f[::7] = (rng.integers(100, 100000, len(f[::7])) / 100.0).astype(np.float32)
    text = rng.integers(32, 127, (rows, W), dtype=np.uint8)
    cut = rng.integers(0, W + 1, rows)
    text[np.arange(W)[None, :] >= cut[:, None]] = 0
    cols = [(A.INT32, 4, rng.integers(-2**31, 2**31, rows).astype(np.int32)),
            (A.FLOAT32, 4, f),
            (A.DATETIME, 8, rng.integers(-2**38, 2**38, rows).astype(np.int64)),
            (A.TEXT, W, text),
            (A.INT64, 8, rng.integers(-2**62, 2**62, rows).astype(np.int64))]
    out = []
    for t, w, v in cols:
        nulls = (rng.random(rows) < 0.1).astype(np.uint8) if rng.random() < 0.7 else None
        out.append((t, w, v, nulls))
    return out


def device_batch(cols):
    dc = []
    for t, w, v, nulls in cols:
        d = torch.from_numpy(np.ascontiguousarray(v)).cuda()
        dc.append(ops.DeviceColumn(d, t, None if nulls is None else torch.from_numpy(nulls).cuda()))
    return ops.DeviceBatch(dc)


def test_writer_matches_oracle(cuda):
    rng = np.random.default_rng(31)
    for rows in (1, 5, 127, 128, 129, 3000, 50_000):
        cols = random_batch(rng, rows)
        got = ops.csv_format(device_batch(cols)).cpu().numpy().tobytes()
        assert got == oracle.csv_format(cols, rows)


def test_writer_unaligned_output_and_capacity(cuda, yq):
    rng = np.random.default_rng(32)
    cols = random_batch(rng, 2000)
    want = oracle.csv_format(cols, 2000)
    b = device_batch(cols)
    bc, keep = b.c()
    n = C.c_uint64(0)
    out = torch.zeros(len(want) + 64, dtype=torch.uint8, device="cuda")
    assert yq.yq_csv_format(C.byref(bc), out.data_ptr() + 3, 10, C.byref(n), None, 0, None) == A.ERR_CAPACITY
    assert n.value == len(want)
    assert yq.yq_csv_format(C.byref(bc), out.data_ptr() + 3, len(want), C.byref(n), None, 0, None) == A.OK
    torch.cuda.synchronize()
    host = out.cpu().numpy().tobytes()
    assert host[3:3 + len(want)] == want and host[:3] == bytes(3) and host[3 + len(want):] == bytes(61)


def test_scan_then_write_round_trip(cuda):
    """Sales CSV text -> device scan -> device writer equals the oracle writer
    over the oracle scan (1M rows, bit-exact text)."""
    header, body = datagen.sales_csv(1_000_000, seed=9)
    types = [A.INT32, A.FLOAT32, A.INT32, A.INT32, A.TEXT, A.DATETIME]
    batch = ops.csv_scan(torch.from_numpy(body).cuda(), types, text_width=16)
    got = ops.csv_format(batch).cpu().numpy().tobytes()
    o = oracle.csv_scan(body.tobytes(), [0, 1, 0, 0, 3, 2], width=16)
    want = oracle.csv_format([(t, 16 if t == 3 else 0, v, n) for t, (v, n) in zip([0, 1, 0, 0, 3, 2], o["cols"])],
                             1_000_000)
    assert got == want
    assert got.count(b"\n") == 1_000_000


# ------------------------------------------------- in the operator tree
def test_plan_csv_scan_filter_aggregate(cuda):
    """GetOperator's place in the C++ operator tree: CSV text -> device scan
    batch by batch -> filter -> aggregate (the benchmark query), against the
    oracle's parse and evaluation."""
    from yallasql_b200.plan import Plan
    from test_filter_gpu import sales_query_exprs
    from helpers import rel_close
    header, body = datagen.sales_csv(300_000, seed=4)
    data = header + body.tobytes()
    pred, aggs = sales_query_exprs()
    for batch_rows in (0, 50_000):
        p = Plan()
        root = p.aggregate(p.filter(p.scan_csv(data, ["price", "qty", "discount", "category"], text_width=16,
                                               batch_rows=batch_rows), pred), aggs)
        res = p.execute(root)
        got = [v[0] for v, n in res]
        o = oracle.csv_scan(body.tobytes(), [-1, 1, 0, 0, 3, -1], width=16)
        cols = {0: (o["cols"][1][0], None, A.FLOAT32), 1: (o["cols"][2][0], None, A.INT32),
                2: (o["cols"][3][0], None, A.INT32), 3: (o["cols"][4][0], None, A.TEXT)}
        want = expr_eval.aggregate(pred, aggs, cols, o["rows"])
        assert int(got[1]) == want[1]
        assert float(got[2]) == want[2] and float(got[3]) == want[3]
        assert rel_close(float(got[0]), want[0], 1e-6)


def test_plan_csv_scan_batches_and_errors(cuda):
    """Batches of 1,000 records over a file with ragged rows: the result
    equals the oracle's parse; a cell stoi rejects fails the plan."""
    from yallasql_b200.plan import Plan
    rng = np.random.default_rng(25)
    lines = []
    for i in range(5000):
        if i % 97 == 5:  # the first data line stays whole: the schema's types come from it
            lines.append(f"{i},only-two")
        else:
            # the header-tag rule splits the first data line at every ',' (quotes or not), so
            # its text stays comma-free there and `v` is typed FLOAT from its '.'
            t = f'"t{i},x"' if i else '"t0"'
            lines.append(f'{i},{t},{rng.uniform(-50, 50):.3f},2020-0{1 + i % 9}-1{i % 10} 0{i % 10}:00:00')
    body = ("\n".join(lines) + "\n").encode()
    header = "id (N),t (T),v (N),d (D)"
    data = (header + "\n").encode() + body
    types = [c.type for c in ops.csv_schema(header, lines[0])]
    assert types == [A.INT32, A.TEXT, A.FLOAT32, A.DATETIME]
    p = Plan()
    res = p.execute(p.scan_csv(data, ["d", "id", "v", "t"], text_width=16, batch_rows=1000))
    o = oracle.csv_scan(body, types, width=16)
    for (gv, gn), (ov, on) in zip(res, [o["cols"][3], o["cols"][0], o["cols"][2], o["cols"][1]]):
        assert gv.tobytes() == ov.tobytes() and np.array_equal(gn, on)
    bad = b"a (N)\n1\n2\nx\n"
    p2 = Plan()
    with pytest.raises(A.YQError):
        p2.execute(p2.scan_csv(bad))
