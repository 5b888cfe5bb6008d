#!/usr/bin/env python3
"""Benchmark of the ORDER BY operator on the 64M-row table (B200).

Workload (one step): over a 64,000,000-row table {key f32 uniform [-1e6, 1e6),
id int64, txt 16-byte text, d date} (seed 1), run
  ORDER BY key DESC   and then   ORDER BY d ASC,
each producing the fully sorted table (all four columns). With --mode
outofcore (default) each query is the reference's out-of-core plan: the
table arrives as 4 MB batches (116,480 rows at 36 B/row), every batch is
sorted into a run, and runs are merged pairwise by merge path until one run
remains. --mode incore sorts the whole table at once. Metric: rows/s (rows
sorted per second, both queries), plus the HBM roofline of the dominant kernel.

`python bench.py --gpus N --steps K --warmup W [--impl reference]`; for N>1
launch under torch.distributed.run: every rank sorts its own table (replicas,
weak scaling), time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "operator rows/s & %HBM peak; query p50/p99 ms, batched vs plain, 1xB200"
UNIT = "rows/s"
ROW_BYTES = 4 + 8 + 16 + 8  # key, id, txt, d
FALLBACK_HBM_GBS = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="yq", choices=["yq", "reference"])
    p.add_argument("--rows", type=int, default=64_000_000)
    p.add_argument("--dist", default="uniform", choices=["uniform", "zipf", "equal"])
    p.add_argument("--mode", default="outofcore", choices=["outofcore", "incore"])
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-ops", action="store_true", help="skip the other operators' workloads")
    p.add_argument("--no-batched", action="store_true", help="skip the batched-form comparison")
    p.add_argument("--batched-tasks", type=int, default=512)
    p.add_argument("--no-serving", action="store_true", help="skip the serving-form comparison")
    p.add_argument("--no-dists", action="store_true", help="skip the other key distributions' ORDER BY runs")
    p.add_argument("--serving-requests", type=int, default=400)
    return p.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for name, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def committed_traffic() -> dict:
    """DRAM bytes and algorithmic bytes of one ncu-captured launch per kernel tag
    (profiles/traffic.json, written from the committed ncu summaries)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


# ---------------------------------------------------------------- workload
def make_table(rows: int, dist: str):
    from yallasql_b200 import datagen
    return datagen.order_table(rows, seed=1, dist=dist)


class OrderByJob:
    """Both ORDER BY queries over one device-resident table."""

    def __init__(self, t: dict, mode: str):
        import torch
        from yallasql_b200 import _abi as A, datagen
        from yallasql_b200.ops import DeviceBatch, DeviceColumn
        self.torch = torch
        self.A = A
        self.rows = int(t["key"].shape[0])
        self.mode = mode
        dev = lambda a, ty: DeviceColumn(torch.from_numpy(a).cuda(), ty)
        self.table = DeviceBatch([dev(t["key"], A.FLOAT32), dev(t["id"], A.INT64), dev(t["txt"], A.TEXT),
                                  dev(t["d"], A.DATETIME)])
        self.batch_rows = datagen.batch_row_counts(self.rows, ROW_BYTES)
        self.offsets = [0]
        for c in self.batch_rows:
            self.offsets.append(self.offsets[-1] + c)
        self.out = [DeviceBatch([DeviceColumn.empty(c.type, self.rows, c.width if c.type == A.TEXT else None)
                                 for c in self.table.columns]) for _ in range(2)]
        if mode == "outofcore":
            from yallasql_b200.ops import OrderByRuns
            self.runs = {k: OrderByRuns(self.table, k, self.offsets) for k in (0, 3)}
        self.perm = torch.empty(self.rows, dtype=torch.int32, device="cuda")
        from yallasql_b200 import ops
        self.ops = ops
        ws = max(ops.sort_workspace_bytes(self.table.columns[0], self.offsets),
                 ops.sort_workspace_bytes(self.table.columns[3], self.offsets),
                 ops.sort_workspace_bytes(self.table.columns[0]), ops.sort_workspace_bytes(self.table.columns[3]))
        self.ws = torch.empty(ws, dtype=torch.uint8, device="cuda")

    def query(self, src, key: int, desc: bool, out):
        ops = self.ops
        if self.mode == "incore":
            ops.sort_indices(src.columns[key], desc, out=self.perm, workspace=self.ws)
            ops.gather(src, self.perm, out=out)
            return out
        # out-of-core: sort every 4 MB batch into a run, merge (key, row id)
        # runs pairwise by merge path, gather the payload once at the end
        return self.runs[key].run(src, desc, out)

    def step(self, src=None):
        src = self.table if src is None else src
        a = self.query(src, 0, True, self.out[0])
        b = self.query(src, 3, False, self.out[1])
        return a, b


def _timed(fn, reps: int):
    """Device ms per call of fn() (CUDA events on the current stream), after one warm call."""
    import torch
    fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def operator_suite(lib, peak: float) -> dict:
    """The other operators of the metric on their config workloads: rows/s and
    the HBM roofline of each operator's kernel (algorithmic bytes from the
    library's per-launch accounting / device time)."""
    import torch
    from yallasql_b200 import _abi as A, datagen, ops
    from yallasql_b200.expr import Aggregate, And, Arith, Cast, ColumnRef, Compare, Constant, between
    dev = lambda a, t: ops.DeviceColumn(torch.from_numpy(np.ascontiguousarray(a)).cuda(), t)
    out = {}

    def profiled(name, fn, rows, reps, tag):
        fn()  # first call compiles the program-specialised kernel
        torch.cuda.synchronize()
        lib.yq_profile_enable(1)
        lib.yq_profile_read(None, 0, 1)
        ms = _timed(fn, reps)
        buf = C.create_string_buffer(1 << 14)
        lib.yq_profile_read(buf, len(buf), 1)
        lib.yq_profile_enable(0)
        prof = json.loads(buf.value.decode() or "{}")
        k = prof.get(tag, {})
        entry = {"rows": rows, "ms": round(ms, 4), "rows_per_s": rows / (ms / 1e3)}
        if k.get("launches"):
            per_ms = k["ms"] / k["launches"]
            gbs = k["units"] / k["launches"] / (per_ms / 1e3) / 1e9
            entry.update({"kernel": tag, "kernel_ms": round(per_ms, 4), "achieved_gbs": round(gbs, 1),
                          "frac_of_measured_hbm": round(gbs / peak, 4),
                          "algorithmic_bytes_per_launch": k["units"] / k["launches"]})
        out[name] = entry

    price, qty, disc, cat = (ColumnRef(0, A.FLOAT32), ColumnRef(1, A.INT32), ColumnRef(2, A.INT32),
                             ColumnRef(3, A.TEXT))
    pred = And(between(disc, Constant(1, A.INT32), Constant(3, A.INT32)), Compare(A.LT, qty, Constant(25, A.INT32)),
               Compare(A.NE, cat, Constant(datagen.EXCLUDED_CATEGORY, A.TEXT)))
    aggs = [Aggregate(A.AGG_SUM, Arith(A.MUL, price, Cast(disc, A.FLOAT32))), Aggregate(A.AGG_COUNT_STAR),
            Aggregate(A.AGG_MIN, price), Aggregate(A.AGG_MAX, price)]
    for rows, name in ((1_000_000, "filter_aggregate_1M"), (64_000_000, "filter_aggregate_64M")):
        t = datagen.sales_table(rows, seed=0)
        b = ops.DeviceBatch([dev(t["price"], A.FLOAT32), dev(t["qty"], A.INT32), dev(t["discount"], A.INT32),
                             dev(t["category"], A.TEXT)])
        plan = ops.AggPlan([A.FLOAT32, A.INT32, A.INT32, A.TEXT], pred, aggs)
        st = ops.AggState(aggs)
        ws = torch.empty(lib.yq_filter_aggregate_workspace_size(rows, len(aggs)), dtype=torch.uint8, device="cuda")
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda") if rows <= 4_000_000 else None

        def fa():
            if flush is not None:
                flush.zero_()  # 256 MB write evicts the 28 MB table from L2 between reps
            plan.run(b, st, workspace=ws)
        profiled(name, fa, rows, 10, "filter_aggregate")
        if rows == 64_000_000:
            sel = [3, 0, Arith(A.MUL, price, Cast(disc, A.FLOAT32))]
            pplan = ops.ProjectPlan([A.FLOAT32, A.INT32, A.INT32, A.TEXT], [4, 4, 4, 16], pred, sel)
            profiled("filter_project_64M", lambda: pplan.run(b, with_nulls=False), rows, 5, "filter_project")
        del b, t
    fact, dim = datagen.star_tables(60_000_000, seed=2)
    fb = ops.DeviceBatch([dev(fact["datekey"], A.INT32), dev(fact["quantity"], A.INT32),
                          dev(fact["discount"], A.INT32), dev(fact["extendedprice"], A.FLOAT32)])
    db = ops.DeviceBatch([dev(dim["datekey"], A.INT32), dev(dim["year"], A.INT32), dev(dim["month"], A.INT32)])
    jp = ops.JoinAggPlan([A.INT32] * 3 + [A.FLOAT32], [A.INT32] * 3,
                         And(between(ColumnRef(2, A.INT32), Constant(1, A.INT32), Constant(3, A.INT32)),
                             Compare(A.LT, ColumnRef(1, A.INT32), Constant(25, A.INT32))), 0,
                         Compare(A.EQ, ColumnRef(1, A.INT32), Constant(1993, A.INT32)), 0,
                         [Aggregate(A.AGG_SUM, Arith(A.MUL, ColumnRef(3, A.FLOAT32),
                                                     Cast(ColumnRef(2, A.INT32), A.FLOAT32)))])
    jst = ops.AggState(jp.aggs)
    profiled("star_join_aggregate_60M", lambda: jp.run(fb, db, jst), 60_000_000, 5, "join_aggregate")
    del fb, fact
    x, y = datagen.cross_tables(20_000, seed=2)
    xb, yb = ops.DeviceBatch([dev(x, A.INT32)]), ops.DeviceBatch([dev(y, A.INT32)])
    res = ops.join_project(xb, yb, [(0, 0, A.LT)], [(0, 0), (1, 0)])
    pairs = res.rows
    outs_c = (A.JoinOutput * 2)(A.JoinOutput(0, 0), A.JoinOutput(1, 0))
    oc = (A.Column * 2)(*[c.c() for c in res.columns])
    lbc, lk = xb.c()
    rbc, rk = yb.c()
    conds = (A.JoinCond * 1)(A.JoinCond(0, 0, A.LT))
    n64 = C.c_uint64()
    profiled("cross_product_lt_20Kx20K",
             lambda: lib.yq_join_project(C.byref(lbc), C.byref(rbc), conds, 1, outs_c, 2, oc, pairs, C.byref(n64),
                                         None, 0, torch.cuda.current_stream().cuda_stream),
             pairs, 5, "join_nested_loop")
    # GROUP BY discount over the 64M-row sales table (sort + group kernels)
    t = datagen.sales_table(64_000_000, seed=0)
    gb = ops.DeviceBatch([dev(t["discount"], A.INT32), dev(t["price"], A.FLOAT32), dev(t["qty"], A.INT32)])
    del t
    gaggs = [(A.AGG_COUNT_STAR, 0), (A.AGG_SUM, 1), (A.AGG_AVG, 2), (A.AGG_MIN, 1), (A.AGG_MAX, 1)]
    g_out = ops.group_by(gb, 0, gaggs, capacity=64)
    gws = torch.empty(lib.yq_group_by_workspace_size(C.byref(gb.columns[0].c()), gb.rows, len(gaggs), 64),
                      dtype=torch.uint8, device="cuda")
    gbc, gkeep = gb.c()
    gag = (A.GroupAgg * len(gaggs))(*[A.GroupAgg(k, c) for k, c in gaggs])
    gout = [ops.DeviceColumn.empty(c.type, 64, nulls=True) for c in g_out.columns]
    goc = (A.Column * len(gout))(*[c.c() for c in gout])
    ng = C.c_uint32()
    profiled("group_by_discount_64M",
             lambda: A.check(lib.yq_group_by(C.byref(gbc), 0, gag, len(gaggs), goc, 64, C.byref(ng), gws.data_ptr(),
                                             gws.numel(), torch.cuda.current_stream().cuda_stream), "yq_group_by"),
             64_000_000, 3, "group_accumulate")
    out["group_by_discount_64M"]["groups"] = int(ng.value)
    del gb, gws, gkeep
    out["cross_product_lt_20Kx20K"]["output_pairs"] = pairs
    out["cross_product_lt_20Kx20K"]["output_bytes_per_s"] = pairs * 8 / (out["cross_product_lt_20Kx20K"]["ms"] / 1e3)
    out["cross_product_lt_20Kx20K"]["frac_of_measured_hbm_output"] = round(
        pairs * 8 / (out["cross_product_lt_20Kx20K"]["ms"] / 1e3) / 1e9 / peak, 4)
    return out


def csv_suite(lib, peak: float, rows: int = 8_000_000) -> dict:
    """CSV scan (the device-side GetOperator::next) over the filter+aggregate
    table written as CSV text: device-resident text (larger than L2) -> typed
    columns; per-kernel HBM roofline; the same from pinned host bytes with the
    host->device copy inside (ingress reported against the measured pinned copy
    rate); the reference's own reader (csv-parser + std::stoi/stof/strptime) on
    a bounded sample on the host."""
    import torch
    import oracle
    from yallasql_b200 import _abi as A, datagen, ops
    header, body = datagen.sales_csv(rows, seed=0)
    nbytes = int(body.size)
    types = [A.INT32, A.FLOAT32, A.INT32, A.INT32, A.TEXT, A.DATETIME]
    host = torch.from_numpy(body).pin_memory()
    text = host.cuda()
    s = torch.cuda.current_stream().cuda_stream
    n = C.c_uint64(0)
    lib.yq_csv_index(text.data_ptr(), nbytes, None, 0, C.byref(n), None, 0, s)
    nrec = int(n.value)
    starts = torch.empty(nrec + 1, dtype=torch.int32, device="cuda")
    iws = torch.empty(lib.yq_csv_index_workspace_size(nbytes), dtype=torch.uint8, device="cuda")
    pws = torch.empty(lib.yq_csv_parse_workspace_size(nrec), dtype=torch.uint8, device="cuda")
    cols = [ops.DeviceColumn.empty(t, nrec, 16 if t == A.TEXT else None, nulls=True) for t in types]
    ccols = (A.Column * len(cols))(*[c.c() for c in cols])
    fc = (C.c_int32 * len(types))(*range(len(types)))
    out_rows = C.c_uint32(0)
    err = A.CsvError()

    def scan(src):
        A.check(lib.yq_csv_index(src.data_ptr(), nbytes, starts.data_ptr(), nrec + 1, C.byref(n), iws.data_ptr(),
                                 iws.numel(), s), "yq_csv_index")
        A.check(lib.yq_csv_parse(src.data_ptr(), nbytes, starts.data_ptr(), nrec, fc, len(types), ccols, len(cols),
                                 C.byref(out_rows), C.byref(err), pws.data_ptr(), pws.numel(), s), "yq_csv_parse")

    scan(text)
    assert out_rows.value == rows
    torch.cuda.synchronize()
    lib.yq_profile_enable(1)
    lib.yq_profile_read(None, 0, 1)
    reps = 5
    ms = _timed(lambda: scan(text), reps)
    buf = C.create_string_buffer(1 << 14)
    lib.yq_profile_read(buf, len(buf), 1)
    lib.yq_profile_enable(0)
    prof = json.loads(buf.value.decode() or "{}")
    kernels = {}
    for tag in ("csv_tiles", "csv_tile_scan", "csv_emit", "csv_parse"):
        k = prof.get(tag, {})
        if k.get("launches"):
            per_ms = k["ms"] / k["launches"]
            gbs = k["units"] / k["launches"] / (per_ms / 1e3) / 1e9
            kernels[tag] = {"kernel_ms": round(per_ms, 4), "achieved_gbs": round(gbs, 1),
                            "frac_of_measured_hbm": round(gbs / peak, 4),
                            "algorithmic_bytes_per_launch": k["units"] / k["launches"]}
    # from pinned host bytes: the copy in, then the scan (what GetOperator::next + storeBuffer do)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    staging = torch.empty_like(text)

    def e2e():
        staging.copy_(host, non_blocking=True)
        scan(staging)
    e2e()
    torch.cuda.synchronize()
    e2e_ms = _timed(e2e, 3)
    ev0.record()
    for _ in range(3):
        staging.copy_(host, non_blocking=True)
    ev1.record()
    torch.cuda.synchronize()
    h2d_gbs = 3 * nbytes / (ev0.elapsed_time(ev1) / 1e3) / 1e9
    out = {"rows": rows, "csv_bytes": nbytes, "ms": round(ms, 4), "rows_per_s": rows / (ms / 1e3),
           "text_gbs": round(nbytes / (ms / 1e3) / 1e9, 1), "kernels": kernels,
           "e2e_from_pinned_host": {"ms": round(e2e_ms, 4), "rows_per_s": rows / (e2e_ms / 1e3),
                                    "h2d_bytes": nbytes, "ingress_pinned_h2d_gbs": round(h2d_gbs, 1)}}
    # the reference's reader on the host: bounded sample, one thread of conversions (+ csv-parser's reader thread)
    sample = min(rows, 1_000_000)
    cut = int(np.flatnonzero(body == ord("\n"))[sample - 1]) + 1
    sub = body[:cut].tobytes()
    t0 = time.perf_counter()
    if oracle.ref_csv_available():
        oracle.ref_csv_scan(header, sub, [0, 1, 0, 0, 3, 2], width=16, guess=True)
        kind = "reference"
    else:
        oracle.csv_scan(sub, [0, 1, 0, 0, 3, 2], width=16)
        kind = "port"
    dt = time.perf_counter() - t0
    out["cpu_baseline"] = {"value": sample / dt, "unit": "rows/s", "cores": 1, "kind": kind,
                           "sample": f"first {sample} of {rows} rows ({cut} bytes): csv-parser read_row + "
                                     "std::stoi/std::stof/strptime+timegm per field, as GetOperator::next"}
    # the writer (CsvWriter::batchToCsv on the device) over the scanned columns
    batch = ops.DeviceBatch(cols)
    bc, keep = batch.c()
    nout = C.c_uint64(0)
    lib.yq_csv_format(C.byref(bc), None, 0, C.byref(nout), None, 0, s)
    text_out = torch.empty(int(nout.value), dtype=torch.uint8, device="cuda")
    fws = torch.empty(lib.yq_csv_format_workspace_size(rows), dtype=torch.uint8, device="cuda")

    def fmt():
        A.check(lib.yq_csv_format(C.byref(bc), text_out.data_ptr(), text_out.numel(), C.byref(nout), fws.data_ptr(),
                                  fws.numel(), s), "yq_csv_format")
    fmt()
    torch.cuda.synchronize()
    lib.yq_profile_enable(1)
    lib.yq_profile_read(None, 0, 1)
    fms = _timed(fmt, reps)
    buf = C.create_string_buffer(1 << 14)
    lib.yq_profile_read(buf, len(buf), 1)
    lib.yq_profile_enable(0)
    prof = json.loads(buf.value.decode() or "{}")
    fk = {}
    for tag in ("csv_format_len", "csv_format_write"):
        k = prof.get(tag, {})
        if k.get("launches"):
            per_ms = k["ms"] / k["launches"]
            entry = {"kernel_ms": round(per_ms, 4)}
            if k["units"]:
                gbs = k["units"] / k["launches"] / (per_ms / 1e3) / 1e9
                entry.update({"achieved_gbs": round(gbs, 1), "frac_of_measured_hbm": round(gbs / peak, 4),
                              "algorithmic_bytes_per_launch": k["units"] / k["launches"]})
            fk[tag] = entry
    w_sample = min(rows, 1_000_000)
    host_cols = [(t, c.width if t == A.TEXT else 0, c.data[:w_sample].cpu().numpy(), c.nulls[:w_sample].cpu().numpy())
                 for t, c in zip([0, 1, 0, 0, 3, 2], cols)]
    t0 = time.perf_counter()
    oracle.csv_format(host_cols, w_sample)
    wdt = time.perf_counter() - t0
    out["write"] = {"rows": rows, "text_bytes": int(nout.value), "ms": round(fms, 4), "rows_per_s": rows / (fms / 1e3),
                    "text_gbs": round(int(nout.value) / (fms / 1e3) / 1e9, 1), "kernels": fk,
                    "cpu_baseline": {"value": w_sample / wdt, "unit": "rows/s", "cores": 1, "kind": "port",
                                     "sample": f"first {w_sample} rows: snprintf / gmtime_r + strftime per cell, "
                                               "as CsvWriter::batchToCsv (std::to_chars) formats them"}}
    del text, staging, cols, batch, keep, text_out
    return out


def batched_form(args) -> dict:
    """Batched form (512 tasks, row counts log-uniform in [1K, 4M], seed 3):
    the plain per-task form against the segmented launches replayed as one CUDA
    graph, on the same GPU and data; tasks/s from device time around each form."""
    import torch
    from yallasql_b200 import batched
    ntasks = args.batched_tasks
    rows = batched.task_rows(ntasks, seed=3)
    ts = batched.TaskSet(rows, seed=3, on_device=True)
    plain = batched.PlainRunner(ts)
    t0 = time.perf_counter()
    pipe = batched.BatchedPipeline(ts, graph=True)
    setup_s = time.perf_counter() - t0
    plain_ms = _timed(plain.run, 2)
    batched_ms = _timed(pipe.run, 3)
    torch.cuda.synchronize()
    same_sorted = all(torch.equal(ts.sout.columns[c].data[a:b], ts.souts[g].columns[c].data)
                      for g, (a, b) in enumerate(zip(ts.soffs[:-1], ts.soffs[1:])) for c in range(6))
    pres, bres = plain.results(), pipe.results()
    same_aggs = all(p[1:] == q[1:] and abs(p[0] - q[0]) <= 1e-6 * max(1.0, abs(p[0])) if p[1] else p == q
                    for p, q in zip(pres, bres))
    total_rows = int(sum(rows))
    return {"tasks": ntasks, "rows": total_rows, "filter_tasks": len(ts.frows), "order_by_tasks": len(ts.srows),
            "plain_ms": round(plain_ms, 3), "batched_ms": round(batched_ms, 3),
            "plain_tasks_per_s": ntasks / (plain_ms / 1e3), "batched_tasks_per_s": ntasks / (batched_ms / 1e3),
            "speedup": round(plain_ms / batched_ms, 3),
            "batched_algorithmic_gbs": round(ts.algorithmic_bytes / (batched_ms / 1e3) / 1e9, 1),
            "sort_autotuned": {"digit_bits": pipe.tuned[0], "items_per_thread": pipe.tuned[1],
                               "block_threads": pipe.tuned[2],
                               "swept": "digit bits {4,6,8} x items {4,8,12,16} x block {128,256,512}, "
                                        "instantiated variants"},
            "graph": True, "setup_s": round(setup_s, 2), "results_equal_plain": bool(same_sorted and same_aggs),
            "error_word": pipe.error_word()}


def serving_form(args) -> dict:
    """Serving form (seed 4): 40/30/20/10 filter / ORDER BY / join / scalar
    subquery mix over resident tables of 10K-60M rows. Saturation throughput of
    the plain form (one request at a time) and the continuous form (streams,
    budgeted admission, co-launched filters), then both at the same Poisson
    arrival rate (70% of the plain form's saturation) with p50/p99 latency."""
    import copy
    import torch
    from yallasql_b200 import serving
    cat = serving.Catalog(ntables=8, lo=10_000, hi=60_000_000, seed=4)
    plans = serving.Plans()
    n = args.serving_requests
    # warm-up: every class on every table alone, all at once (shared and not),
    # and a Poisson trace, so every kernel variant is compiled before timing
    warm = serving.warm_trace(cat)
    serving.serve_plain(copy.deepcopy(warm), cat, plans)
    serving.serve_continuous(copy.deepcopy(warm), cat, plans)
    serving.serve_continuous(copy.deepcopy(warm), cat, plans, share=False)
    serving.serve_continuous(copy.deepcopy(serving.make_trace(120, 1500.0, cat, seed=5)), cat, plans)
    burst = serving.make_trace(n, 0.0, cat, seed=4)

    def median_of(fn, trace, k=3):
        """The run with the median throughput of k runs of the same trace (a
        single run can lose hundreds of ms to a host stall: on the GPU box one
        run in three or four did, in either form, with no kernel compiled
        during it); the median run carries every run's throughput."""
        outs = sorted((fn(copy.deepcopy(trace)) for _ in range(k)), key=lambda d: d["queries_per_s"])
        med = dict(outs[k // 2])
        med["runs_queries_per_s"] = [round(o["queries_per_s"], 1) for o in outs]
        return med

    plain_sat = median_of(lambda tr: serving.serve_plain(tr, cat, plans), burst, 5)
    cont_sat = median_of(lambda tr: serving.serve_continuous(tr, cat, plans, slots=8, budget=40e9), burst, 5)
    # the same loop without sharing work between requests (no coalescing of
    # identical requests, one scan per filter request, no resident permutations)
    cont_sat_noshare = median_of(
        lambda tr: serving.serve_continuous(tr, cat, plans, slots=8, budget=40e9, share=False), burst, 5)
    rate = 0.7 * plain_sat["queries_per_s"]
    trace = serving.make_trace(n, rate, cat, seed=4)
    plain_open = serving.serve_plain(copy.deepcopy(trace), cat, plans)
    cont_open = serving.serve_continuous(copy.deepcopy(trace), cat, plans, slots=8, budget=40e9)
    # Poisson-rate sweep: a form "sustains" a rate when it completes the trace
    # at >= 95% of the offered rate; at a p99 budget, each form's best rate is
    # the highest sustained rate whose p99 stays within the budget
    # (rates from a quarter of the plain form's saturation throughput up to
    # 90% of the continuous form's; each point the median of three runs)
    grid = sorted({round(f * plain_sat["queries_per_s"]) for f in (0.25, 0.5, 0.75, 1.0)} |
                  {round(f * cont_sat["queries_per_s"]) for f in (0.4, 0.55, 0.7, 0.8, 0.9)})
    sweep = []
    for rr in grid:
        tr = serving.make_trace(n, float(rr), cat, seed=6)
        pl = median_of(lambda x: serving.serve_plain(x, cat, plans), tr)
        co = median_of(lambda x: serving.serve_continuous(x, cat, plans, slots=8, budget=40e9), tr)
        cn = median_of(lambda x: serving.serve_continuous(x, cat, plans, slots=8, budget=40e9, share=False), tr)
        pick = lambda d: {k: round(d[k], 3) for k in ("queries_per_s", "p50_ms", "p99_ms")}
        sweep.append({"offered_per_s": rr, "plain": pick(pl), "continuous": pick(co),
                      "continuous_without_sharing": pick(cn)})

    def best(form, budget_ms):
        ok = [e["offered_per_s"] for e in sweep if e[form]["queries_per_s"] >= 0.95 * e["offered_per_s"]
              and e[form]["p99_ms"] <= budget_ms]
        return max(ok) if ok else 0

    matched = {}
    for budget_ms in (25, 50, 100):
        bp, bc, bn = best("plain", budget_ms), best("continuous", budget_ms), best("continuous_without_sharing",
                                                                                   budget_ms)
        matched[f"p99_le_{budget_ms}ms"] = {"plain_rate": bp, "continuous_rate": bc,
                                            "ratio": round(bc / bp, 3) if bp else None,
                                            "continuous_without_sharing_rate": bn,
                                            "ratio_without_sharing": round(bn / bp, 3) if bp else None}
    torch.cuda.synchronize()
    r = lambda d: {k: (round(v, 3) if isinstance(v, float) else v) for k, v in d.items()}
    return {"requests": n, "mix": dict(zip(serving.CLASSES, serving.MIX)), "table_rows": "log-uniform 10K-60M",
            "budget_gb": 40, "slots": 8,
            "saturation": {"plain": r(plain_sat), "continuous": r(cont_sat),
                           "throughput_ratio": round(cont_sat["queries_per_s"] / plain_sat["queries_per_s"], 3),
                           "continuous_without_sharing": r(cont_sat_noshare),
                           "throughput_ratio_without_sharing": round(
                               cont_sat_noshare["queries_per_s"] / plain_sat["queries_per_s"], 3)},
            "open_loop": {"arrival_rate_per_s": round(rate, 1), "plain": r(plain_open), "continuous": r(cont_open)},
            "rate_sweep": sweep, "matched_p99": matched}


def reference_gpu_kernels() -> dict:
    """The reference's own GPU kernels (its src/kernels built for sm_100a into
    oracle/_ref/libyqref.so) timed on this GPU with CUDA events, on the config
    workloads in the reference's own batch shapes. Its filter compaction and
    radix sort are not run (their prefix-sum kernels shift by 32 or more bits and
    faulted on this GPU); the timed sequences leave out the reference's per-batch
    allocations and host syncs, which favours the reference."""
    import torch
    from yallasql_b200 import datagen
    path = os.path.join(ROOT, "oracle", "_ref", "libyqref.so")
    if not torch.cuda.is_available() or not os.path.exists(path):
        return {"unavailable": "no GPU or oracle/_ref/libyqref.so not built"}
    L = C.CDLL(path)
    vp, u32, i32, fp = C.c_void_p, C.c_uint32, C.c_int, C.POINTER(C.c_float)
    L.ref_time_aggregate.argtypes = [vp, vp, vp, u32, u32, vp, vp, vp, i32, fp]
    L.ref_time_merge_window.argtypes = [vp, vp, u32, vp, vp, vp, vp, i32, fp]
    L.ref_time_join_batch.argtypes = [vp, u32, vp, u32, vp, vp, i32, fp]
    L.ref_time_cross.argtypes = [vp, vp, u32, vp, vp, u32, u32, vp, vp, vp, vp, i32, fp]
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    ms = C.c_float()
    out = {}

    def check(rc, what):
        if rc != 0:
            raise RuntimeError(f"{what}: CUDA error {rc}")

    # filter+aggregate query's aggregates (cast, mul, SUM/MIN/MAX/COUNT per 15,616-row batch: 268 B/row layout)
    for rows, name in ((1_000_000, "aggregate_1M"), (64_000_000, "aggregate_64M")):
        t = datagen.sales_table(rows, seed=0)
        price, disc = dev(t["price"]), dev(t["discount"])
        nulls = torch.zeros(rows, dtype=torch.uint8, device="cuda")
        fd, prod = torch.empty(rows, dtype=torch.float32, device="cuda"), torch.empty(rows, dtype=torch.float32,
                                                                                         device="cuda")
        acc = torch.zeros(8, dtype=torch.int32, device="cuda")
        check(L.ref_time_aggregate(price.data_ptr(), disc.data_ptr(), nulls.data_ptr(), rows, 15_616, fd.data_ptr(),
                                   prod.data_ptr(), acc.data_ptr(), 3 if rows > 1_000_000 else 10, C.byref(ms)), name)
        out[name] = {"rows": rows, "batch_rows": 15_616, "ms": round(ms.value, 4),
                     "rows_per_s": rows / (ms.value / 1e3),
                     "launches": "cast, mul, reduction_sum_wrap SUM/MIN/MAX, reduction_count_notnull per batch",
                     "note": "no WHERE compaction (the reference's prefix-sum kernels are not run): aggregates over "
                             "every row"}
        del t, price, disc, nulls, fd, prod
    # ORDER BY merge: one 15,360-row window (272 B/row layout) of merge_sorted_array_kernel_v1
    w = 15_360
    rng = np.random.default_rng(1)
    a = -np.sort(-rng.uniform(-1e6, 1e6, w).astype(np.float32))
    b = -np.sort(-rng.uniform(-1e6, 1e6, w).astype(np.float32))
    da, db = dev(a), dev(b)
    c = torch.empty(w, dtype=torch.float32, device="cuda")
    idx = torch.empty(w, dtype=torch.int32, device="cuda")
    fa = torch.empty(w, dtype=torch.uint8, device="cuda")
    la = torch.zeros(1, dtype=torch.int32, device="cuda")
    check(L.ref_time_merge_window(da.data_ptr(), db.data_ptr(), w, c.data_ptr(), idx.data_ptr(), fa.data_ptr(),
                                  la.data_ptr(), 200, C.byref(ms)), "merge")
    runs = -(-64_000_000 // w)
    levels = int(np.ceil(np.log2(runs)))
    out["merge_window_15360"] = {"window_rows": w, "ms_per_window": round(ms.value, 5),
                                 "merged_rows_per_s": w / (ms.value / 1e3),
                                 "orderby_64M_merge_phase_ms_est": round(levels * (64_000_000 / w) * ms.value, 1),
                                 "estimate": f"{levels} merge levels x 64M rows / {w}-row windows x the window's "
                                             "kernel time (key merge only; the host loop, its blocking copies and "
                                             "the per-window column moves not counted)"}
    # star join: one 262,144-row fact batch (16 B/row layout) x the 2,556-row date table
    fact, dim = datagen.star_tables(262_144, seed=2)
    fk, dk = dev(fact["datekey"]), dev(dim["datekey"])
    pairs = torch.empty(2 * 1_048_576, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    check(L.ref_time_join_batch(fk.data_ptr(), 262_144, dk.data_ptr(), 2556, pairs.data_ptr(), cnt.data_ptr(), 5,
                                C.byref(ms)), "join")
    nb = -(-60_000_000 // 262_144)
    out["join_batch_262144x2556"] = {"ms_per_batch": round(ms.value, 4), "pairs_per_batch": int(cnt.item()),
                                     "star_join_60M_join_phase_ms_est": round(nb * ms.value, 1),
                                     "estimate": f"{nb} fact batches x the batch's outer_join_batches time (the "
                                                 "pair gathers, filters and the aggregate not counted)"}
    # cross product 20K x 20K, right side in 256-row chunks
    x, y = datagen.cross_tables(20_000, seed=2)
    dx, dy = dev(x), dev(y)
    zn = torch.zeros(20_000, dtype=torch.uint8, device="cuda")
    ol, orr = (torch.empty(20_000 * 256, dtype=torch.int32, device="cuda") for _ in range(2))
    oln, orn = (torch.empty(20_000 * 256, dtype=torch.uint8, device="cuda") for _ in range(2))
    check(L.ref_time_cross(dx.data_ptr(), zn.data_ptr(), 20_000, dy.data_ptr(), zn.data_ptr(), 20_000, 256,
                           ol.data_ptr(), oln.data_ptr(), orr.data_ptr(), orn.data_ptr(), 2, C.byref(ms)), "cross")
    out["cross_product_20Kx20K"] = {"ms": round(ms.value, 3), "output_rows": 400_000_000,
                                    "note": "materialisation only (both columns + null bytes, 256-row right chunks); "
                                            "the reference then filters a.x < b.y with its compaction, not run"}
    torch.cuda.synchronize()
    return out


def run_reference(args, rank: int):
    """Reference arm: the CPU port of the operator (oracle/ stable ORDER BY +
    row gather), all host threads, the whole table every step (a sample
    would flatter an N log N sort; a 64M-row step takes seconds)."""
    import oracle
    threads = os.cpu_count() or 1
    sample = args.rows
    t = make_table(sample, args.dist)

    def one():
        for key, desc in (("key", True), ("d", False)):
            perm = oracle.sort_perm(t[key], desc=desc, threads=threads,
                                    type_=oracle.DATETIME if key == "d" else None)
            for name in ("key", "id", "txt", "d"):
                np.take(t[name], perm, axis=0)

    for _ in range(args.warmup):
        one()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        one()
    dt = (time.perf_counter() - t0) / args.steps
    value = 2 * sample / dt
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 keys, int64/text/date payload",
            "data": "synthetic", "config": config(args),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"the whole {sample}-row table, both ORDER BY queries per step"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if rank == 0 and not args.no_ops:
        try:
            line["reference_gpu"] = reference_gpu_kernels()
        except Exception as ex:  # the CPU figure above stands on its own
            line["reference_gpu"] = {"unavailable": f"{type(ex).__name__}: {ex}"}
    if rank == 0:
        print(json.dumps(line))


def config(args) -> dict:
    return {"workload": f"ORDER BY key DESC then ORDER BY d ASC on a {args.rows}-row table (key f32 {args.dist}, "
                        f"id int64, txt 16-byte, d date; seed 1), {args.mode}"
                        + (" as 4 MB batches sorted then merge-path merged" if args.mode == "outofcore" else ""),
            "rows": args.rows, "row_bytes": ROW_BYTES, "key_distribution": args.dist, "mode": args.mode,
            "l2": "inputs larger than L2 (64M rows x 36 B = 2.3 GB per table)", "parallelism": f"replicas x{args.gpus}"}


def cpu_baseline(args, t: dict) -> dict:
    import oracle
    threads = os.cpu_count() or 1
    sample = min(args.rows, 8_000_000)
    sub = {k: v[:sample] for k, v in t.items()}
    t0 = time.perf_counter()
    for key, desc in (("key", True), ("d", False)):
        perm = oracle.sort_perm(sub[key], desc=desc, threads=threads, type_=oracle.DATETIME if key == "d" else None)
        for name in ("key", "id", "txt", "d"):
            np.take(sub[name], perm, axis=0)
    dt = time.perf_counter() - t0
    return {"value": 2 * sample / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"first {sample} of {args.rows} rows, both ORDER BY queries (stable sort + gather of 4 columns)"}


QUERIES = (("key", True), ("d", False))
COLUMNS = ("key", "id", "txt", "d")


def host_outputs(job) -> list:
    """The device results of the last step, copied to host memory (one list of columns per query)."""
    return [[c.data.cpu().numpy() for c in out.columns] for out in job.out]


def oracle_parity(t: dict, outs: list) -> dict:
    """CPU check of a timed step's results (part of the CPU-baseline leg): every
    column of both queries against the oracle's stable sort + gather of the whole table."""
    import oracle
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    bad = []
    for (key, desc), cols in zip(QUERIES, outs):
        perm = oracle.sort_perm(t[key], desc=desc, threads=threads, type_=oracle.DATETIME if key == "d" else None)
        for name, got in zip(COLUMNS, cols):
            if not np.array_equal(got, np.take(t[name], perm, axis=0)):
                bad.append(f"ORDER BY {key}: {name}")
        del perm
    return {"ok": not bad, "mismatched": bad, "rows": int(t["key"].shape[0]), "check_s": round(time.perf_counter() - t0, 1),
            "what": "every column of both queries' output in the last timed step against the oracle's stable sort "
                    "+ gather of the whole table (bit-exact, stable tie order)"}


def other_distribution(args, dist: str, check: bool) -> dict:
    """The same two ORDER BY queries over a table whose key follows `dist` (the
    config's other key distributions): device ms per step and parity of the last
    timed step's output."""
    import torch
    t = make_table(args.rows, dist)
    job = OrderByJob(t, args.mode)
    for _ in range(args.warmup):
        job.step()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(args.steps):
        job.step()
    e.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(e) / args.steps
    out = {"ms_per_step": round(ms, 3), "value": 2 * args.rows / (ms / 1e3), "unit": UNIT,
           "steps": args.steps, "warmup": args.warmup}
    if check:
        outs = host_outputs(job)
        del job
        torch.cuda.empty_cache()
        out["parity"] = oracle_parity(t, outs)
    return out


def max_over_ranks(ms: float, dist, device="cuda") -> float:
    """Step time of the whole job: the slowest rank's (every rank calls this)."""
    if dist is None:
        return ms
    import torch
    tt = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def whole_job_rows_per_s(world: int, rows_per_step: int, ms: float) -> float:
    """Units all ranks processed (weak scaling: each rank runs the full workload) / the slowest rank's time."""
    return world * rows_per_step / (ms / 1e3)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args, rank)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    from yallasql_b200 import _abi as A
    lib = A.load()
    t = make_table(args.rows, args.dist)
    job = OrderByJob(t, args.mode)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        job.step()
    barrier()
    launches0 = lib.yq_launch_count()
    lib.yq_profile_enable(1)
    lib.yq_profile_read(None, 0, 1)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        s.record()
        for _ in range(args.steps):
            job.step()
        e.record()
        torch.cuda.synchronize()
    lib.yq_profile_enable(0)
    buf = C.create_string_buffer(1 << 16)
    lib.yq_profile_read(buf, len(buf), 1)
    prof = json.loads(buf.value.decode() or "{}")
    launches = int(lib.yq_launch_count() - launches0)
    ms = max_over_ranks(s.elapsed_time(e) / args.steps, dist)
    rows_per_step = 2 * args.rows
    value = whole_job_rows_per_s(world, rows_per_step, ms)

    # the last timed step's results, kept for the oracle check of the CPU-baseline leg
    timed_outs = host_outputs(job) if rank == 0 and not args.no_cpu else None

    # end to end: pinned host table -> device -> both queries -> host (every
    # step). Three streams pipeline the steps: the table of step i+1 goes to
    # the device while step i computes and its results come back, query A's
    # result goes back while query B runs (the link's two directions overlap),
    # and the device tables and results are double-buffered.
    e2e = None
    if not args.no_e2e:
        from yallasql_b200.ops import DeviceBatch, DeviceColumn
        pin = {k: torch.from_numpy(v).pin_memory() for k, v in t.items()}
        outs = [{k: torch.empty_like(v).pin_memory() for k, v in pin.items()} for _ in range(2)]
        names = ("key", "id", "txt", "d")
        like = lambda bt: DeviceBatch([DeviceColumn(torch.empty_like(c.data), c.type) for c in bt.columns])
        stages = [job.table, like(job.table)]  # device tables, refilled from host memory every step
        dev_out = [job.out, [like(o) for o in job.out]]
        s_in, s_cmp, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
        ev = {k: [torch.cuda.Event(), torch.cuda.Event()] for k in ("staged", "a", "read", "done")}

        chunk = 64 << 20

        def copy_chunked(dst, src):
            # bulk copies go in 64 MB pieces: the operators' own small transfers
            # (histogram read-back, merge-pair uploads, error words) share the
            # copy engines and would otherwise queue behind a multi-GB copy
            d, h = dst.view(-1).view(torch.uint8), src.view(-1).view(torch.uint8)
            for o in range(0, d.numel(), chunk):
                d[o:o + chunk].copy_(h[o:o + chunk], non_blocking=True)

        def stage_in(i):
            k = i & 1
            s_in.wait_event(ev["read"][k])  # step i-2 no longer reads this table
            with torch.cuda.stream(s_in):
                for c, n in zip(stages[k].columns, names):
                    copy_chunked(c.data, pin[n])
                ev["staged"][k].record(s_in)

        def compute_out(i):
            k = i & 1
            st, (oa, ob) = stages[k], dev_out[k]
            s_cmp.wait_event(ev["staged"][k])
            s_cmp.wait_event(ev["done"][k])  # step i-2's results are back on the host
            with torch.cuda.stream(s_cmp):
                job.query(st, 0, True, oa)
                ev["a"][k].record(s_cmp)
                job.query(st, 3, False, ob)
                ev["read"][k].record(s_cmp)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev["a"][k])
                for c, n in zip(oa.columns, names):
                    copy_chunked(outs[0][n], c.data)
                s_out.wait_event(ev["read"][k])
                for c, n in zip(ob.columns, names):
                    copy_chunked(outs[1][n], c.data)
                ev["done"][k].record(s_out)

        def e2e_run(nsteps):
            # the next step's table is on its way in before this step's queries
            # run: the ORDER BY calls return only once their stream is done, so
            # the copy is issued first and overlaps them and the copies out
            stage_in(0)
            for i in range(nsteps):
                if i + 1 < nsteps:
                    stage_in(i + 1)
                compute_out(i)

        def around(first: bool):
            cur = torch.cuda.current_stream()
            for q in (s_in, s_cmp, s_out):
                if first:
                    q.wait_stream(cur)
                else:
                    cur.wait_stream(q)

        around(True)
        e2e_run(max(1, args.warmup // 2))
        around(False)
        barrier()
        s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s2.record()
        around(True)
        e2e_run(args.steps)
        around(False)
        e2.record()
        torch.cuda.synchronize()
        ms2 = max_over_ranks(s2.elapsed_time(e2) / args.steps, dist)
        tab_bytes = sum(v.nbytes for v in t.values())
        e2e = {"value": whole_job_rows_per_s(world, rows_per_step, ms2), "unit": UNIT, "h2d_bytes_per_step": tab_bytes,
               "d2h_bytes_per_step": 2 * tab_bytes, "ms_per_step": ms2,
               "path": "pinned host columns -> cudaMemcpyAsync -> C-ABI operators -> pinned host, every step; "
                       "copies in, compute and copies out on three streams, steps double-buffered, the next "
                       "step's copy in issued before this step's queries, bulk copies in 64 MB pieces"}
        del stages, dev_out, pin, outs

    peak, peak_kind = peaks()
    roof = None
    if prof:
        dom = max(prof.items(), key=lambda kv: kv[1]["ms"])
        name, d = dom
        per_launch_bytes = d["units"] / max(1, d["launches"])
        per_launch_ms = d["ms"] / max(1, d["launches"])
        achieved = per_launch_bytes / (per_launch_ms / 1e3) / 1e9
        tr = committed_traffic().get(name, {})
        traffic = None
        if tr.get("dram_bytes") and tr.get("algorithmic_bytes"):
            # ncu capture of a smaller case of the same kernel, scaled by the units this launch processes
            traffic = round(tr["dram_bytes"] / tr["algorithmic_bytes"] * per_launch_bytes)
        roof = {"bound": "hbm", "kernel": name, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                if peak_kind == "measured" else "fallback 6650 GB/s",
                "traffic": traffic, "algorithmic_bytes_per_launch": per_launch_bytes,
                "avg_launch_ms": round(per_launch_ms, 4)}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 keys, int64/text/date payload", "data": "synthetic",
            "config": config(args), "roofline": roof, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk.summary(), "kernels": prof}
    del job
    torch.cuda.empty_cache()
    if timed_outs is not None:
        line["parity"] = oracle_parity(t, timed_outs)
        del timed_outs
    if rank == 0 and not args.no_dists:
        line["distributions"] = {d: other_distribution(args, d, check=not args.no_cpu)
                                 for d in ("uniform", "zipf", "equal") if d != args.dist}
        torch.cuda.empty_cache()
    if rank == 0 and not args.no_ops:
        line["operators"] = operator_suite(lib, peak)
        line["operators"]["csv_scan_8M"] = csv_suite(lib, peak)
    if rank == 0 and not args.no_batched:
        torch.cuda.empty_cache()
        line["batched"] = batched_form(args)
    if rank == 0 and not args.no_serving:
        torch.cuda.empty_cache()
        line["serving"] = serving_form(args)
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(args, t)
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
