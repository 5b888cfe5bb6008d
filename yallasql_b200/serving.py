"""Serving form: a request loop with continuous batching over resident tables.

Requests arrive as a Poisson stream (seed 4) with a 40/30/20/10 mix of
  filter    - SUM(price*discount), COUNT(*), MIN(price), MAX(price) WHERE the
              sales predicate, over one sales table;
  order     - ORDER BY key DESC over one order table (four columns move);
  join      - SUM(extendedprice*discount) over fact JOIN date ON datekey WHERE
              year = 1993 AND discount BETWEEN 1 AND 3 AND quantity < 25;
  subquery  - the rows WHERE category = c AND price*discount >
              (SELECT AVG(price*discount) WHERE category = c), projected as
              (price*discount, qty);
over tables whose sizes are log-uniform in [lo, hi] rows. Every table stays
resident in HBM for the whole run (the sales tables back to back in one
arena), so a request only allocates its outputs and workspace.

Plain form: one request at a time, in arrival order, on one stream.
Continuous form: requests are admitted as soon as a slot (a CUDA stream) and
the device-memory budget allow; their work overlaps on the device; all
pending filter requests are co-launched as one segmented launch over their
tables' row ranges; a subquery's second stage is dispatched when its first
completes. Latency = completion - arrival, measured on the host clock; a
completion is seen by polling each request's CUDA event.
"""
from __future__ import annotations

import ctypes as C
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _abi as A
from . import batched, datagen, ops
from .expr import Aggregate, And, Arith, Cast, ColumnRef, Compare, Constant, between

CLASSES = ("filter", "order", "join", "subquery")
MIX = (0.4, 0.3, 0.2, 0.1)
ORDER_TYPES = [A.FLOAT32, A.INT64, A.TEXT, A.DATETIME]
ORDER_WIDTHS = [4, 8, 16, 8]
SALES_TYPES = [A.FLOAT32, A.INT32, A.INT32, A.TEXT]  # price qty discount category


def log_uniform(rng, n, lo, hi):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.int64)


class Catalog:
    """Resident tables: `ntables` per query class."""

    def __init__(self, ntables: int = 8, lo: int = 10_000, hi: int = 60_000_000, seed: int = 4):
        rng = np.random.Generator(np.random.PCG64(seed))
        g = torch.Generator(device="cuda")
        g.manual_seed(seed)
        # sales arena: filter tables then subquery tables
        self.sales_rows = [int(x) for x in log_uniform(rng, 2 * ntables, lo, hi)]
        offs = [0] + list(np.cumsum(self.sales_rows).astype(int))
        self.sales_begin, self.sales_end = offs[:-1], offs[1:]
        s = batched._device_sales(offs[-1], seed)
        self.arena = ops.DeviceBatch([ops.DeviceColumn(s[k], t) for k, t in
                                      zip(["price", "qty", "discount", "category"], SALES_TYPES)])
        self.order = []
        for n in log_uniform(rng, ntables, lo, hi):
            n = int(n)
            key = torch.rand(n, generator=g, device="cuda") * 2e6 - 1e6
            txt = torch.randint(97, 123, (n, 16), generator=g, device="cuda", dtype=torch.uint8)
            txt[:, 15] = 0
            d = torch.randint(datagen.DATE_LO, datagen.DATE_HI + 1, (n,), generator=g, device="cuda",
                              dtype=torch.int64)
            self.order.append(ops.DeviceBatch([ops.DeviceColumn(key.to(torch.float32), A.FLOAT32),
                                               ops.DeviceColumn(torch.arange(n, dtype=torch.int64, device="cuda"),
                                                                A.INT64),
                                               ops.DeviceColumn(txt, A.TEXT), ops.DeviceColumn(d, A.DATETIME)]))
        self.facts = []
        for n in log_uniform(rng, ntables, lo, hi):
            n = int(n)
            self.facts.append(ops.DeviceBatch([
                ops.DeviceColumn(torch.randint(0, 2556, (n,), generator=g, device="cuda", dtype=torch.int32), A.INT32),
                ops.DeviceColumn(torch.randint(1, 51, (n,), generator=g, device="cuda", dtype=torch.int32), A.INT32),
                ops.DeviceColumn(torch.randint(0, 11, (n,), generator=g, device="cuda", dtype=torch.int32), A.INT32),
                ops.DeviceColumn((torch.rand(n, generator=g, device="cuda") * 104100 + 900).to(torch.float32),
                                 A.FLOAT32)]))
        _, dim = datagen.star_tables(1, seed=2)
        self.dim = ops.DeviceBatch([ops.DeviceColumn(torch.from_numpy(dim[k]).cuda(), A.INT32)
                                    for k in ("datekey", "year", "month")])
        self.ntables = ntables

    def slot_buffers(self, slot: int) -> SlotBuffers:
        """The reusable buffers of serving slot `slot` (created on first use)."""
        if not hasattr(self, "_slots"):
            self._slots = {}
        if slot not in self._slots:
            self._slots[slot] = SlotBuffers(self)
        return self._slots[slot]

    def sales_view(self, i: int) -> ops.DeviceBatch:
        return self.arena.slice(self.sales_begin[i], self.sales_end[i])

    def rows_of(self, klass: str, table: int) -> int:
        if klass == "filter":
            return self.sales_rows[table]
        if klass == "subquery":
            return self.sales_rows[self.ntables + table]
        if klass == "order":
            return self.order[table].rows
        return self.facts[table].rows


@dataclass
class Request:
    rid: int
    klass: str
    table: int
    arrival: float
    param: int = 0
    done: float = -1.0
    result: object = None


def make_trace(n: int, rate: float, catalog: Catalog, seed: int = 4) -> list[Request]:
    """n requests with exponential inter-arrival gaps (mean 1/rate seconds)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    gaps = rng.exponential(1.0 / rate, n) if rate > 0 else np.zeros(n)
    t = np.cumsum(gaps) - gaps[0]
    kinds = rng.choice(len(CLASSES), n, p=MIX)
    tables = rng.integers(0, catalog.ntables, n)
    cats = rng.integers(0, len(datagen.CATEGORIES), n)
    return [Request(i, CLASSES[k], int(tb), float(a), int(c)) for i, (k, tb, a, c) in
            enumerate(zip(kinds, tables, t, cats))]


class Plans:
    """Compiled programs shared by every request."""

    def __init__(self):
        pred, aggs = batched.sales_query()
        self.aggs = aggs
        self.filter = ops.AggPlan(SALES_TYPES, pred, aggs)
        self.join = ops.JoinAggPlan(
            [A.INT32] * 3 + [A.FLOAT32], [A.INT32] * 3,
            And(between(ColumnRef(2, A.INT32), Constant(1, A.INT32), Constant(3, A.INT32)),
                Compare(A.LT, ColumnRef(1, A.INT32), Constant(25, A.INT32))), 0,
            Compare(A.EQ, ColumnRef(1, A.INT32), Constant(1993, A.INT32)), 0,
            [Aggregate(A.AGG_SUM, Arith(A.MUL, ColumnRef(3, A.FLOAT32), Cast(ColumnRef(2, A.INT32), A.FLOAT32)))])
        self.revenue = Arith(A.MUL, ColumnRef(0, A.FLOAT32), Cast(ColumnRef(2, A.INT32), A.FLOAT32))
        self.avg = {}
        for c in range(len(datagen.CATEGORIES)):
            eq = Compare(A.EQ, ColumnRef(3, A.TEXT), Constant(datagen.CATEGORIES[c], A.TEXT))
            self.avg[c] = ops.AggPlan(SALES_TYPES, eq, [Aggregate(A.AGG_AVG, self.revenue)])
        self.order_cfg = ops.sort_config(digit_bits=0, keep_trivial=True)


# ------------------------------------------------------------------- jobs
class SlotBuffers:
    """Outputs and workspaces one slot (stream) reuses from request to request:
    an ORDER BY result and workspace sized for the largest order table and a
    subquery's projected columns sized for the largest sales table, allocated
    before the slot serves its first request. Requests then allocate nothing large on the
    request path (no allocator calls, no device-wide synchronisation from
    them); results that must outlive the request (keep=True) are allocated
    per request instead."""

    def __init__(self, cat: "Catalog"):
        self.cat = cat
        self._order = None
        self._sub = None

    def ensure(self):
        """Allocate both buffers now (before a timed run)."""
        self.order(0, 0)
        self.subquery(0)
        return self

    def order(self, n: int, ws_bytes: int):
        if self._order is None:
            nmax = max(t.rows for t in self.cat.order)
            out = ops.DeviceBatch([ops.DeviceColumn.empty(t, nmax, w if t == A.TEXT else None)
                                   for t, w in zip(ORDER_TYPES, ORDER_WIDTHS)])
            big = max(self.cat.order, key=lambda t: t.rows)
            wsb = max(256, ops.order_by_segments_workspace_bytes(big.columns[0], [0, big.rows]))
            self._order = (out, torch.empty(wsb, dtype=torch.uint8, device="cuda"))
        out, ws = self._order
        if n > out.rows or ws_bytes > ws.numel():
            raise ValueError("ORDER BY request larger than the slot's buffers")
        return out.slice(0, n), ws[:ws_bytes]

    def subquery(self, n: int):
        if self._sub is None:
            nmax = max(1, max(e - b for b, e in zip(self.cat.sales_begin, self.cat.sales_end)))
            self._sub = [ops.DeviceColumn.empty(A.FLOAT32, nmax), ops.DeviceColumn.empty(A.INT32, nmax)]
        if n > self._sub[0].rows:
            raise ValueError("subquery larger than the slot's buffers")
        return [c.slice(0, n) for c in self._sub]


class Job:
    """Device work of one dispatch on one stream; `event` fires when it is done."""
    mem = 0
    reqs: list = []

    def launch(self, stream: torch.cuda.Stream, bufs: "SlotBuffers | None" = None): ...

    def finish(self): ...

    def next_stage(self):
        return None


class FilterGroup(Job):
    def __init__(self, cat: Catalog, plans: Plans, reqs: list[Request]):
        self.cat, self.plans, self.reqs = cat, plans, reqs
        self.begin = [cat.sales_begin[r.table] for r in reqs]
        self.end = [cat.sales_end[r.table] for r in reqs]
        self.mem = 256 * len(reqs) + 8 * sum(e - b for b, e in zip(self.begin, self.end)) // 1024 + (1 << 16)

    def launch(self, stream, bufs=None):
        self.stream = stream
        with torch.cuda.stream(stream):
            self.states = ops.AggStates(self.plans.aggs, len(self.reqs), stream=stream.cuda_stream)
            self.plans.filter.run_ranges(self.cat.arena, self.begin, self.end, self.states, stream=stream.cuda_stream)
            self.event = torch.cuda.Event()
            self.event.record(stream)

    def finish(self):
        res = self.states.read(self.stream)
        for r, v in zip(self.reqs, res):
            r.result = v
        self.states = None


class OrderJob(Job):
    def __init__(self, cat: Catalog, plans: Plans, req: Request, keep: bool):
        self.cat, self.plans, self.reqs, self.keep = cat, plans, [req], keep
        self.tbl = cat.order[req.table]
        n = self.tbl.rows
        self.offs = (C.c_uint32 * 2)(0, n)
        self.ws_bytes = max(256, ops.order_by_segments_workspace_bytes(self.tbl.columns[0], [0, n]))
        self.mem = 36 * n + self.ws_bytes

    def launch(self, stream, bufs: SlotBuffers | None = None):
        n = self.tbl.rows
        self.stream = stream
        with torch.cuda.stream(stream):
            if bufs is not None and not self.keep:
                self.out, self.ws = bufs.order(n, self.ws_bytes)
            else:
                self.out = ops.DeviceBatch([ops.DeviceColumn.empty(t, n, w if t == A.TEXT else None)
                                            for t, w in zip(ORDER_TYPES, ORDER_WIDTHS)])
                self.ws = torch.empty(self.ws_bytes, dtype=torch.uint8, device="cuda")
            ops.order_by_segments(self.tbl, 0, True, self.offs, self.out, config=self.plans.order_cfg,
                                  workspace=self.ws, stream=stream.cuda_stream)
            self.event = torch.cuda.Event()
            self.event.record(stream)

    def finish(self):
        with torch.cuda.stream(self.stream):
            err = int(self.ws[:4].view(torch.int32)[0].item())
        if err:
            raise RuntimeError(f"ORDER BY request {self.reqs[0].rid}: device error word {err}")
        self.reqs[0].result = self.out if self.keep else ("ok", self.tbl.rows)
        self.out = self.ws = None


class JoinJob(Job):
    def __init__(self, cat: Catalog, plans: Plans, req: Request):
        self.cat, self.plans, self.reqs = cat, plans, [req]
        self.mem = 1 << 20

    def launch(self, stream, bufs=None):
        self.stream = stream
        with torch.cuda.stream(stream):
            self.state = ops.AggState(self.plans.join.aggs, stream=stream.cuda_stream)
            self.plans.join.run(self.cat.facts[self.reqs[0].table], self.cat.dim, self.state,
                                stream=stream.cuda_stream)
            self.event = torch.cuda.Event()
            self.event.record(stream)

    def finish(self):
        self.reqs[0].result = self.state.read(self.stream)
        self.state = None


class SubqueryJob(Job):
    """Stage 1: AVG(revenue) WHERE category = c. Stage 2 (SubqueryRows)."""

    def __init__(self, cat: Catalog, plans: Plans, req: Request, keep: bool):
        self.cat, self.plans, self.reqs, self.keep = cat, plans, [req], keep
        self.tbl = cat.sales_view(cat.ntables + req.table)
        self.mem = (1 << 20) + 8 * self.tbl.rows

    def launch(self, stream, bufs=None):
        self.stream = stream
        with torch.cuda.stream(stream):
            plan = self.plans.avg[self.reqs[0].param]
            self.state = ops.AggState(plan.aggs, stream=stream.cuda_stream)
            plan.run(self.tbl, self.state, stream=stream.cuda_stream)
            self.event = torch.cuda.Event()
            self.event.record(stream)

    def finish(self):
        self.avg = self.state.read(self.stream)[0]
        self.state = None

    def next_stage(self):
        return SubqueryRows(self, self.avg)


class SubqueryRows(Job):
    def __init__(self, first: SubqueryJob, avg):
        self.first, self.reqs, self.avg = first, first.reqs, avg
        self.tbl = first.tbl
        self.mem = 8 * self.tbl.rows + (1 << 20)

    def launch(self, stream, bufs=None):
        p = self.first.plans
        c = self.reqs[0].param
        eq = Compare(A.EQ, ColumnRef(3, A.TEXT), Constant(datagen.CATEGORIES[c], A.TEXT))
        # AVG over no rows is NULL: then no row qualifies (the comparison is NULL)
        thr = Constant(float(np.float32(self.avg)) if self.avg is not None else 0.0, A.FLOAT32)
        pred = And(eq, Compare(A.GT, p.revenue, thr)) if self.avg is not None else \
            And(eq, Compare(A.NE, ColumnRef(1, A.INT32), ColumnRef(1, A.INT32)))
        self.plan = ops.ProjectPlan(SALES_TYPES, [4, 4, 4, 16], pred, [p.revenue, 1])
        n = max(1, self.tbl.rows)
        self.stream = stream
        with torch.cuda.stream(stream):
            if bufs is not None and not self.first.keep:
                self.outs = bufs.subquery(n)
            else:
                self.outs = [ops.DeviceColumn.empty(A.FLOAT32, n), ops.DeviceColumn.empty(A.INT32, n)]
            self.cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
            oc = (A.Column * 2)(*[o.c() for o in self.outs])
            b, keep = self.tbl.c()
            self._keep = (oc, b, keep)
            cnt_ptr = C.cast(C.c_void_p(self.cnt.data_ptr()), C.POINTER(C.c_uint32))
            st = ops.lib().yq_filter_project(C.byref(b), C.byref(self.plan.pred.prog), C.byref(self.plan.consts),
                                             self.plan.proj, 2, oc, n, cnt_ptr, None, None, 0, stream.cuda_stream)
            ops._check(st, "yq_filter_project")
            self.event = torch.cuda.Event()
            self.event.record(stream)

    def finish(self):
        with torch.cuda.stream(self.stream):
            n = int(self.cnt.item())
            if self.first.keep:
                self.reqs[0].result = (n, self.outs[0].data[:n].clone(), self.outs[1].data[:n].clone())
            else:
                self.reqs[0].result = (n,)
        self.outs = None


def make_job(cat, plans, req: Request, keep: bool) -> Job:
    if req.klass == "order":
        return OrderJob(cat, plans, req, keep)
    if req.klass == "join":
        return JoinJob(cat, plans, req)
    if req.klass == "subquery":
        return SubqueryJob(cat, plans, req, keep)
    return FilterGroup(cat, plans, [req])


# ---------------------------------------------------------------- servers
def _wait_until(t0: float, at: float):
    while time.perf_counter() - t0 < at:
        pass


def serve_plain(trace: list[Request], cat: Catalog, plans: Plans, keep: bool = False) -> dict:
    """One request at a time, in arrival order, on one stream."""
    stream = torch.cuda.Stream()
    bufs = cat.slot_buffers(0).ensure()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r in trace:
        _wait_until(t0, r.arrival)
        job = make_job(cat, plans, r, keep)
        while job is not None:
            job.launch(stream, bufs)
            job.event.synchronize()
            job.finish()
            job = job.next_stage()
        r.done = time.perf_counter() - t0
    return summary(trace)


def serve_continuous(trace: list[Request], cat: Catalog, plans: Plans, slots: int = 8, budget: float = 40e9,
                     max_group: int = 64, keep: bool = False) -> dict:
    """Admit requests as streams and budget free up; overlap their work on the
    device; co-launch pending filter requests as one segmented launch."""
    streams = [torch.cuda.Stream() for _ in range(slots)]
    for sl in range(slots):
        cat.slot_buffers(sl).ensure()
    free = list(range(slots))
    pending: deque[Request] = deque()
    ready: deque[Job] = deque()  # later stages of admitted requests (go first)
    inflight: list[tuple[Job, int]] = []
    used = 0.0
    i = 0
    n = len(trace)
    finished = 0
    peak_inflight = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    while finished < n:
        now = time.perf_counter() - t0
        while i < n and trace[i].arrival <= now:
            pending.append(trace[i])
            i += 1
        progressed = False
        still = []
        for job, sl in inflight:
            if job.event.query():
                job.finish()
                used -= job.mem
                free.append(sl)
                nxt = job.next_stage()
                if nxt is not None:
                    ready.append(nxt)
                else:
                    t = time.perf_counter() - t0
                    for r in job.reqs:
                        r.done = t
                        finished += 1
                progressed = True
            else:
                still.append((job, sl))
        inflight = still
        while free and (ready or pending):
            if ready:
                job = ready[0]
            else:
                head = pending[0]
                if head.klass == "filter":
                    group = [r for r in pending if r.klass == "filter"][:max_group]
                    job = FilterGroup(cat, plans, group)
                else:
                    job = make_job(cat, plans, head, keep)
            if used + job.mem > budget and inflight:
                break  # wait for memory (first-come first-served)
            if ready and job is ready[0]:
                ready.popleft()
            elif isinstance(job, FilterGroup):
                ids = {id(r) for r in job.reqs}
                pending = deque(r for r in pending if id(r) not in ids)
            else:
                pending.popleft()
            sl = free.pop()
            job.launch(streams[sl], cat.slot_buffers(sl))
            used += job.mem
            inflight.append((job, sl))
            peak_inflight = max(peak_inflight, len(inflight))
            progressed = True
        if not progressed:
            time.sleep(0)
    out = summary(trace)
    out["peak_inflight"] = peak_inflight
    return out


def summary(trace: list[Request]) -> dict:
    lat = np.array([(r.done - r.arrival) * 1e3 for r in trace])
    span = max(r.done for r in trace) - min(r.arrival for r in trace)
    return {"queries": len(trace), "queries_per_s": len(trace) / span if span > 0 else float("inf"),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "span_s": span}
