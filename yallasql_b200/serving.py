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
MAX_GROUP = 64  # filter requests co-launched in one segmented call at most
MIX = (0.4, 0.3, 0.2, 0.1)
ORDER_TYPES = [A.FLOAT32, A.INT64, A.TEXT, A.DATETIME]
ORDER_WIDTHS = [4, 8, 16, 8]
THRESHOLD_MARK = -3.0e38  # placeholder of the subquery's threshold in its compiled plan
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


def warm_trace(catalog: Catalog) -> list[Request]:
    """Every request class on every table, with two parameters each, all
    arriving at once. Each distinct expression program compiles its kernel
    once per variant (staged or not, by size), so serving this trace before a
    timed run keeps compilations out of it."""
    out = []
    for k in CLASSES:
        for t in range(catalog.ntables):
            for c in (0, 1):
                out.append(Request(len(out), k, t, 0.0, c))
    return out


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
        self.rows_gt = {}  # stage 2 of the subquery per category, its threshold patched per request
        mark = Constant(THRESHOLD_MARK, A.FLOAT32)
        for c in range(len(datagen.CATEGORIES)):
            eq = Compare(A.EQ, ColumnRef(3, A.TEXT), Constant(datagen.CATEGORIES[c], A.TEXT))
            self.avg[c] = ops.AggPlan(SALES_TYPES, eq, [Aggregate(A.AGG_AVG, self.revenue)])
            plan = ops.ProjectPlan(SALES_TYPES, [4, 4, 4, 16], And(eq, Compare(A.GT, self.revenue, mark)),
                                   [self.revenue, 1])
            slot = [w for _, w in plan.pool.words].index(mark.word())
            self.rows_gt[c] = (plan, slot)
        # AVG over no rows is NULL, so no row qualifies: a predicate false on every row
        self.rows_none = ops.ProjectPlan(SALES_TYPES, [4, 4, 4, 16],
                                         Compare(A.NE, ColumnRef(1, A.INT32), ColumnRef(1, A.INT32)),
                                         [self.revenue, 1])
        self.order_cfg = ops.sort_config(digit_bits=0, keep_trivial=True)
        self.join_dim = None
        self._join_dim_of = None

    def prepared_dim(self, cat: "Catalog") -> ops.PreparedDim:
        """The join's dimension side (date rows of year 1993, hashed), built once
        per catalog and kept resident for every join request."""
        if self._join_dim_of is not cat:
            self.join_dim = self.join.prepare(cat.dim)
            self._join_dim_of = cat
        return self.join_dim

    def subquery_rows_plan(self, category: int, avg) -> ops.ProjectPlan:
        """Stage 2 of the subquery: category = c AND revenue > avg (the compiled
        plan of category c with `avg` written into its threshold constant)."""
        if avg is None:
            return self.rows_none
        plan, slot = self.rows_gt[category]
        plan._keep[0][slot] = Constant(float(np.float32(avg)), A.FLOAT32).word()
        return plan


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
        self._states = None

    def ensure(self, plans: "Plans | None" = None):
        """Allocate the buffers now (before a timed run)."""
        self.order(0, 0)
        self.subquery(0)
        if plans is not None:
            self.states(plans)
        return self

    def states(self, plans: "Plans"):
        """Aggregate states and workspaces the slot reuses: up to MAX_GROUP
        co-launched filter states, one join state with its probe workspace, one
        subquery AVG state and the subquery's row counter."""
        if self._states is None:
            jws = torch.empty(max(256, int(ops.lib().yq_join_aggregate_prepared_workspace_size(
                len(plans.join.aggs)))), dtype=torch.uint8, device="cuda")
            self._states = {"filter": ops.AggStates(plans.aggs, MAX_GROUP), "join": ops.AggState(plans.join.aggs),
                            "join_ws": jws, "avg": ops.AggState(plans.avg[0].aggs),
                            "count": torch.zeros(1, dtype=torch.int32, device="cuda")}
        return self._states

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
    """Filter requests co-launched as one segmented filter+aggregate over their
    tables' row ranges. With `shared`, requests on the same table share one
    range (the query has no parameters: their results are the same)."""

    def __init__(self, cat: Catalog, plans: Plans, reqs: list[Request], shared: bool = False):
        self.cat, self.plans, self.reqs = cat, plans, reqs
        tables = []
        self.slot_of = []
        for r in reqs:
            if not shared or r.table not in tables:
                tables.append(r.table)
            self.slot_of.append(tables.index(r.table) if shared else len(tables) - 1)
        self.begin = [cat.sales_begin[t] for t in tables]
        self.end = [cat.sales_end[t] for t in tables]
        self.mem = 256 * len(tables) + 8 * sum(e - b for b, e in zip(self.begin, self.end)) // 1024 + (1 << 16)

    def launch(self, stream, bufs=None):
        self.stream = stream
        n = len(self.begin)
        with torch.cuda.stream(stream):
            if bufs is not None and n <= MAX_GROUP:
                self.states = bufs.states(self.plans)["filter"]
                self.states.reset(stream.cuda_stream, count=n)
            else:
                self.states = ops.AggStates(self.plans.aggs, n, stream=stream.cuda_stream)
            self.plans.filter.run_ranges(self.cat.arena, self.begin, self.end, self.states, stream=stream.cuda_stream)
            self.event = torch.cuda.Event()
            self.event.record(stream)

    def finish(self):
        res = self.states.read(self.stream, count=len(self.begin))
        for r, k in zip(self.reqs, self.slot_of):
            r.result = res[k]
        self.states = None


class OrderJob(Job):
    """ORDER BY key DESC over one table. With `perms` (the serving loop's
    resident intermediates), the first request on a table keeps its sort
    permutation; later ones wait for it and only gather."""

    def __init__(self, cat: Catalog, plans: Plans, req: Request, keep: bool, perms: dict | None = None):
        self.cat, self.plans, self.reqs, self.keep = cat, plans, [req], keep
        self.tbl = cat.order[req.table]
        self.perms = perms
        n = self.tbl.rows
        self.offs = (C.c_uint32 * 2)(0, n)
        self.ws_bytes = max(256, ops.order_by_segments_workspace_bytes(self.tbl.columns[0], [0, n]))
        self.mem = 36 * n + self.ws_bytes
        self.gather_only = perms is not None and req.table in perms

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
            t = self.reqs[0].table
            if self.gather_only:
                perm, ready = self.perms[t]
                stream.wait_event(ready)  # the permutation's sort may still run on another stream
                ops.gather(self.tbl, perm, stream=stream.cuda_stream, out=self.out)
            elif self.perms is not None:
                perm = torch.empty(n, dtype=torch.int32, device="cuda")
                ops.order_by_segments(self.tbl, 0, True, self.offs, self.out, config=self.plans.order_cfg,
                                      workspace=self.ws, stream=stream.cuda_stream, perm_out=perm)
                ready = torch.cuda.Event()
                ready.record(stream)
                self.perms[t] = (perm, ready)
            else:
                ops.order_by_segments(self.tbl, 0, True, self.offs, self.out, config=self.plans.order_cfg,
                                      workspace=self.ws, stream=stream.cuda_stream)
            self.event = torch.cuda.Event()
            self.event.record(stream)

    def finish(self):
        if not self.gather_only:
            with torch.cuda.stream(self.stream):
                err = int(self.ws[:4].view(torch.int32)[0].item())
            if err:
                raise RuntimeError(f"ORDER BY request {self.reqs[0].rid}: device error word {err}")
        for r in self.reqs:
            r.result = self.out if self.keep else ("ok", self.tbl.rows)
        self.out = self.ws = None


class JoinJob(Job):
    def __init__(self, cat: Catalog, plans: Plans, req: Request):
        self.cat, self.plans, self.reqs = cat, plans, [req]
        self.mem = 1 << 20

    def launch(self, stream, bufs=None):
        self.stream = stream
        with torch.cuda.stream(stream):
            fact = self.cat.facts[self.reqs[0].table]
            if bufs is not None:  # the slot's state, the resident dimension table: no host wait
                st = bufs.states(self.plans)
                self.state = st["join"]
                self.state.reset(stream.cuda_stream)
                self.plans.join.run_prepared(fact, self.plans.prepared_dim(self.cat), self.state,
                                             stream=stream.cuda_stream, workspace=st["join_ws"])
            else:
                self.state = ops.AggState(self.plans.join.aggs, stream=stream.cuda_stream)
                self.plans.join.run(fact, self.cat.dim, self.state, stream=stream.cuda_stream)
            self.event = torch.cuda.Event()
            self.event.record(stream)

    def finish(self):
        res = self.state.read(self.stream)
        for r in self.reqs:
            r.result = res
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
            if bufs is not None:
                self.state = bufs.states(self.plans)["avg"]
                self.state.reset(stream.cuda_stream)
            else:
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
        # AVG over no rows is NULL: then no row qualifies (the comparison is NULL)
        self.plan = p.subquery_rows_plan(self.reqs[0].param, self.avg)
        n = max(1, self.tbl.rows)
        self.stream = stream
        with torch.cuda.stream(stream):
            if bufs is not None and not self.first.keep:
                self.outs = bufs.subquery(n)
                self.cnt = bufs.states(p)["count"]
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
                res = (n, self.outs[0].data[:n].clone(), self.outs[1].data[:n].clone())
            else:
                res = (n,)
            for r in self.reqs:
                r.result = res
        self.outs = None


def make_job(cat, plans, req: Request, keep: bool, perms: dict | None = None) -> Job:
    if req.klass == "order":
        return OrderJob(cat, plans, req, keep, perms)
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
    bufs = cat.slot_buffers(0).ensure(plans)
    plans.prepared_dim(cat)
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
                     max_group: int = MAX_GROUP, keep: bool = False, share: bool = True) -> dict:
    """Admit requests as streams and budget free up; overlap their work on the
    device; co-launch pending filter requests as one segmented launch.

    With `share` (the default) the loop also shares work between requests:
    pending requests identical to the one being dispatched (same class, table
    and parameter) ride on its dispatch and complete with it; co-launched
    filter requests on one table share one scan; and the sort permutation of
    each ORDER BY table is kept resident (counted in the budget) once a request
    has sorted it, so later ORDER BY requests on that table only gather."""
    streams = [torch.cuda.Stream() for _ in range(slots)]
    perms: dict | None = {} if share else None
    for sl in range(slots):
        cat.slot_buffers(sl).ensure(plans)
    plans.prepared_dim(cat)
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
                    group = [r for r in pending if r.klass == "filter"]
                    if not share:
                        group = group[:max_group]
                    job = FilterGroup(cat, plans, group, shared=share)
                    if len(job.begin) > max_group:  # more distinct tables than states: the first max_group
                        keep_t = set(sorted({r.table for r in group}, key=[r.table for r in group].index)[:max_group])
                        job = FilterGroup(cat, plans, [r for r in group if r.table in keep_t], shared=share)
                else:
                    job = make_job(cat, plans, head, keep, perms)
                    if share:  # identical pending requests complete with this one
                        key = (head.klass, head.table, head.param)
                        job.reqs = [r for r in pending if (r.klass, r.table, r.param) == key]
            if used + job.mem > budget and inflight:
                break  # wait for memory (first-come first-served)
            if ready and job is ready[0]:
                ready.popleft()
            else:
                ids = {id(r) for r in job.reqs}
                pending = deque(r for r in pending if id(r) not in ids)
            sl = free.pop()
            had = set(perms) if perms is not None else None
            job.launch(streams[sl], cat.slot_buffers(sl))
            if perms is not None and len(perms) > len(had):  # a permutation became resident
                used += 4.0 * job.tbl.rows
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
