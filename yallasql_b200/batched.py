"""Batched form: hundreds of independent filter+aggregate and ORDER BY tasks.

Task row counts are log-uniform in [lo, hi] (seeded). Even tasks run the
filter+aggregate query of the sales table (SUM(price*discount), COUNT(*),
MIN(price), MAX(price) WHERE discount BETWEEN 1 AND 3 AND qty < 25 AND
category <> 'category_007'); odd tasks run ORDER BY price DESC over a
sales table, moving all six columns.

Plain form: one operator call per task, each task its own allocation, as the
reference runs one launch sequence per batch (operator.hpp:45-47).
Batched form: every task of a kind sits back to back in one arena; one
segmented filter+aggregate launch walks all filter tasks' steps as a device
queue, and one segmented sort + gather orders all ORDER BY tasks; the sort's
digit width and items per thread come from the autotuner, and the whole
pipeline is captured once as a CUDA graph and replayed.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _abi as A
from . import datagen, ops
from .expr import Aggregate, And, Arith, Cast, ColumnRef, Compare, Constant, between

SALES_TYPES = [A.INT64, A.FLOAT32, A.INT32, A.INT32, A.TEXT, A.DATETIME]  # id price qty discount category updated_at
SALES_WIDTHS = [8, 4, 4, 4, 16, 8]
FILTER_COLS = ["price", "qty", "discount", "category"]


def task_rows(ntasks: int, seed: int, lo: int = 1_000, hi: int = 4_000_000) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.exp(rng.uniform(np.log(lo), np.log(hi), ntasks)).astype(np.int64)


def sales_query():
    price, qty, disc, cat = (ColumnRef(0, A.FLOAT32), ColumnRef(1, A.INT32), ColumnRef(2, A.INT32),
                             ColumnRef(3, A.TEXT))
    pred = And(between(disc, Constant(1, A.INT32), Constant(3, A.INT32)), Compare(A.LT, qty, Constant(25, A.INT32)),
               Compare(A.NE, cat, Constant(datagen.EXCLUDED_CATEGORY, A.TEXT)))
    aggs = [Aggregate(A.AGG_SUM, Arith(A.MUL, price, Cast(disc, A.FLOAT32))), Aggregate(A.AGG_COUNT_STAR),
            Aggregate(A.AGG_MIN, price), Aggregate(A.AGG_MAX, price)]
    return pred, aggs


def _device_sales(rows: int, seed: int) -> dict:
    """Sales columns generated on the device (same distributions as datagen.sales_table)."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    cats = torch.from_numpy(datagen.text_slots(datagen.CATEGORIES)).cuda()
    price = (torch.rand(rows, generator=g, device="cuda") * 999.0 + 1.0).clamp_(max=999.9999)
    return {
        "id": torch.arange(rows, dtype=torch.int64, device="cuda"),
        "price": price.to(torch.float32),
        "qty": torch.randint(1, 51, (rows,), generator=g, device="cuda", dtype=torch.int32),
        "discount": torch.randint(0, 11, (rows,), generator=g, device="cuda", dtype=torch.int32),
        "category": cats[torch.randint(0, len(datagen.CATEGORIES), (rows,), generator=g, device="cuda")],
        "updated_at": torch.randint(datagen.DATE_LO, datagen.DATE_HI + 1, (rows,), generator=g, device="cuda",
                                    dtype=torch.int64),
    }


def _host_sales(rows: int, seed: int) -> dict:
    t = datagen.sales_table(rows, seed=seed)
    return {k: torch.from_numpy(np.ascontiguousarray(t[k])).cuda() for k in
            ("id", "price", "qty", "discount", "category", "updated_at")}, t


class TaskSet:
    """The tasks of one run: arenas for the batched form and per-task tables
    for the plain form (copies of the arena slices, each its own allocation)."""

    def __init__(self, rows: np.ndarray, seed: int, on_device: bool = True):
        self.rows = [int(r) for r in rows]
        self.frows = self.rows[0::2]
        self.srows = self.rows[1::2]
        self.foffs = [0] + list(np.cumsum(self.frows).astype(int))
        self.soffs = [0] + list(np.cumsum(self.srows).astype(int))
        self.host = None
        if on_device:
            f = _device_sales(self.foffs[-1], seed)
            s = _device_sales(self.soffs[-1], seed + 1)
        else:
            f, hf = _host_sales(self.foffs[-1], seed)
            s, hs = _host_sales(self.soffs[-1], seed + 1)
            self.host = (hf, hs)
        self.farena = ops.DeviceBatch([ops.DeviceColumn(f[k], t) for k, t in
                                       zip(FILTER_COLS, [A.FLOAT32, A.INT32, A.INT32, A.TEXT])])
        names = ["id", "price", "qty", "discount", "category", "updated_at"]
        self.sarena = ops.DeviceBatch([ops.DeviceColumn(s[k], t) for k, t in zip(names, SALES_TYPES)])
        self.sout = ops.DeviceBatch([ops.DeviceColumn.empty(t, self.soffs[-1], w if t == A.TEXT else None)
                                     for t, w in zip(SALES_TYPES, SALES_WIDTHS)])
        # plain form: each task its own tables
        self.ftasks = [ops.DeviceBatch([ops.DeviceColumn(c.data[a:b].clone(), c.type) for c in self.farena.columns])
                       for a, b in zip(self.foffs[:-1], self.foffs[1:])]
        self.stasks = [ops.DeviceBatch([ops.DeviceColumn(c.data[a:b].clone(), c.type) for c in self.sarena.columns])
                       for a, b in zip(self.soffs[:-1], self.soffs[1:])]
        self.souts = [ops.DeviceBatch([ops.DeviceColumn.empty(t, n, w if t == A.TEXT else None)
                                       for t, w in zip(SALES_TYPES, SALES_WIDTHS)]) for n in self.srows]
        self.algorithmic_bytes = 28.0 * self.foffs[-1] + self.sort_bytes()

    def sort_bytes(self) -> float:
        # f32 key with 8-bit digits: key read + 4 passes x (key + id) in and out + 44-byte rows gathered
        return float(self.soffs[-1]) * (4 + 4 * 16 + 2 * 44)


class PlainRunner:
    """One call per task (per-task workspaces allocated up front)."""

    def __init__(self, ts: TaskSet):
        self.ts = ts
        self.pred, self.aggs = sales_query()
        self.plan = ops.AggPlan([A.FLOAT32, A.INT32, A.INT32, A.TEXT], self.pred, self.aggs)
        self.states = [ops.AggState(self.aggs) for _ in ts.ftasks]
        lib = ops.lib()
        self.fws = [torch.empty(lib.yq_filter_aggregate_workspace_size(b.rows, len(self.aggs)), dtype=torch.uint8,
                                device="cuda") for b in ts.ftasks]
        self.sws = [torch.empty(max(256, ops.order_by_segments_workspace_bytes(b.columns[1], [0, b.rows])),
                                dtype=torch.uint8, device="cuda") for b in ts.stasks]
        self.soffs = [(C.c_uint32 * 2)(0, b.rows) for b in ts.stasks]

    def run(self):
        for b, st, ws in zip(self.ts.ftasks, self.states, self.fws):
            ops.lib().yq_agg_state_init(st.buf.data_ptr(), st._specs, len(self.aggs),
                                        torch.cuda.current_stream().cuda_stream)
            self.plan.run(b, st, workspace=ws)
        for b, o, ws, offs in zip(self.ts.stasks, self.ts.souts, self.sws, self.soffs):
            ops.order_by_segments(b, 1, True, offs, o, workspace=ws)

    def results(self):
        return [st.read() for st in self.states]


class BatchedPipeline:
    """Two segmented launches sequences (filter+aggregate, ORDER BY) over the
    arenas, autotuned and captured once as a CUDA graph."""

    def __init__(self, ts: TaskSet, graph: bool = True):
        self.ts = ts
        self.pred, self.aggs = sales_query()
        self.plan = ops.AggPlan([A.FLOAT32, A.INT32, A.INT32, A.TEXT], self.pred, self.aggs)
        self.states = ops.AggStates(self.aggs, len(ts.frows))
        lib = ops.lib()
        self.fws = torch.empty(lib.yq_filter_aggregate_segments_workspace_size(ts.foffs[-1], len(ts.frows)),
                               dtype=torch.uint8, device="cuda")
        self.foffs = (C.c_uint32 * len(ts.foffs))(*ts.foffs)
        self.soffs = (C.c_uint32 * len(ts.soffs))(*ts.soffs)
        self.sws = torch.empty(max(256, ops.order_by_segments_workspace_bytes(ts.sarena.columns[1], ts.soffs)),
                               dtype=torch.uint8, device="cuda")
        tuned = ops.sort_autotune(ts.sarena.columns[1], ts.soffs, descending=True)
        self.tuned = (tuned.digit_bits, tuned.items_per_thread, tuned.block_threads)
        # digit width / items from the autotuner's cache, no host read-back: capturable
        self.cfg = ops.sort_config(digit_bits=0, keep_trivial=True)
        self.graph = None
        if graph:
            self._eager()  # warm-up outside the capture (attributes, occupancy queries)
            torch.cuda.synchronize()
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                self._eager()
            torch.cuda.current_stream().wait_stream(s)
            torch.cuda.synchronize()
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph):
                self._eager()
            torch.cuda.synchronize()

    def _eager(self):
        s = torch.cuda.current_stream().cuda_stream
        ops.lib().yq_agg_states_init(self.states.buf.data_ptr(), self.states.count, self.states._specs,
                                     len(self.aggs), s)
        self.plan.run_segments(self.ts.farena, self.foffs, self.states, workspace=self.fws)
        ops.order_by_segments(self.ts.sarena, 1, True, self.soffs, self.ts.sout, config=self.cfg, workspace=self.sws)

    def run(self):
        if self.graph is not None:
            self.graph.replay()
        else:
            self._eager()

    def error_word(self) -> int:
        return int(self.sws[:4].view(torch.int32)[0].item())

    def results(self):
        return self.states.read()
