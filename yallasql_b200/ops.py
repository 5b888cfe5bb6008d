"""Python entry points over the C ABI, on torch CUDA tensors.

PyTorch supplies device memory and streams only; every operator runs in
libyq_ops.so. There is no CPU fallback: without the library (or a GPU) these
functions raise.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from . import _abi as A
from .expr import Aggregate, ConstPool, Expr, compile_expr, Compiled

TORCH_DTYPE = {A.INT32: torch.int32, A.FLOAT32: torch.float32, A.INT64: torch.int64, A.DATETIME: torch.int64,
               A.FLOAT64: torch.float64, A.BOOL: torch.uint8, A.TEXT: torch.uint8}


def lib():
    return A.load()


def _stream(stream=None) -> int:
    """Raw cudaStream_t of a torch stream, a raw handle, or the current stream."""
    if isinstance(stream, int):
        return stream
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


@dataclass
class DeviceColumn:
    """One column of a batch in HBM: values plus an optional null-byte array
    (the reference's Batch::columnData[i] + NullBitSet, include/batch.hpp:21-60)."""
    data: torch.Tensor
    type: int
    nulls: torch.Tensor | None = None

    @property
    def width(self) -> int:
        if self.type == A.TEXT:
            return int(self.data.shape[1])
        return self.data.element_size()

    @property
    def rows(self) -> int:
        return int(self.data.shape[0])

    def c(self) -> A.Column:
        return A.Column(self.data.data_ptr(), self.nulls.data_ptr() if self.nulls is not None else None,
                        self.type, self.width)

    @staticmethod
    def empty(type_: int, rows: int, width: int | None = None, nulls: bool = False, device="cuda"):
        if type_ == A.TEXT:
            data = torch.empty((rows, width), dtype=torch.uint8, device=device)
        else:
            data = torch.empty(rows, dtype=TORCH_DTYPE[type_], device=device)
        n = torch.empty(rows, dtype=torch.uint8, device=device) if nulls else None
        return DeviceColumn(data, type_, n)

    def slice(self, start: int, stop: int) -> "DeviceColumn":
        return DeviceColumn(self.data[start:stop], self.type, None if self.nulls is None else self.nulls[start:stop])


@dataclass
class DeviceBatch:
    columns: list

    @property
    def rows(self) -> int:
        return self.columns[0].rows if self.columns else 0

    def c(self):
        arr = (A.Column * max(1, len(self.columns)))(*[c.c() for c in self.columns])
        b = A.Batch(arr, len(self.columns), self.rows)
        return b, arr

    def slice(self, start: int, stop: int) -> "DeviceBatch":
        return DeviceBatch([c.slice(start, stop) for c in self.columns])


def _check(st: int, where: str):
    A.check(st, where)


# ----------------------------------------------------------- aggregates
class AggState:
    """Device accumulator for a list of aggregates (AggregateExpression's
    accumlator/counter, include/engine/operators/expressions/aggregate.hpp:20-40)."""

    def __init__(self, aggs: list[Aggregate], stream=None):
        self.aggs = aggs
        self.buf = torch.empty(max(256, lib().yq_agg_state_bytes(len(aggs))), dtype=torch.uint8, device="cuda")
        self._specs = _agg_specs_stub(aggs)
        self.reset(stream)

    def reset(self, stream=None):
        """Back to the aggregates' identities, so the state serves another query."""
        _check(lib().yq_agg_state_init(self.buf.data_ptr(), self._specs, len(self.aggs), _stream(stream)),
               "yq_agg_state_init")

    def read(self, stream=None) -> list:
        out = (A.AggResult * max(1, len(self.aggs)))()
        _check(lib().yq_agg_state_read(self.buf.data_ptr(), self._specs, len(self.aggs), out, _stream(stream)),
               "yq_agg_state_read")
        vals = []
        for a, r in zip(self.aggs, out):
            if r.is_null:
                vals.append(None)
            elif a.kind in (A.AGG_COUNT, A.AGG_COUNT_STAR):
                vals.append(int(r.i))
            elif a.kind == A.AGG_AVG or a.input_type in (A.FLOAT32, A.FLOAT64):
                vals.append(float(r.f))
            else:
                vals.append(int(r.i))
        return vals


def _agg_specs_stub(aggs):
    arr = (A.AggSpec * max(1, len(aggs)))()
    for i, a in enumerate(aggs):
        arr[i].kind = a.kind
        arr[i].input_type = a.input_type
    return arr


class AggPlan:
    """Compiled predicate + aggregate inputs, reusable across batches."""

    def __init__(self, col_types: list[int], predicate: Expr | None, aggs: list[Aggregate]):
        self.pool = ConstPool()
        self.pred = Compiled(compile_expr(predicate, self.pool, col_types) if predicate is not None else [])
        self.inputs = [Compiled(compile_expr(a.arg, self.pool, col_types) if a.arg is not None else [])
                       for a in aggs]
        self.aggs = aggs
        self.specs = (A.AggSpec * max(1, len(aggs)))()
        for i, (a, p) in enumerate(zip(aggs, self.inputs)):
            self.specs[i].kind = a.kind
            self.specs[i].input_type = a.input_type
            self.specs[i].input = p.prog
        self.consts, self._keep = self.pool.to_c()

    def run(self, batch: DeviceBatch, state: AggState, stream=None, workspace: torch.Tensor | None = None):
        b, keep = batch.c()
        ws = workspace.data_ptr() if workspace is not None else None
        wsb = workspace.numel() if workspace is not None else 0
        _check(lib().yq_filter_aggregate(C.byref(b), C.byref(self.pred.prog), C.byref(self.consts), self.specs,
                                         len(self.aggs), state.buf.data_ptr(), ws, wsb, _stream(stream)),
               "yq_filter_aggregate")


    def run_segments(self, batch: DeviceBatch, seg_offsets, states: "AggStates", stream=None,
                     workspace: torch.Tensor | None = None):
        """One launch for many tasks: task g = rows [seg_offsets[g], seg_offsets[g+1])."""
        b, keep = batch.c()
        offs = seg_offsets if isinstance(seg_offsets, C.Array) else (C.c_uint32 * len(seg_offsets))(*seg_offsets)
        ws = workspace.data_ptr() if workspace is not None else None
        wsb = workspace.numel() if workspace is not None else 0
        _check(lib().yq_filter_aggregate_segments(C.byref(b), offs, len(offs) - 1, C.byref(self.pred.prog),
                                                  C.byref(self.consts), self.specs, len(self.aggs),
                                                  states.buf.data_ptr(), ws, wsb, _stream(stream)),
               "yq_filter_aggregate_segments")


    def run_ranges(self, batch: DeviceBatch, begin: list, end: list, states: "AggStates", stream=None,
                   workspace: torch.Tensor | None = None):
        """One launch for tasks given as row ranges [begin[g], end[g]) of the batch."""
        b, keep = batch.c()
        n = len(begin)
        cb, ce = (C.c_uint32 * n)(*begin), (C.c_uint32 * n)(*end)
        ws = workspace.data_ptr() if workspace is not None else None
        wsb = workspace.numel() if workspace is not None else 0
        _check(lib().yq_filter_aggregate_ranges(C.byref(b), cb, ce, n, C.byref(self.pred.prog), C.byref(self.consts),
                                                self.specs, len(self.aggs), states.buf.data_ptr(), ws, wsb,
                                                _stream(stream)), "yq_filter_aggregate_ranges")


class AggStates:
    """`count` aggregate states back to back (one per task of a batched call)."""

    def __init__(self, aggs: list[Aggregate], count: int, stream=None):
        self.aggs, self.count = aggs, count
        self.step = int(lib().yq_agg_state_bytes(len(aggs)))
        self.buf = torch.empty(max(1, count) * self.step, dtype=torch.uint8, device="cuda")
        self._specs = _agg_specs_stub(aggs)
        self.reset(stream)

    def reset(self, stream=None, count: int | None = None):
        """The first `count` states (all by default) back to the identities."""
        k = self.count if count is None else count
        if k < 0 or k > self.count:
            raise ValueError("count beyond the states allocated")
        _check(lib().yq_agg_states_init(self.buf.data_ptr(), k, self._specs, len(self.aggs),
                                        _stream(stream)), "yq_agg_states_init")

    def read(self, stream=None, count: int | None = None) -> list:
        """Results of the first `count` states (all by default)."""
        k = self.count if count is None else count
        n = len(self.aggs)
        out = (A.AggResult * max(1, k * n))()
        _check(lib().yq_agg_states_read(self.buf.data_ptr(), k, self._specs, n, out, _stream(stream)),
               "yq_agg_states_read")
        res = []
        for g in range(k):
            vals = []
            for i, a in enumerate(self.aggs):
                r = out[g * n + i]
                if r.is_null:
                    vals.append(None)
                elif a.kind in (A.AGG_COUNT, A.AGG_COUNT_STAR):
                    vals.append(int(r.i))
                elif a.kind == A.AGG_AVG or a.input_type in (A.FLOAT32, A.FLOAT64):
                    vals.append(float(r.f))
                else:
                    vals.append(int(r.i))
            res.append(vals)
        return res


def filter_aggregate(batch: DeviceBatch, predicate: Expr | None, aggs: list[Aggregate], stream=None) -> list:
    plan = AggPlan([c.type for c in batch.columns], predicate, aggs)
    st = AggState(aggs, stream)
    plan.run(batch, st, stream)
    return st.read(stream)


# ----------------------------------------------------------- projection
class ProjectPlan:
    """Compiled WHERE + SELECT list (FilterOperator + ProjectionOperator)."""

    def __init__(self, col_types: list[int], col_widths: list[int], predicate: Expr | None, select: list):
        self.pool = ConstPool()
        self.pred = Compiled(compile_expr(predicate, self.pool, col_types) if predicate is not None else [])
        self.select = select
        self.progs = []
        self.proj = (A.Projection * max(1, len(select)))()
        self.out_types, self.out_widths = [], []
        for i, s in enumerate(select):
            if isinstance(s, int):
                self.proj[i].column = s
                self.proj[i].out_type = col_types[s]
                self.out_types.append(col_types[s])
                self.out_widths.append(col_widths[s])
                self.progs.append(None)
            else:
                p = Compiled(compile_expr(s, self.pool, col_types))
                self.progs.append(p)
                self.proj[i].column = -1
                self.proj[i].out_type = s.type
                self.proj[i].program = p.prog
                self.out_types.append(s.type)
                self.out_widths.append({A.INT32: 4, A.FLOAT32: 4, A.INT64: 8, A.DATETIME: 8, A.FLOAT64: 8,
                                        A.BOOL: 1}[s.type])
        self.consts, self._keep = self.pool.to_c()

    def run(self, batch: DeviceBatch, capacity: int | None = None, with_nulls: bool = True, stream=None):
        cap = batch.rows if capacity is None else capacity
        outs = [DeviceColumn.empty(t, max(cap, 1), w if t == A.TEXT else None, nulls=with_nulls)
                for t, w in zip(self.out_types, self.out_widths)]
        oc = (A.Column * max(1, len(outs)))(*[o.c() for o in outs])
        b, keep = batch.c()
        cnt = C.c_uint32(0)
        st = lib().yq_filter_project(C.byref(b), C.byref(self.pred.prog), C.byref(self.consts), self.proj,
                                     len(self.select), oc, cap, None, C.byref(cnt), None, 0, _stream(stream))
        _check(st, "yq_filter_project")
        n = cnt.value
        return DeviceBatch([o.slice(0, n) for o in outs])


def filter_project(batch: DeviceBatch, predicate: Expr | None, select: list, stream=None) -> DeviceBatch:
    plan = ProjectPlan([c.type for c in batch.columns], [c.width for c in batch.columns], predicate, select)
    return plan.run(batch, stream=stream)


# ----------------------------------------------------------------- sort
def sort_config(digit_bits=0, keep_trivial=False, items_per_thread=0, block_threads=0):
    c = A.SortConfig()
    c.digit_bits = digit_bits
    c.items_per_thread = items_per_thread
    c.block_threads = block_threads
    c.keep_trivial = 1 if keep_trivial else 0
    return c


def sort_indices(col: DeviceColumn, descending=False, nulls_first=False, config=None, stream=None,
                 out: torch.Tensor | None = None, workspace: torch.Tensor | None = None) -> torch.Tensor:
    perm = out if out is not None else torch.empty(col.rows, dtype=torch.int32, device="cuda")
    cc = col.c()
    ws = workspace.data_ptr() if workspace is not None else None
    wsb = workspace.numel() if workspace is not None else 0
    _check(lib().yq_sort_indices(C.byref(cc), col.rows, int(descending), int(nulls_first), perm.data_ptr(),
                                 C.byref(config) if config is not None else None, ws, wsb, _stream(stream)),
           "yq_sort_indices")
    return perm


def sort_indices_multi(cols: list, descending: list, nulls_first: list | None = None, config=None, stream=None):
    n = cols[0].rows
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    arr = (A.Column * len(cols))(*[c.c() for c in cols])
    d = (C.c_int32 * len(cols))(*[int(x) for x in descending])
    nf = (C.c_int32 * len(cols))(*[int(x) for x in (nulls_first or [0] * len(cols))])
    _check(lib().yq_sort_indices_multi(arr, d, nf, len(cols), n, perm.data_ptr(),
                                       C.byref(config) if config is not None else None, None, 0, _stream(stream)),
           "yq_sort_indices_multi")
    return perm


def sort_segments(col: DeviceColumn, seg_offsets: list[int], descending=False, nulls_first=False, config=None,
                  stream=None, out: torch.Tensor | None = None, workspace: torch.Tensor | None = None):
    perm = out if out is not None else torch.empty(col.rows, dtype=torch.int32, device="cuda")
    offs = (C.c_uint32 * len(seg_offsets))(*seg_offsets)
    cc = col.c()
    ws = workspace.data_ptr() if workspace is not None else None
    wsb = workspace.numel() if workspace is not None else 0
    _check(lib().yq_sort_segments(C.byref(cc), col.rows, offs, len(seg_offsets) - 1, int(descending),
                                  int(nulls_first), perm.data_ptr(),
                                  C.byref(config) if config is not None else None, ws, wsb, _stream(stream)),
           "yq_sort_segments")
    return perm


def sort_workspace_bytes(col: DeviceColumn, seg_offsets: list[int] | None = None) -> int:
    cc = col.c()
    if seg_offsets is None:
        return int(lib().yq_sort_workspace_size(C.byref(cc), col.rows))
    offs = (C.c_uint32 * len(seg_offsets))(*seg_offsets)
    return int(lib().yq_sort_segments_workspace_size(C.byref(cc), col.rows, offs, len(seg_offsets) - 1))


def gather(batch: DeviceBatch, perm: torch.Tensor, stream=None, out: DeviceBatch | None = None) -> DeviceBatch:
    n = int(perm.numel())
    if out is None:
        out = DeviceBatch([DeviceColumn.empty(c.type, n, c.width if c.type == A.TEXT else None,
                                              nulls=c.nulls is not None) for c in batch.columns])
    src = (A.Column * len(batch.columns))(*[c.c() for c in batch.columns])
    dst = (A.Column * len(out.columns))(*[c.c() for c in out.columns])
    _check(lib().yq_gather(src, len(batch.columns), perm.data_ptr(), n, dst, _stream(stream)), "yq_gather")
    return out


def sort_batch(batch: DeviceBatch, key: int, descending=False, nulls_first=False, config=None, stream=None):
    """ORDER BY one key: argsort + gather every column (OrderOperator for one run)."""
    perm = sort_indices(batch.columns[key], descending, nulls_first, config, stream)
    return gather(batch, perm, stream)


# ---------------------------------------------------------------- merge
def merge_pass(src: DeviceBatch, key: int, descending: bool, offsets: list[int], dst: DeviceBatch,
               nulls_first=False, stream=None) -> list[int]:
    """Merge runs (0,1), (2,3), ... of `src` into `dst`; returns the new run offsets."""
    offs = (C.c_uint32 * len(offsets))(*offsets)
    sc = (A.Column * len(src.columns))(*[c.c() for c in src.columns])
    dc = (A.Column * len(dst.columns))(*[c.c() for c in dst.columns])
    _check(lib().yq_merge_pass(sc, len(src.columns), key, int(descending), int(nulls_first), offs,
                               len(offsets) - 1, dc, None, 0, _stream(stream)), "yq_merge_pass")
    return [offsets[i] for i in range(0, len(offsets) - 1, 2)] + [offsets[-1]]


def merge_runs(runs: DeviceBatch, key: int, descending: bool, offsets: list[int], out: DeviceBatch,
               scratch: DeviceBatch | None = None, nulls_first=False, stream=None) -> DeviceBatch:
    """Merge sorted runs pairwise, level by level, until one run remains
    (OrderOperator::merge_all_sorted, include/engine/operators/order_operator.hpp:160-193).
    The final level writes into `out`; `runs` and `scratch` are clobbered."""
    nruns = len(offsets) - 1
    levels = 0
    while (nruns + (1 << levels) - 1) >> levels > 1:
        levels += 1
    if levels == 0:
        if runs is not out:
            for a, b in zip(runs.columns, out.columns):
                b.data.copy_(a.data)
                if b.nulls is not None and a.nulls is not None:
                    b.nulls.copy_(a.nulls)
        return out
    if scratch is None:
        scratch = DeviceBatch([DeviceColumn.empty(c.type, c.rows, c.width if c.type == A.TEXT else None,
                                                  nulls=c.nulls is not None) for c in runs.columns])
    # alternate so that the last level lands in `out`
    bufs = [out, scratch] if levels % 2 == 1 else [scratch, out]
    src = runs
    for lvl in range(levels):
        dst = bufs[lvl % 2]
        offsets = merge_pass(src, key, descending, offsets, dst, nulls_first, stream)
        src = dst
    return out


# ----------------------------------------------------------------- joins
def _conds(conds):
    arr = (A.JoinCond * max(1, len(conds)))(*[A.JoinCond(l, r, c) for l, r, c in conds])
    return arr


def _disjunct(disjunct, conds):
    if len(disjunct) != len(conds):
        raise ValueError("one disjunct group per condition")
    return (C.c_int32 * len(conds))(*disjunct)


def join_pairs(left: DeviceBatch, right: DeviceBatch, conds: list, capacity: int | None = None, stream=None,
               disjunct: list | None = None):
    """Inner join pairs (left row, right row) in (left, right) order; conds =
    [(left_col, right_col, yq_cmp)], all ANDed (JoinOperator + ComparisonJoinExpression);
    with `disjunct` (a group per condition) an OR of the groups' ANDs."""
    lb, lk = left.c()
    rb, rk = right.c()
    cap = capacity if capacity is not None else max(1, left.rows * right.rows if len(conds) == 0 else left.rows * 4)
    dj = None if disjunct is None else _disjunct(disjunct, conds)
    while True:
        ol = torch.empty(max(1, cap), dtype=torch.int32, device="cuda")
        orr = torch.empty(max(1, cap), dtype=torch.int32, device="cuda")
        cnt = C.c_uint64(0)
        if dj is None:
            st = lib().yq_join_pairs(C.byref(lb), C.byref(rb), _conds(conds), len(conds), ol.data_ptr(),
                                     orr.data_ptr(), cap, C.byref(cnt), None, 0, _stream(stream))
        else:
            st = lib().yq_join_pairs_or(C.byref(lb), C.byref(rb), _conds(conds), C.cast(dj, C.c_void_p), len(conds),
                                        ol.data_ptr(), orr.data_ptr(), cap, C.byref(cnt), None, 0, _stream(stream))
        if st == A.ERR_CAPACITY and capacity is None:
            cap = int(cnt.value)  # count-then-retry with the exact size
            continue
        _check(st, "yq_join_pairs")
        n = int(cnt.value)
        return ol[:n], orr[:n]


def join_project(left: DeviceBatch, right: DeviceBatch, conds: list, outputs: list, capacity: int | None = None,
                 stream=None, disjunct: list | None = None) -> DeviceBatch:
    """Join and write the chosen columns [(side, column)] of every matching
    pair; `disjunct` as in join_pairs."""
    lb, lk = left.c()
    rb, rk = right.c()
    srcs = [(right if s else left).columns[c] for s, c in outputs]
    cap = capacity if capacity is not None else (left.rows * right.rows if not conds else max(1, left.rows * 4))
    outs_c = (A.JoinOutput * len(outputs))(*[A.JoinOutput(s, c) for s, c in outputs])
    dj = None if disjunct is None else _disjunct(disjunct, conds)
    while True:
        outs = [DeviceColumn.empty(c.type, max(1, cap), c.width if c.type == A.TEXT else None,
                                   nulls=c.nulls is not None) for c in srcs]
        oc = (A.Column * len(outs))(*[o.c() for o in outs])
        cnt = C.c_uint64(0)
        if dj is None:
            st = lib().yq_join_project(C.byref(lb), C.byref(rb), _conds(conds), len(conds), outs_c, len(outputs),
                                       oc, cap, C.byref(cnt), None, 0, _stream(stream))
        else:
            st = lib().yq_join_project_or(C.byref(lb), C.byref(rb), _conds(conds), C.cast(dj, C.c_void_p),
                                          len(conds), outs_c, len(outputs), oc, cap, C.byref(cnt), None, 0,
                                          _stream(stream))
        if st == A.ERR_CAPACITY and capacity is None:
            cap = int(cnt.value)
            continue
        _check(st, "yq_join_project")
        n = int(cnt.value)
        return DeviceBatch([o.slice(0, n) for o in outs])


def cross_product(left: DeviceBatch, right: DeviceBatch, stream=None) -> DeviceBatch:
    """Every (l, r) pair, left-major, all columns of both sides (CrossProductOperator)."""
    outputs = [(0, i) for i in range(len(left.columns))] + [(1, i) for i in range(len(right.columns))]
    return join_project(left, right, [], outputs, stream=stream)


class JoinAggPlan:
    """Fused star join + aggregate: fact rows passing `fact_pred` that find their
    key among the dimension rows passing `dim_pred` feed the aggregates."""

    def __init__(self, fact_types, dim_types, fact_pred, fact_key, dim_pred, dim_key, aggs):
        self.pool = ConstPool()
        self.fpred = Compiled(compile_expr(fact_pred, self.pool, fact_types) if fact_pred is not None else [])
        self.dpred = Compiled(compile_expr(dim_pred, self.pool, dim_types) if dim_pred is not None else [])
        self.inputs = [Compiled(compile_expr(a.arg, self.pool, fact_types) if a.arg is not None else []) for a in aggs]
        self.aggs = aggs
        self.fact_key, self.dim_key = fact_key, dim_key
        self.specs = (A.AggSpec * max(1, len(aggs)))()
        for i, (a, p) in enumerate(zip(aggs, self.inputs)):
            self.specs[i].kind = a.kind
            self.specs[i].input_type = a.input_type
            self.specs[i].input = p.prog
        self.consts, self._keep = self.pool.to_c()

    def run(self, fact: DeviceBatch, dim: DeviceBatch, state: AggState, stream=None):
        fb, fk = fact.c()
        db, dk = dim.c()
        _check(lib().yq_join_aggregate(C.byref(fb), C.byref(self.fpred.prog), self.fact_key, C.byref(db),
                                       C.byref(self.dpred.prog), self.dim_key, C.byref(self.consts), self.specs,
                                       len(self.aggs), state.buf.data_ptr(), None, 0, _stream(stream)),
               "yq_join_aggregate")

    def prepare(self, dim: DeviceBatch, stream=None) -> "PreparedDim":
        """Build the dimension side once (filtered, hashed, kept resident)."""
        return PreparedDim(self, dim, stream)

    def run_prepared(self, fact: DeviceBatch, prepared: "PreparedDim", state: AggState, stream=None,
                     workspace: torch.Tensor | None = None):
        """Probe a prepared dimension table: no host synchronisation."""
        fb, fk = fact.c()
        ws = workspace.data_ptr() if workspace is not None else None
        wsb = workspace.numel() if workspace is not None else 0
        _check(lib().yq_join_aggregate_prepared(C.byref(fb), C.byref(self.fpred.prog), self.fact_key,
                                                prepared.table.data_ptr(), prepared.dim_rows, prepared.kept,
                                                prepared.key_type, C.byref(self.consts), self.specs, len(self.aggs),
                                                state.buf.data_ptr(), ws, wsb, _stream(stream)),
               "yq_join_aggregate_prepared")


class PreparedDim:
    """A star join's dimension side built once and kept in device memory."""

    def __init__(self, plan: JoinAggPlan, dim: DeviceBatch, stream=None):
        self.dim_rows = dim.rows
        self.key_type = dim.columns[plan.dim_key].type
        self.table = torch.empty(int(lib().yq_join_dim_table_size(dim.rows)), dtype=torch.uint8, device="cuda")
        db, dk = dim.c()
        kept = C.c_uint32(0)
        _check(lib().yq_join_dim_table_build(C.byref(db), C.byref(plan.dpred.prog), plan.dim_key,
                                             C.byref(plan.consts), self.table.data_ptr(), self.table.numel(),
                                             C.byref(kept), _stream(stream)), "yq_join_dim_table_build")
        self.kept = int(kept.value)


def order_by_workspace_bytes(col: DeviceColumn, offsets: list[int]) -> int:
    """Least workspace of yq_order_by (one-level gather)."""
    offs = (C.c_uint32 * len(offsets))(*offsets)
    cc = col.c()
    return int(lib().yq_order_by_workspace_size(C.byref(cc), col.rows, offs, len(offsets) - 1))


def order_by_batch_workspace_bytes(batch: DeviceBatch, key: int, offsets: list[int]) -> int:
    """Workspace of yq_order_by including the sorted-run copy of the columns."""
    offs = (C.c_uint32 * len(offsets))(*offsets)
    b, _keep = batch.c()
    return int(lib().yq_order_by_batch_workspace_size(C.byref(b), key, offs, len(offsets) - 1))


class OrderByRuns:
    """Out-of-core ORDER BY of one key over a batch made of runs (4 MB
    batches), through yq_order_by: the runs are sorted by the segmented radix
    sort, merged level by level as (key words, row id) pairs, and every column
    is gathered once by the merged row ids (OrderOperator::firstPass +
    merge_all_sorted, order_operator.hpp:89-193 / order_operator.cpp:14-220).
    The workspace is allocated once and reused across calls; `two_level`
    sizes it for the sorted-run copy that the two-level gather uses on large
    tables."""

    def __init__(self, batch: DeviceBatch, key: int, offsets: list[int], two_level: bool = True):
        self.key, self.offsets, self.n = key, list(offsets), batch.rows
        self._offs = (C.c_uint32 * len(self.offsets))(*self.offsets)
        need = (order_by_batch_workspace_bytes(batch, key, self.offsets) if two_level
                else order_by_workspace_bytes(batch.columns[key], self.offsets))
        self.ws = torch.empty(max(need, 256), dtype=torch.uint8, device="cuda")

    def run(self, batch: DeviceBatch, descending: bool, out: DeviceBatch, nulls_first=False, stream=None):
        ib, _ia = batch.c()
        ob, _oa = out.c()
        _check(lib().yq_order_by(C.byref(ib), self.key, int(descending), int(nulls_first), self._offs,
                                 len(self.offsets) - 1, C.byref(ob), self.ws.data_ptr(), self.ws.numel(),
                                 _stream(stream)), "yq_order_by")
        return out


def order_by(batch: DeviceBatch, key: int, descending: bool, offsets: list[int], nulls_first=False,
             stream=None, merge_items: int | None = None) -> DeviceBatch:
    """One-shot yq_order_by into a new batch (workspace from the library);
    `merge_items` picks the merge tile (yq_order_by_tiled)."""
    out = DeviceBatch([DeviceColumn.empty(c.type, c.rows, c.width if c.type == A.TEXT else None,
                                          nulls=c.nulls is not None) for c in batch.columns])
    offs = (C.c_uint32 * len(offsets))(*offsets)
    ib, _ia = batch.c()
    ob, _oa = out.c()
    if merge_items is None:
        _check(lib().yq_order_by(C.byref(ib), key, int(descending), int(nulls_first), offs, len(offsets) - 1,
                                 C.byref(ob), None, 0, _stream(stream)), "yq_order_by")
    else:
        _check(lib().yq_order_by_tiled(C.byref(ib), key, int(descending), int(nulls_first), offs, len(offsets) - 1,
                                       C.byref(ob), merge_items, None, 0, _stream(stream)), "yq_order_by_tiled")
    return out


def order_by_segments_workspace_bytes(col: DeviceColumn, offsets) -> int:
    offs = (C.c_uint32 * len(offsets))(*offsets)
    cc = col.c()
    return int(lib().yq_order_by_segments_workspace_size(C.byref(cc), col.rows, offs, len(offsets) - 1))


def order_by_segments(batch: DeviceBatch, key: int, descending: bool, offsets, out: DeviceBatch, config=None,
                      workspace: torch.Tensor | None = None, nulls_first=False, stream=None,
                      perm_out: torch.Tensor | None = None) -> DeviceBatch:
    """ORDER BY per task: task g = rows [offsets[g], offsets[g+1]) (yq_order_by_segments);
    with `perm_out` the permutation is kept there (yq_order_by_segments_perm)."""
    offs = offsets if isinstance(offsets, C.Array) else (C.c_uint32 * len(offsets))(*offsets)
    ib, _ia = batch.c()
    ob, _oa = out.c()
    ws = workspace.data_ptr() if workspace is not None else None
    wsb = workspace.numel() if workspace is not None else 0
    cfg = C.byref(config) if config is not None else None
    if perm_out is not None:
        _check(lib().yq_order_by_segments_perm(C.byref(ib), key, int(descending), int(nulls_first), offs,
                                               len(offs) - 1, C.byref(ob), perm_out.data_ptr(), cfg, ws, wsb,
                                               _stream(stream)), "yq_order_by_segments_perm")
    else:
        _check(lib().yq_order_by_segments(C.byref(ib), key, int(descending), int(nulls_first), offs, len(offs) - 1,
                                          C.byref(ob), cfg, ws, wsb, _stream(stream)), "yq_order_by_segments")
    return out


def sort_autotune(col: DeviceColumn, offsets, descending=False, stream=None) -> "A.SortConfig":
    """Time every sort variant on this key and segments; the winner is remembered
    for this key width and segment size and returned."""
    offs = (C.c_uint32 * len(offsets))(*offsets)
    cc = col.c()
    best = A.SortConfig()
    _check(lib().yq_sort_autotune(C.byref(cc), col.rows, offs, len(offsets) - 1, int(descending), C.byref(best),
                                  _stream(stream)), "yq_sort_autotune")
    return best


def order_by_autotune(batch: DeviceBatch, key: int, descending: bool, offsets, nulls_first=False,
                      stream=None) -> tuple["A.SortConfig", int]:
    """Tune yq_order_by for this input (yq_order_by_autotune): the run sort's
    (digit bits, items per thread, block threads) and the merge tile's outputs
    per thread, remembered for later calls on inputs of this shape."""
    offs = offsets if isinstance(offsets, C.Array) else (C.c_uint32 * len(offsets))(*offsets)
    ib, _ia = batch.c()
    best = A.SortConfig()
    items = C.c_int32(0)
    _check(lib().yq_order_by_autotune(C.byref(ib), key, int(descending), int(nulls_first), offs, len(offs) - 1,
                                      C.byref(best), C.byref(items), _stream(stream)), "yq_order_by_autotune")
    return best, int(items.value)


# ------------------------------------------------------------------ CSV scan
@dataclass
class CsvColumn:
    """One column of a CSV table: name without its tags, type, primary-key tag."""
    name: str
    type: int
    pk: bool = False


def csv_schema(header: str, first_line: str = "") -> list[CsvColumn]:
    """Column names and types from a header line in the reference's tag
    convention (Table::inferDBSchema, src/db/table.cpp:43-150): the header and
    the first data line are split at every ',' (pairwise, stopping at the
    shorter), quotes/CR/LF removed; "(P)" marks a primary key; "(N)" is FLOAT
    when the first data line's value contains '.', else INT; "(D)" DATETIME;
    "(T)" or no tag STRING."""
    names = header.split(",")
    values = first_line.split(",")
    out = []
    for name, value in zip(names, values):
        for ch in '"\r\n':
            name = name.replace(ch, "")
            value = value.replace(ch, "")
        base = name.strip(" \t")
        pk = base.endswith("(P)")
        if pk:
            base = base[:-3].rstrip(" \t")
        if base.endswith("(N)"):
            type_ = A.FLOAT32 if "." in value.strip(" \t") else A.INT32
            base = base[:-3]
        elif base.endswith("(D)"):
            type_, base = A.DATETIME, base[:-3]
        elif base.endswith("(T)"):
            type_, base = A.TEXT, base[:-3]
        else:
            type_ = A.TEXT
        base = base.rstrip(" \t")
        if not base:
            raise ValueError(f"invalid column name in CSV header: {name!r}")
        out.append(CsvColumn(base, type_, pk))
    return out


class CsvScanError(ValueError):
    """A cell that std::stoi / std::stof would reject (the reference exits there)."""

    def __init__(self, err: "A.CsvError", batch: "DeviceBatch"):
        kind = {1: "no conversion (invalid_argument)", 2: "out of range"}.get(err.kind, str(err.kind))
        super().__init__(f"{err.bad_cells} bad cell(s); first at row {err.first_row}, field {err.first_field}: {kind}")
        self.error = err
        self.batch = batch


def csv_scan(text: torch.Tensor, types: list[int], project: list[int] | None = None, text_width: int = 256,
             stream=None) -> DeviceBatch:
    """Parse CSV text resident on the device (uint8 tensor, the header line
    removed) into a DeviceBatch: the device-side GetOperator::next
    (src/engine/operators/get_operator.cpp:56-109). `types[f]` is the type of
    CSV field f (from csv_schema); `project` lists the fields to keep, in output
    order (default: all). Text columns get slots of `text_width` bytes (the
    reference's slot is 256). Raises CsvScanError (batch attached) when a cell
    fails to convert."""
    L = lib()
    s = _stream(stream)
    nbytes = int(text.numel())
    project = list(range(len(types))) if project is None else list(project)
    if text.dtype != torch.uint8 or not text.is_cuda or not text.is_contiguous():
        raise ValueError("text must be a contiguous uint8 CUDA tensor")
    records = C.c_uint64(0)
    ptr = text.data_ptr() if nbytes else None
    # one index call with room for records of 16 bytes on average; a second
    # one, with the exact count, only for text of shorter records
    cap = nbytes // 16 + 1024
    starts = torch.empty(cap, dtype=torch.int32, device=text.device)
    st = L.yq_csv_index(ptr, nbytes, starts.data_ptr(), cap, C.byref(records), None, 0, s)
    if st == A.ERR_CAPACITY:
        starts = torch.empty(int(records.value), dtype=torch.int32, device=text.device)
        st = L.yq_csv_index(ptr, nbytes, starts.data_ptr(), int(records.value), C.byref(records), None, 0, s)
    _check(st, "yq_csv_index")
    n = int(records.value)
    cols = []
    field_col = [-1] * len(types)
    for i, f in enumerate(project):
        field_col[f] = i
        cols.append(DeviceColumn.empty(types[f], n, text_width if types[f] == A.TEXT else None, nulls=True,
                                       device=text.device))
    ccols = (A.Column * max(1, len(cols)))(*[c.c() for c in cols])
    fc = (C.c_int32 * len(types))(*field_col)
    rows = C.c_uint32(0)
    err = A.CsvError()
    st = L.yq_csv_parse(ptr, nbytes, starts.data_ptr(), n, fc, len(types), ccols, len(cols), C.byref(rows),
                        C.byref(err), None, 0, s)
    if st not in (A.OK, A.ERR_INVALID_ARG) or (st == A.ERR_INVALID_ARG and err.bad_cells == 0):
        _check(st, "yq_csv_parse")
    r = int(rows.value)
    batch = DeviceBatch([DeviceColumn(c.data[:r], c.type, c.nulls[:r]) for c in cols])
    if st == A.ERR_INVALID_ARG:
        raise CsvScanError(err, batch)
    return batch


def read_csv(data: bytes, project: list[str] | None = None, text_width: int = 256, device="cuda",
             stream=None) -> tuple[list[CsvColumn], DeviceBatch]:
    """A whole CSV file (header line included): schema from the header on the
    host, the body copied to the device and scanned there."""
    if data.startswith(b"\xef\xbb\xbf"):
        data = data[3:]  # csv-parser drops a UTF-8 byte-order mark
    nl = data.find(b"\n")
    header = data[: nl if nl >= 0 else len(data)].decode("utf-8", "replace")
    body = data[nl + 1:] if nl >= 0 else b""
    nl2 = body.find(b"\n")
    first = body[: nl2 if nl2 >= 0 else len(body)].decode("utf-8", "replace")
    schema = csv_schema(header, first)
    fields = list(range(len(schema))) if project is None else [[c.name for c in schema].index(p) for p in project]
    host = torch.frombuffer(bytearray(body), dtype=torch.uint8) if body else torch.empty(0, dtype=torch.uint8)
    text = host.to(device, non_blocking=False)
    batch = csv_scan(text, [c.type for c in schema], fields, text_width, stream)
    return [schema[f] for f in fields], batch


def csv_format(batch: DeviceBatch, stream=None) -> torch.Tensor:
    """The rows of a device batch as CSV text on the device (uint8 tensor),
    formatted as the reference's CsvWriter::batchToCsv formats them
    (include/engine/operators/csv_writer.hpp:24-76), without the header line."""
    L = lib()
    s = _stream(stream)
    cols, keep = batch.c()
    n = C.c_uint64(0)
    st = L.yq_csv_format(C.byref(cols), None, 0, C.byref(n), None, 0, s)
    if st not in (A.OK, A.ERR_CAPACITY):
        _check(st, "yq_csv_format")
    out = torch.empty(max(int(n.value), 1), dtype=torch.uint8, device="cuda")
    if n.value:
        _check(L.yq_csv_format(C.byref(cols), out.data_ptr(), int(n.value), C.byref(n), None, 0, s), "yq_csv_format")
    del keep
    return out[: int(n.value)]


def write_csv(names: list[str], batch: DeviceBatch, stream=None) -> bytes:
    """A whole CSV file as the reference writes it: the header line (column
    names joined by ',') and the formatted rows, copied to the host."""
    text = csv_format(batch, stream)
    return (",".join(names) + "\n").encode() + bytes(text.cpu().numpy().tobytes())


# ------------------------------------------------------------------ GROUP BY
def group_by_out_type(kind: int, in_type: int) -> int:
    if kind in (A.AGG_COUNT, A.AGG_COUNT_STAR):
        return A.INT64
    if kind == A.AGG_SUM:
        return A.FLOAT64 if in_type in (A.FLOAT32, A.FLOAT64) else A.INT64
    if kind == A.AGG_AVG:
        return A.FLOAT64
    return in_type


def group_by(batch: DeviceBatch, key: int, aggs: list[tuple[int, int]], capacity: int | None = None,
             stream=None) -> DeviceBatch:
    """SELECT key, aggs... GROUP BY key over a device batch (yq_group_by):
    `aggs` are (yq_agg_kind, input column) pairs; returns the key column then
    one column per aggregate, one row per group in ascending key order."""
    if len(aggs) > A.MAX_AGGREGATES:
        raise ValueError(f"group_by takes at most {A.MAX_AGGREGATES} aggregates a call, got {len(aggs)}")
    L = lib()
    s = _stream(stream)
    kc = batch.columns[key]
    cap = batch.rows if capacity is None else capacity
    outs = [DeviceColumn.empty(kc.type, max(cap, 1), kc.width if kc.type == A.TEXT else None, nulls=True)]
    for kind, col in aggs:
        t = group_by_out_type(kind, batch.columns[col].type if kind != A.AGG_COUNT_STAR else A.INT64)
        outs.append(DeviceColumn.empty(t, max(cap, 1), nulls=True))
    bc, keep = batch.c()
    ga = (A.GroupAgg * max(1, len(aggs)))(*[A.GroupAgg(k, c) for k, c in aggs])
    oc = (A.Column * len(outs))(*[c.c() for c in outs])
    g = C.c_uint32(0)
    _check(L.yq_group_by(C.byref(bc), key, ga, len(aggs), oc, cap, C.byref(g), None, 0, s), "yq_group_by")
    n = int(g.value)
    return DeviceBatch([DeviceColumn(c.data[:n], c.type, c.nulls[:n]) for c in outs])
