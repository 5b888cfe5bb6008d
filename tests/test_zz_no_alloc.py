"""yq_filter_project_noalloc: WHERE + projection without any device allocation.

Some hosts cannot let a library allocate device memory during a call: an
engine that embeds this library and hands out every byte of device memory
from its own fixed arena, or a serving loop that cannot afford allocator calls
(and the synchronisation they can cause) on its latency path. For them the
library keeps the look-back scratch of one operator in a static device array.
This test calls that entry point through the C ABI and checks that two calls
in a row produce exactly what the allocating entry point, yq_filter_project,
produces (exact equality: integer, date, text and float values are copied or
computed identically, not accumulated), and that batches above the array's
row limit are refused before any device work.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from yallasql_b200 import _abi as A
from yallasql_b200 import datagen, ops
from yallasql_b200.expr import And, Arith, Cast, ColumnRef, Compare, Constant, between

pytestmark = pytest.mark.gpu


def _table(rows):
    t = datagen.sales_table(rows, seed=9)
    cols = [ops.DeviceColumn(torch.from_numpy(t["price"]).cuda(), A.FLOAT32),
            ops.DeviceColumn(torch.from_numpy(t["qty"]).cuda(), A.INT32),
            ops.DeviceColumn(torch.from_numpy(t["discount"]).cuda(), A.INT32),
            ops.DeviceColumn(torch.from_numpy(t["category"]).cuda(), A.TEXT),
            ops.DeviceColumn(torch.from_numpy(t["updated_at"]).cuda(), A.DATETIME)]
    return ops.DeviceBatch(cols)


def _plan():
    price, qty, disc = ColumnRef(0, A.FLOAT32), ColumnRef(1, A.INT32), ColumnRef(2, A.INT32)
    pred = And(between(disc, Constant(1, A.INT32), Constant(3, A.INT32)), Compare(A.LT, qty, Constant(25, A.INT32)),
               Compare(A.NE, ColumnRef(3, A.TEXT), Constant(datagen.EXCLUDED_CATEGORY, A.TEXT)))
    select = [3, 4, 0, Arith(A.MUL, price, Cast(disc, A.FLOAT32))]
    return ops.ProjectPlan([A.FLOAT32, A.INT32, A.INT32, A.TEXT, A.DATETIME], [4, 4, 4, 16, 8], pred, select)


def _outputs(plan, cap):
    return [ops.DeviceColumn.empty(t, cap, w if t == A.TEXT else None, nulls=True)
            for t, w in zip(plan.out_types, plan.out_widths)]


def _noalloc(lib, plan, batch, outs, count_device=None):
    """One call of yq_filter_project_noalloc into `outs` (allocated by torch
    before the call, as a host that owns its memory would hand them in).
    With `count_device` the call returns without waiting and the surviving
    row count is read from that device word afterwards."""
    cap = batch.rows
    oc = (A.Column * len(outs))(*[o.c() for o in outs])
    b, keep = batch.c()
    cnt = C.c_uint32(0)
    st = lib.yq_filter_project_noalloc(C.byref(b), C.byref(plan.pred.prog), C.byref(plan.consts), plan.proj,
                                       len(plan.select), oc, cap,
                                       None if count_device is None else
                                       C.cast(count_device.data_ptr(), C.POINTER(C.c_uint32)),
                                       None if count_device is not None else C.byref(cnt),
                                       torch.cuda.current_stream().cuda_stream)
    assert st == A.OK, lib.yq_status_string(st)
    n = int(count_device.item()) if count_device is not None else cnt.value
    return [o.slice(0, n) for o in outs]


def _same(got, want):
    assert len(got) == len(want.columns)
    for g, w in zip(got, want.columns):
        assert g.rows == w.rows
        assert torch.equal(g.data, w.data)
        assert torch.equal(g.nulls, w.nulls)


def test_noalloc_matches_allocating_entry_point_twice(cuda, yq):
    batch = _table(300_001)
    plan = _plan()
    want = plan.run(batch)  # yq_filter_project, library-allocated workspace
    assert 0 < want.rows < batch.rows
    for _ in range(2):  # the second call must not see the first call's scratch
        _same(_noalloc(yq, plan, batch, _outputs(plan, batch.rows)), want)


def test_noalloc_allocates_nothing_large_then_small(cuda, yq):
    """Device memory in use is the same before and after a call, and a larger
    batch followed by a smaller one leaves nothing of the first in the second
    (the scratch is cleared as far as the second call reads it). One call
    reports its count through a device word instead of the host."""
    plan = _plan()
    big, small = _table(2_000_003), _table(70_001)
    want_big, want_small = plan.run(big), plan.run(small)
    outs_big, outs_small = _outputs(plan, big.rows), _outputs(plan, small.rows)
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    _noalloc(yq, plan, small, outs_small)  # warm-up: loads the kernel, looks up the scratch address
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    got_big = _noalloc(yq, plan, big, outs_big)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    got_small = _noalloc(yq, plan, small, outs_small, count_device=count)
    torch.cuda.synchronize()
    free2, _ = torch.cuda.mem_get_info()
    assert free0 == free1 == free2, (free0, free1, free2)
    _same(got_big, want_big)
    _same(got_small, want_small)


def test_noalloc_rejects_batches_above_its_limit(cuda, yq):
    plan = _plan()
    small = _table(16)
    cols, keep = small.c()
    cols.rows = A_MAX_ROWS + 1  # pointers are never touched: the size check comes first
    outs = (A.Column * 4)()
    cnt = C.c_uint32(7)
    st = yq.yq_filter_project_noalloc(C.byref(cols), C.byref(plan.pred.prog), C.byref(plan.consts), plan.proj, 4,
                                      outs, 0, None, C.byref(cnt), None)
    assert st == A.ERR_INVALID_ARG


A_MAX_ROWS = 1 << 26  # YQ_FILTER_PROJECT_NOALLOC_MAX_ROWS in include/yq_ops.h
