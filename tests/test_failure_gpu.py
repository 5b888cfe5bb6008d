"""Failure paths of the bounded device waits, and launches from two host threads.

The reference's kernels either finish or hang, and its host code exits on any
CUDA error (include/utils/macros.hpp:6-22). Here every spin wait carries a poll
bound; when it runs out the kernel records kErrTimeout and the entry point
returns YQ_ERR_TIMEOUT instead of waiting forever. These tests make a wait run
out on purpose (a look-back predecessor that never publishes, with the bound
lowered to a few thousand polls), check the status, and check that the device
still serves ordinary calls afterwards. No kernel here faults or hangs.
"""
import threading
import time

import numpy as np
import pytest
import torch

import oracle
from yallasql_b200 import _abi as A
from yallasql_b200 import datagen, ops
from yallasql_b200.expr import And, Compare, Constant, ColumnRef, between

pytestmark = pytest.mark.gpu


def test_lookback_wait_runs_out_and_returns_timeout(cuda, yq):
    ws = torch.zeros(64, dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    t0 = time.perf_counter()
    st = yq.yq_debug_lookback_stall(2000, ws.data_ptr(), ws.numel(), s)
    dt = time.perf_counter() - t0
    assert st == A.ERR_TIMEOUT
    assert dt < 5.0
    # the stalled tile published an inclusive value on giving up: nothing after it waits
    words = ws.view(torch.int64).cpu().numpy().view(np.uint64)
    assert words[1] >> np.uint64(62) == 2  # kFlagIncl
    # the bound is checked: an out-of-range limit is refused before any launch
    assert yq.yq_debug_lookback_stall(0, ws.data_ptr(), ws.numel(), s) == A.ERR_INVALID_ARG
    assert yq.yq_debug_lookback_stall(2000, ws.data_ptr(), 8, s) == A.ERR_INVALID_ARG


def _sales_query(rows, seed):
    t = datagen.sales_table(rows, seed=seed)
    b = ops.DeviceBatch([ops.DeviceColumn(torch.from_numpy(t["price"]).cuda(), A.FLOAT32),
                         ops.DeviceColumn(torch.from_numpy(t["qty"]).cuda(), A.INT32),
                         ops.DeviceColumn(torch.from_numpy(t["discount"]).cuda(), A.INT32)])
    pred = And(between(ColumnRef(2, A.INT32), Constant(1, A.INT32), Constant(3, A.INT32)),
               Compare(A.LT, ColumnRef(1, A.INT32), Constant(25, A.INT32)))
    plan = ops.ProjectPlan([A.FLOAT32, A.INT32, A.INT32], [4, 4, 4], pred, [0, 1])
    keep = (t["discount"] >= 1) & (t["discount"] <= 3) & (t["qty"] < 25)
    return b, plan, t["price"][keep], t["qty"][keep]


def test_device_usable_after_a_timeout(cuda, yq):
    ws = torch.zeros(64, dtype=torch.uint8, device="cuda")
    assert yq.yq_debug_lookback_stall(500, ws.data_ptr(), ws.numel(),
                                      torch.cuda.current_stream().cuda_stream) == A.ERR_TIMEOUT
    b, plan, wp, wq = _sales_query(500_000, 3)
    out = plan.run(b)
    np.testing.assert_array_equal(out.columns[0].data.cpu().numpy(), wp)
    np.testing.assert_array_equal(out.columns[1].data.cpu().numpy(), wq)


def test_two_host_threads_launch_concurrently(cuda, yq):
    """Launch settings (shared-memory opt-ins, resident-grid sizes) are cached
    per device under a lock: two host threads, each on its own stream, run
    WHERE + projection, ORDER BY and the CSV scan at the same time and get the
    single-threaded results."""
    jobs = [_sales_query(300_000 + 7919 * i, 10 + i) for i in range(2)]
    tabs = [datagen.order_table(200_000, seed=20 + i, dist="zipf") for i in range(2)]
    errors = []

    def work(i):
        try:
            torch.cuda.set_device(0)
            st = torch.cuda.Stream()
            with torch.cuda.stream(st):
                b, plan, wp, wq = jobs[i]
                t = tabs[i]
                key = ops.DeviceColumn(torch.from_numpy(t["key"]).cuda(), A.FLOAT32)
                ids = ops.DeviceColumn(torch.from_numpy(t["id"]).cuda(), A.INT64)
                for _ in range(20):
                    out = plan.run(b, stream=st)
                    srt = ops.sort_batch(ops.DeviceBatch([key, ids]), 0, descending=True, stream=st)
                st.synchronize()
                np.testing.assert_array_equal(out.columns[0].data.cpu().numpy(), wp)
                np.testing.assert_array_equal(out.columns[1].data.cpu().numpy(), wq)
                perm = oracle.sort_perm(t["key"], desc=True)
                np.testing.assert_array_equal(srt.columns[1].data.cpu().numpy(), t["id"][perm])
        except Exception as ex:  # reported on the main thread
            errors.append(ex)

    th = [threading.Thread(target=work, args=(i,)) for i in range(2)]
    for x in th:
        x.start()
    for x in th:
        x.join(timeout=300)
    assert not any(x.is_alive() for x in th)
    assert not errors, errors
