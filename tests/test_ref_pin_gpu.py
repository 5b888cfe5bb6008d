"""Pin the oracle to the reference itself: the reference's OWN kernels
(its src/kernels/*.cu built into oracle/_ref/libyqref.so by oracle/Makefile)
run on the same inputs as the oracle and as this repository's kernels.
Where the reference and DuckDB semantics agree the three must match exactly;
the known divergence (MAX(float) of all-negative input) is asserted as one.

ORDER BY order semantics (ascending/descending comparisons, ties taking the
earlier run) are pinned through the reference's merge-path kernel. Its radix
sort and filter compaction are not run: both sit on the reference's
prefix-sum kernels, whose shared-memory index macro shifts by 32 or more bits
(include/kernels/constants.hpp:12); on sm_100a the sort returned a
non-permutation and the filter path made an illegal memory access."""
import ctypes as C
import os

import numpy as np
import pytest
import torch

import oracle
from oracle import expr_eval
from yallasql_b200 import _abi as A
from yallasql_b200 import datagen, ops
from yallasql_b200.expr import Arith, Cast, ColumnRef

from helpers import dev_batch, dev_col, oracle_cols

pytestmark = pytest.mark.gpu

REF_LIB = os.path.join(os.path.dirname(oracle.__file__), "_ref", "libyqref.so")


@pytest.fixture(scope="module")
def ref(cuda):
    if not os.path.exists(REF_LIB):
        pytest.skip("oracle/_ref/libyqref.so not built (needs the reference sources: make -C oracle ref)")
    L = C.CDLL(REF_LIB)
    vp, u32, i32 = C.c_void_p, C.c_uint32, C.c_int
    L.ref_reduce.argtypes = [vp, vp, u32, i32, vp]
    L.ref_merge_f32.argtypes = [vp, vp, u32, u32, u32, i32, vp, vp, vp, vp]
    L.ref_join_eq_i32.argtypes = [vp, u32, vp, u32, vp, vp]
    L.ref_cross_col_i32.argtypes = [vp, vp, u32, u32, i32, vp, vp]
    L.ref_mul_cast_f32.argtypes = [vp, vp, u32, vp]
    return L


def d(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_reduce_pin(ref):
    rng = np.random.default_rng(4)
    n = 123_457
    f = rng.normal(0, 100, n).astype(np.float32)
    i = rng.integers(-1000, 1000, n).astype(np.int32)
    nulls = (rng.random(n) < 0.1).astype(np.uint8)
    df, di, dn = d(f), d(i), d(nulls)
    cols = {0: (f, nulls, A.FLOAT32), 1: (i, nulls, A.INT32)}
    want = expr_eval.aggregate(None, [expr_eval.Aggregate(A.AGG_SUM, ColumnRef(0, A.FLOAT32)),
                                      expr_eval.Aggregate(A.AGG_MIN, ColumnRef(0, A.FLOAT32)),
                                      expr_eval.Aggregate(A.AGG_MAX, ColumnRef(0, A.FLOAT32)),
                                      expr_eval.Aggregate(A.AGG_SUM, ColumnRef(1, A.INT32)),
                                      expr_eval.Aggregate(A.AGG_MIN, ColumnRef(1, A.INT32)),
                                      expr_eval.Aggregate(A.AGG_MAX, ColumnRef(1, A.INT32)),
                                      expr_eval.Aggregate(A.AGG_COUNT, ColumnRef(1, A.INT32))], cols, n)
    out = []
    for kind, x in ((0, df), (1, df), (2, df), (3, di), (4, di), (5, di), (6, di)):
        buf = (C.c_double if kind == 0 else (C.c_float if kind in (1, 2) else C.c_int))()
        assert ref.ref_reduce(x.data_ptr(), dn.data_ptr(), n, kind, C.addressof(buf)) == 0
        out.append(buf.value)
    assert abs(out[0] - want[0]) <= 1e-9 * abs(want[0])
    assert out[1:] == want[1:]


def test_reduce_pin_max_float_divergence(ref):
    f = -np.abs(np.random.default_rng(5).normal(0, 10, 1000)).astype(np.float32) - 1
    buf = C.c_float()
    df, dn = d(f), d(np.zeros(1000, np.uint8))  # the reference's kernels always read the null bytes
    assert ref.ref_reduce(df.data_ptr(), dn.data_ptr(), 1000, 2, C.addressof(buf)) == 0
    assert buf.value == np.float32(1.175494351e-38)  # reference: MAX starts at FLT_MIN
    assert ops.filter_aggregate(dev_batch([f]), None, [expr_eval.Aggregate(A.AGG_MAX, ColumnRef(0, A.FLOAT32))]) \
        == [float(f.max())]


@pytest.mark.parametrize("desc", [0, 1])
def test_merge_pin(ref, desc):
    rng = np.random.default_rng(7 + desc)
    a = np.sort(datagen.zipf_values(rng, 7000, distinct=300))
    b = np.sort(datagen.zipf_values(rng, 5000, distinct=300))
    if desc:
        a, b = a[::-1].copy(), b[::-1].copy()
    k = 9000
    C_ = torch.empty(k, dtype=torch.float32, device="cuda")
    idx = torch.empty(k, dtype=torch.int32, device="cuda")
    fa = torch.empty(k, dtype=torch.uint8, device="cuda")
    last = torch.zeros(1, dtype=torch.int32, device="cuda")
    da, db = d(a), d(b)
    assert ref.ref_merge_f32(da.data_ptr(), db.data_ptr(), len(a), len(b), k, desc, C_.data_ptr(), idx.data_ptr(),
                             fa.data_ptr(), last.data_ptr()) == 0
    both = np.concatenate([a, b])
    order = oracle.sort_perm(both, desc=bool(desc))[:k]
    np.testing.assert_array_equal(C_.cpu().numpy(), both[order])
    np.testing.assert_array_equal(fa.cpu().numpy(), (order < len(a)).astype(np.uint8))
    assert last.item() == int((order < len(a)).sum())


def test_join_pin(ref):
    rng = np.random.default_rng(8)
    left = rng.integers(0, 300, 2000).astype(np.int32)
    right = rng.integers(0, 300, 700).astype(np.int32)
    dl, dr = d(left), d(right)
    pairs = torch.empty(2 * 200_000, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert ref.ref_join_eq_i32(dl.data_ptr(), 2000, dr.data_ptr(), 700, pairs.data_ptr(), cnt.data_ptr()) == 0
    m = cnt.item()
    p = pairs[: 2 * m].cpu().numpy().view(np.uint32).reshape(m, 2)
    ref_set = sorted(map(tuple, p.tolist()))
    wl, wr = oracle.join_pairs([left], [right], [(0, 0, A.EQ)])
    assert ref_set == sorted(zip(wl.tolist(), wr.tolist()))
    gl, gr = ops.join_pairs(dev_batch([left]), dev_batch([right]), [(0, 0, A.EQ)])
    assert ref_set == list(zip(gl.cpu().numpy().view(np.uint32).tolist(), gr.cpu().numpy().view(np.uint32).tolist()))


def test_cross_product_pin(ref):
    x = np.arange(50, dtype=np.int32) * 3
    nulls = np.zeros(50, np.uint8)
    dx, dn = d(x), d(nulls)
    out = torch.empty(50 * 20, dtype=torch.int32, device="cuda")
    onl = torch.empty(50 * 20, dtype=torch.uint8, device="cuda")
    assert ref.ref_cross_col_i32(dx.data_ptr(), dn.data_ptr(), 50, 20, 1, out.data_ptr(), onl.data_ptr()) == 0
    np.testing.assert_array_equal(out.cpu().numpy(), np.repeat(x, 20))


def test_projection_arithmetic_pin(ref):
    t = datagen.sales_table(100_000, seed=3)
    dp, dd = d(t["price"]), d(t["discount"])
    out = torch.empty(100_000, dtype=torch.float32, device="cuda")
    assert ref.ref_mul_cast_f32(dp.data_ptr(), dd.data_ptr(), 100_000, out.data_ptr()) == 0
    e = Arith(A.MUL, ColumnRef(0, A.FLOAT32), Cast(ColumnRef(1, A.INT32), A.FLOAT32))
    cols = [t["price"], t["discount"]]
    want = expr_eval.evaluate(e, oracle_cols(cols), 100_000)[0]
    np.testing.assert_array_equal(out.cpu().numpy(), want)
    mine = ops.filter_project(dev_batch(cols), None, [e]).columns[0].data.cpu().numpy()
    np.testing.assert_array_equal(mine, want)
