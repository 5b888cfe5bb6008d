"""Reference-compatible element kernels (one per YallaSQL::Kernel::launch_*):
results must equal the reference's semantics restated with numpy
(DIV/MOD by zero -> 0, static_cast truncation, null cells skipped by the
filter move, strcmp order on NUL-padded slots, raw-value merge path)."""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle
from yallasql_b200 import _abi as A
from yallasql_b200 import datagen

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def operand(t, type_, width, scalar=False):
    return A.Operand(t.data_ptr(), type_, width, int(scalar))


def s():
    return torch.cuda.current_stream().cuda_stream


CMP = {A.LT: np.less, A.LE: np.less_equal, A.GT: np.greater, A.GE: np.greater_equal, A.EQ: np.equal,
       A.NE: np.not_equal}


@pytest.mark.parametrize("op", list(CMP))
@pytest.mark.parametrize("scalar", [False, True])
@pytest.mark.parametrize("neg", [0, 1])
def test_compare_numeric(cuda, yq, op, scalar, neg):
    rng = np.random.default_rng(op * 4 + neg)
    n = 10_007
    for arr, t in ((rng.integers(-5, 5, n).astype(np.int32), A.INT32),
                   (rng.normal(0, 2, n).astype(np.float32), A.FLOAT32),
                   (rng.integers(-5, 5, n).astype(np.int64), A.INT64)):
        rhs = arr[:1].copy() if scalar else rng.permutation(arr)
        out = torch.empty(n, dtype=torch.uint8, device="cuda")
        la, ra = dev(arr), dev(rhs)  # keep both alive across the call
        st = yq.yq_compare(operand(la, t, arr.itemsize), operand(ra, t, arr.itemsize, scalar), op, neg,
                           out.data_ptr(), n, s())
        assert st == A.OK
        want = CMP[op](arr, rhs[0] if scalar else rhs) ^ bool(neg)
        np.testing.assert_array_equal(out.cpu().numpy().astype(bool), want)


def test_compare_text_strcmp_order(cuda, yq):
    words = ["", "a", "ab", "abc", "b", "hello", "hellp", "\xff"]
    a = datagen.text_slots(words * 3, width=256)
    b = datagen.text_slots(list(reversed(words)) * 3, width=256)
    n = len(a)
    for op in CMP:
        out = torch.empty(n, dtype=torch.uint8, device="cuda")
        da, db = dev(a), dev(b)
        assert yq.yq_compare(operand(da, A.TEXT, 256), operand(db, A.TEXT, 256), op, 0, out.data_ptr(), n,
                             s()) == A.OK
        sign = np.array([(x > y) - (x < y) for x, y in zip([w.encode() for w in words * 3],
                                                            [w.encode() for w in list(reversed(words)) * 3])])
        np.testing.assert_array_equal(out.cpu().numpy().astype(bool), CMP[op](sign, 0))


@pytest.mark.parametrize("is_or", [0, 1])
def test_logic(cuda, yq, is_or):
    rng = np.random.default_rng(is_or)
    a = rng.integers(0, 2, 5000).astype(np.uint8)
    b = rng.integers(0, 2, 5000).astype(np.uint8)
    out = torch.empty(5000, dtype=torch.uint8, device="cuda")
    da, db = dev(a), dev(b)
    assert yq.yq_logic(operand(da, A.BOOL, 1), operand(db, A.BOOL, 1), is_or, out.data_ptr(), 5000,
                       s()) == A.OK
    want = (a | b) if is_or else (a & b)
    np.testing.assert_array_equal(out.cpu().numpy(), want)


@pytest.mark.parametrize("op", [A.ADD, A.SUB, A.MUL, A.DIV, A.MOD])
def test_binary_reference_semantics(cuda, yq, op):
    rng = np.random.default_rng(op)
    n = 4096
    a = rng.integers(-100, 100, n).astype(np.int32)
    b = rng.integers(-3, 3, n).astype(np.int32)  # includes zeros
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    da, db = dev(a), dev(b)
    assert yq.yq_binary(operand(da, A.INT32, 4), operand(db, A.INT32, 4), op, out.data_ptr(), n, s()) == A.OK
    bz = np.where(b == 0, 1, b)
    with np.errstate(all="ignore"):
        want = {A.ADD: a + b, A.SUB: a - b, A.MUL: a * b,
                A.DIV: np.where(b == 0, 0, np.trunc(a / bz)).astype(np.int32),
                A.MOD: np.where(b == 0, 0, np.fmod(a, bz)).astype(np.int32)}[op]
    np.testing.assert_array_equal(out.cpu().numpy(), want)
    f = rng.normal(0, 10, n).astype(np.float32)
    g = np.where(rng.random(n) < 0.1, 0, rng.normal(0, 3, n)).astype(np.float32)
    outf = torch.empty(n, dtype=torch.float32, device="cuda")
    if op != A.MOD:
        df, dg = dev(f), dev(g)
        assert yq.yq_binary(operand(df, A.FLOAT32, 4), operand(dg, A.FLOAT32, 4), op, outf.data_ptr(), n,
                            s()) == A.OK
        with np.errstate(all="ignore"):
            wf = {A.ADD: f + g, A.SUB: f - g, A.MUL: f * g, A.DIV: np.where(g == 0, 0, f / np.where(g == 0, 1, g))}[op]
        np.testing.assert_array_equal(outf.cpu().numpy(), wf.astype(np.float32))


def test_cast_truncates_like_static_cast(cuda, yq):
    f = np.array([1.9, -1.9, 2.5, -2.5, 0.0, 1e6 + 0.7], np.float32)
    out = torch.empty(len(f), dtype=torch.int32, device="cuda")
    df = dev(f)
    assert yq.yq_cast(df.data_ptr(), A.FLOAT32, out.data_ptr(), A.INT32, len(f), s()) == A.OK
    np.testing.assert_array_equal(out.cpu().numpy(), f.astype(np.int32))
    i = np.array([1, -7, 123456789], np.int32)
    outf = torch.empty(3, dtype=torch.float32, device="cuda")
    di = dev(i)
    assert yq.yq_cast(di.data_ptr(), A.INT32, outf.data_ptr(), A.FLOAT32, 3, s()) == A.OK
    np.testing.assert_array_equal(outf.cpu().numpy(), i.astype(np.float32))


@pytest.mark.parametrize("n", [1, 2047, 2048, 2049, 3_000_001])
def test_prefix_sums(cuda, yq, n):
    rng = np.random.default_rng(n)
    m = rng.integers(0, 2, n).astype(np.uint8)
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    dm = dev(m)
    assert yq.yq_prefix_sum_mask(dm.data_ptr(), out.data_ptr(), n, None, 0, s()) == A.OK
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), np.cumsum(m, dtype=np.uint32))
    u = rng.integers(0, 1000, n).astype(np.uint32)
    du = dev(u)
    assert yq.yq_prefix_sum_u32(du.data_ptr(), out.data_ptr(), n, None, 0, s()) == A.OK
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), np.cumsum(u, dtype=np.uint32))


@pytest.mark.parametrize("offset", [1, 3, 4])
def test_prefix_sums_unaligned_input(cuda, yq, offset):
    """Inputs that start off a 16-byte boundary take the element-wise loads;
    several tiles, a partial last tile."""
    n = 300_001
    rng = np.random.default_rng(offset)
    m = rng.integers(0, 2, n + offset).astype(np.uint8)
    dm = dev(m)
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    assert yq.yq_prefix_sum_mask(dm.data_ptr() + offset, out.data_ptr(), n, None, 0, s()) == A.OK
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), np.cumsum(m[offset:], dtype=np.uint32))
    u = rng.integers(0, 1000, n + offset).astype(np.uint32)
    du = dev(u)
    assert yq.yq_prefix_sum_u32(du.data_ptr() + 4 * offset, out.data_ptr(), n, None, 0, s()) == A.OK
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), np.cumsum(u[offset:], dtype=np.uint32))


def test_move_rows_filter_skips_null_cells(cuda, yq):
    rng = np.random.default_rng(1)
    n = 10_000
    x = rng.integers(0, 1000, n).astype(np.int64)
    mask = rng.integers(0, 2, n).astype(np.uint8)
    nulls = (rng.random(n) < 0.1).astype(np.uint8)
    mp = np.cumsum(mask, dtype=np.uint32)
    out = torch.full((int(mp[-1]),), -1, dtype=torch.int64, device="cuda")
    dst = A.Column(out.data_ptr(), None, A.INT64, 8)
    xs, ns, ms, mps = dev(x), dev(nulls), dev(mask), dev(mp)
    src = A.Column(xs.data_ptr(), ns.data_ptr(), A.INT64, 8)
    assert yq.yq_move_rows_filter(C.byref(src), mps.data_ptr(), ms.data_ptr(), n, C.byref(dst), s()) == A.OK
    want = np.full(int(mp[-1]), -1, np.int64)
    keep = (mask == 1) & (nulls == 0)
    want[mp[keep] - 1] = x[keep]
    np.testing.assert_array_equal(out.cpu().numpy(), want)


def test_move_rows_join_and_merge(cuda, yq):
    rng = np.random.default_rng(2)
    x = rng.integers(0, 100, 500).astype(np.int32)
    y = rng.integers(0, 100, 300).astype(np.int32)
    pairs = np.stack([rng.integers(0, 500, 1000), rng.integers(0, 300, 1000)], axis=1).astype(np.uint32).ravel()
    xs, ys, ps = dev(x), dev(y), dev(pairs)
    out = torch.empty(1000, dtype=torch.int32, device="cuda")
    for side, src_arr, src_t in ((0, x, xs), (1, y, ys)):
        src = A.Column(src_t.data_ptr(), None, A.INT32, 4)
        dst = A.Column(out.data_ptr(), None, A.INT32, 4)
        assert yq.yq_move_rows_join(C.byref(src), ps.data_ptr(), 1000, side, C.byref(dst), s()) == A.OK
        np.testing.assert_array_equal(out.cpu().numpy(), src_arr[pairs[side::2]])
    idx = rng.integers(0, 300, 800).astype(np.uint32)
    fa = rng.integers(0, 2, 800).astype(np.uint8)
    ids, fas = dev(idx), dev(fa)
    out2 = torch.empty(800, dtype=torch.int32, device="cuda")
    for asc in (1, 0):
        a_c, b_c = A.Column(xs.data_ptr(), None, A.INT32, 4), A.Column(ys.data_ptr(), None, A.INT32, 4)
        d_c = A.Column(out2.data_ptr(), None, A.INT32, 4)
        assert yq.yq_move_rows_merge(C.byref(a_c), C.byref(b_c), ids.data_ptr(), fas.data_ptr(), asc, 800,
                                     C.byref(d_c), s()) == A.OK
        want = np.where(fa == 1, x[idx], y[idx])
        np.testing.assert_array_equal(out2.cpu().numpy(), want if asc else want[::-1])


def test_reductions(cuda, yq):
    rng = np.random.default_rng(3)
    n = 100_003
    f = rng.normal(0, 100, n).astype(np.float32)
    nulls = (rng.random(n) < 0.1).astype(np.uint8)
    fs, ns = dev(f), dev(nulls)
    acc = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert yq.yq_reduce(fs.data_ptr(), A.FLOAT32, ns.data_ptr(), n, A.AGG_SUM, acc.data_ptr(), s()) == A.OK
    assert abs(acc.item() - f[nulls == 0].astype(np.float64).sum()) <= 1e-6 * abs(f[nulls == 0]).sum()
    mx = torch.full((1,), -np.inf, dtype=torch.float32, device="cuda")
    assert yq.yq_reduce(fs.data_ptr(), A.FLOAT32, ns.data_ptr(), n, A.AGG_MAX, mx.data_ptr(), s()) == A.OK
    assert mx.item() == f[nulls == 0].max()
    i = rng.integers(-1000, 1000, n).astype(np.int32)
    isum = torch.zeros(1, dtype=torch.int32, device="cuda")
    di = dev(i)
    assert yq.yq_reduce(di.data_ptr(), A.INT32, None, n, A.AGG_SUM, isum.data_ptr(), s()) == A.OK
    assert isum.item() == int(i.astype(np.int64).sum())
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert yq.yq_reduce(None, A.INT32, ns.data_ptr(), n, A.AGG_COUNT, cnt.data_ptr(), s()) == A.OK
    assert cnt.item() == int((nulls == 0).sum())


def test_key_transform_round_trip(cuda, yq):
    f = np.array([-2.5, -0.0, 0.0, 1.0, np.inf, -np.inf], np.float32)
    k = torch.empty(len(f), dtype=torch.int32, device="cuda")
    back = torch.empty(len(f), dtype=torch.int32, device="cuda")
    fs = dev(f)
    assert yq.yq_key_transform(fs.data_ptr(), A.FLOAT32, k.data_ptr(), len(f), 0, s()) == A.OK
    keys = k.cpu().numpy().view(np.uint32)
    assert list(np.argsort(keys, kind="stable")) == [5, 0, 1, 2, 3, 4]
    assert yq.yq_key_transform(k.data_ptr(), A.FLOAT32, back.data_ptr(), len(f), 1, s()) == A.OK
    np.testing.assert_array_equal(back.cpu().numpy().view(np.float32), f)


@pytest.mark.parametrize("desc", [0, 1])
def test_merge_path_reference_semantics(cuda, yq, desc):
    rng = np.random.default_rng(desc)
    a = np.sort(rng.integers(0, 50, 3000)).astype(np.int32)
    b = np.sort(rng.integers(0, 50, 2000)).astype(np.int32)
    if desc:
        a, b = a[::-1].copy(), b[::-1].copy()
    k = 4000
    keys = torch.empty(k, dtype=torch.int32, device="cuda")
    idx = torch.empty(k, dtype=torch.int32, device="cuda")
    fa = torch.empty(k, dtype=torch.uint8, device="cuda")
    last = torch.zeros(1, dtype=torch.int32, device="cuda")
    da, db = dev(a), dev(b)
    assert yq.yq_merge_path(da.data_ptr(), db.data_ptr(), A.INT32, 4, desc, len(a), len(b), k,
                            keys.data_ptr(), idx.data_ptr(), fa.data_ptr(), last.data_ptr(), s()) == A.OK
    both = np.concatenate([a, b])
    src = np.concatenate([np.ones(len(a), np.uint8), np.zeros(len(b), np.uint8)])
    order = oracle.sort_perm(both, desc=bool(desc))  # stable: ties keep A first
    np.testing.assert_array_equal(keys.cpu().numpy(), both[order][:k])
    np.testing.assert_array_equal(fa.cpu().numpy(), src[order][:k])
    assert last.item() == int(src[order][:k].sum())


def test_cross_product_col(cuda, yq):
    x = np.arange(7, dtype=np.int32)
    out = torch.empty(7 * 5, dtype=torch.int32, device="cuda")
    xs = dev(x)
    for is_left in (1, 0):
        src = A.Column(xs.data_ptr(), None, A.INT32, 4)
        dst = A.Column(out.data_ptr(), None, A.INT32, 4)
        L, R = (7, 5) if is_left else (5, 7)
        assert yq.yq_cross_product_col(C.byref(src), L, R, is_left, C.byref(dst), s()) == A.OK
        want = np.repeat(x, 5) if is_left else np.tile(x, 5)
        np.testing.assert_array_equal(out.cpu().numpy(), want)
