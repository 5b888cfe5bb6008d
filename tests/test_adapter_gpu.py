"""The reference's kernel-layer API, forwarded to this library, on the GPU.

oracle/_ref/libyq_forward.so links yallasql_b200/adapter/yq_forward.cu (the
reference's YallaSQL::Kernel::launch_* templates defined by forwarding to
libyq_ops.so) with a harness that calls those templates exactly as the
reference's operators do. Results are checked against numpy / the oracle with
the reference's semantics: comparisons with the reference's functor names
(LE is "<", GE is ">"), SCALAR right operands and negation; AND/OR of masks;
the inclusive mask scan FilterOperator uses for its output slots; and
launch_radix_sort's contract (keys sorted in place, a callee-allocated stable
permutation, unsigned order for the uint32/uint64 keys the reference's key
transforms produce, byte order for 256-byte String slots).
"""
import ctypes as C
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libyq_forward.so")


@pytest.fixture(scope="module")
def fwd(cuda, yq):
    if not os.path.exists(LIB):
        pytest.skip("oracle/_ref/libyq_forward.so not built (make -C oracle ref)")
    return C.CDLL(LIB)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


OPS = [np.less, np.less_equal, np.greater, np.greater_equal, np.equal, np.not_equal]


@pytest.mark.parametrize("kind", ["i32", "f32", "i64"])
@pytest.mark.parametrize("scalar", [False, True])
def test_conditional_operators(fwd, kind, scalar):
    rng = np.random.default_rng(3)
    n = 100_003
    if kind == "i32":
        a, b, fn = rng.integers(-50, 50, n).astype(np.int32), rng.integers(-50, 50, n).astype(np.int32), fwd.fwd_compare_i32
    elif kind == "f32":
        a, b, fn = rng.normal(0, 5, n).astype(np.float32), rng.normal(0, 5, n).astype(np.float32), fwd.fwd_compare_f32
        a[::7] = b[::7]
    else:
        a = rng.integers(-(1 << 40), 1 << 40, n).astype(np.int64)
        b = rng.integers(-(1 << 40), 1 << 40, n).astype(np.int64)
        b[::5] = a[::5]
        fn = fwd.fwd_compare_i64
    if scalar:
        b = b[:1].copy()
    da, db = dev(a), dev(b)
    out = torch.empty(n, dtype=torch.uint8, device="cuda")
    for op in range(6):
        for neg in (0, 1):
            assert fn(C.c_void_p(da.data_ptr()), C.c_void_p(db.data_ptr()), int(scalar), op, neg,
                      C.c_void_p(out.data_ptr()), n) == 0
            want = OPS[op](a, b[0] if scalar else b) ^ bool(neg)
            np.testing.assert_array_equal(out.cpu().numpy().astype(bool), want)


def test_string_comparisons(fwd):
    rng = np.random.default_rng(4)
    n = 20_000
    pool = [b"", b"a", b"ab", b"abc", b"b", b"zz", b"hello", b"hellp"]
    ia, ib = rng.integers(0, len(pool), n), rng.integers(0, len(pool), n)
    sa, sb = np.zeros((n, 256), np.uint8), np.zeros((n, 256), np.uint8)
    for i in range(n):
        sa[i, :len(pool[ia[i]])] = np.frombuffer(pool[ia[i]], np.uint8)
        sb[i, :len(pool[ib[i]])] = np.frombuffer(pool[ib[i]], np.uint8)
    da, db = dev(sa), dev(sb)
    out = torch.empty(n, dtype=torch.uint8, device="cuda")
    ka = np.array([pool[i] for i in ia], dtype=object)
    kb = np.array([pool[i] for i in ib], dtype=object)
    for op in range(6):
        assert fwd.fwd_compare_str(C.c_void_p(da.data_ptr()), C.c_void_p(db.data_ptr()), 0, op, 0,
                                   C.c_void_p(out.data_ptr()), n) == 0
        want = np.array([OPS[op](x, y) for x, y in zip(ka, kb)])
        np.testing.assert_array_equal(out.cpu().numpy().astype(bool), want)


def test_and_or_and_mask_scan(fwd):
    rng = np.random.default_rng(5)
    n = 1_000_003
    a, b = (rng.random(n) < 0.5).astype(np.uint8), (rng.random(n) < 0.3).astype(np.uint8)
    da, db = dev(a), dev(b)
    out = torch.empty(n, dtype=torch.uint8, device="cuda")
    assert fwd.fwd_logic(C.c_void_p(da.data_ptr()), C.c_void_p(db.data_ptr()), 0, C.c_void_p(out.data_ptr()), n) == 0
    np.testing.assert_array_equal(out.cpu().numpy(), a & b)
    assert fwd.fwd_logic(C.c_void_p(da.data_ptr()), C.c_void_p(db.data_ptr()), 1, C.c_void_p(out.data_ptr()), n) == 0
    np.testing.assert_array_equal(out.cpu().numpy(), a | b)
    scan = torch.empty(n, dtype=torch.int32, device="cuda")
    assert fwd.fwd_prefix_sum_mask(C.c_void_p(da.data_ptr()), C.c_void_p(scan.data_ptr()), n) == 0
    np.testing.assert_array_equal(scan.cpu().numpy().view(np.uint32), np.cumsum(a, dtype=np.uint32))
    v = rng.integers(0, 1000, n).astype(np.uint32)
    dv = dev(v)
    assert fwd.fwd_prefix_sum_u32(C.c_void_p(dv.data_ptr()), C.c_void_p(scan.data_ptr()), n) == 0
    np.testing.assert_array_equal(scan.cpu().numpy().view(np.uint32), np.cumsum(v, dtype=np.uint32))


@pytest.mark.parametrize("desc", [0, 1])
def test_radix_sort_contract(fwd, desc):
    rng = np.random.default_rng(6 + desc)
    n = 300_001
    # uint32 keys as the reference's float_to_uint32 makes them
    f = rng.normal(0, 100, n).astype(np.float32)
    f[1::3] = f[0::3][: len(f[1::3])]  # ties
    df = dev(f)
    keys = torch.empty(n, dtype=torch.int32, device="cuda")
    assert fwd.fwd_float_to_uint32(C.c_void_p(df.data_ptr()), C.c_void_p(keys.data_ptr()), n) == 0
    k32 = keys.cpu().numpy().view(np.uint32).copy()
    neg = f < 0
    want_t = np.where(neg, ~f.view(np.uint32), f.view(np.uint32) ^ np.uint32(0x80000000))
    np.testing.assert_array_equal(k32, want_t)
    idx = torch.empty(n, dtype=torch.int32, device="cuda")
    assert fwd.fwd_radix_sort_u32(C.c_void_p(keys.data_ptr()), C.c_void_p(idx.data_ptr()), n, desc) == 0
    order = np.argsort(-k32.astype(np.int64) if desc else k32, kind="stable")
    np.testing.assert_array_equal(idx.cpu().numpy(), order)
    np.testing.assert_array_equal(keys.cpu().numpy().view(np.uint32), k32[order])  # keys sorted in place
    # uint64 keys (dates read as unsigned, values above 2^63 included)
    k64 = rng.integers(0, 1 << 62, n).astype(np.uint64) * np.uint64(3)
    k64[1::3] = k64[0::3][: len(k64[1::3])]
    dk = dev(k64.view(np.int64))
    assert fwd.fwd_radix_sort_u64(C.c_void_p(dk.data_ptr()), C.c_void_p(idx.data_ptr()), n, desc) == 0
    order = np.lexsort((np.arange(n), ~k64)) if desc else np.argsort(k64, kind="stable")
    np.testing.assert_array_equal(idx.cpu().numpy(), order)
    np.testing.assert_array_equal(dk.cpu().numpy().view(np.uint64), k64[order])


@pytest.mark.parametrize("desc", [0, 1])
def test_radix_sort_strings(fwd, desc):
    """256-byte String slots (MAX_STR), values agreeing on up to 100 bytes."""
    rng = np.random.default_rng(8 + desc)
    n = 40_000
    words = [("q" * int(rng.integers(0, 100)) + "".join(rng.choice(list("abcd"), 4))).encode() for _ in range(n)]
    s = np.zeros((n, 256), np.uint8)
    for i, w in enumerate(words):
        s[i, :len(w)] = np.frombuffer(w, np.uint8)
    ds = dev(s)
    idx = torch.empty(n, dtype=torch.int32, device="cuda")
    assert fwd.fwd_radix_sort_str(C.c_void_p(ds.data_ptr()), C.c_void_p(idx.data_ptr()), n, desc) == 0
    keys = [bytes(r) for r in s]
    order = sorted(range(n), key=lambda i: keys[i], reverse=bool(desc))  # stable: ties keep input order
    np.testing.assert_array_equal(idx.cpu().numpy(), np.array(order))
    np.testing.assert_array_equal(ds.cpu().numpy(), s[np.array(order)])
