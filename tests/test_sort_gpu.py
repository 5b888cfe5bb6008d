"""ORDER BY parity: the onesweep radix argsort must reproduce the oracle's
stable permutation exactly (ties in input order), for every key type, both
directions, nulls first/last, digit widths 4/6/8, segments and multi-key."""
import zlib

import numpy as np
import pytest
import torch

import oracle
from yallasql_b200 import _abi as A
from yallasql_b200 import datagen, ops

from helpers import dev_col

pytestmark = pytest.mark.gpu


def gpu_perm(col, **kw):
    return ops.sort_indices(col, **kw).cpu().numpy().view(np.uint32)


def keys(kind, n, rng):
    if kind == "f32_uniform":
        return rng.uniform(-1e6, 1e6, n).astype(np.float32)
    if kind == "f32_zipf":
        return datagen.zipf_values(rng, n, distinct=min(1000, max(1, n)))
    if kind == "f32_equal":
        return np.full(n, 42.0, np.float32)
    if kind == "f32_special":
        pool = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, -np.nan, 1.5, -1.5, 1e-40, -1e-40,
                         np.finfo(np.float32).max, np.finfo(np.float32).min], np.float32)
        return pool[rng.integers(0, len(pool), n)]
    if kind == "i32":
        return rng.integers(-50, 50, n).astype(np.int32)
    if kind == "i32_full":
        return rng.integers(np.iinfo(np.int32).min, np.iinfo(np.int32).max, n, dtype=np.int32, endpoint=True)
    if kind == "i64":
        return rng.integers(-(1 << 62), 1 << 62, n).astype(np.int64)
    if kind == "date":
        return rng.integers(-86400 * 365 * 10, datagen.DATE_HI, n).astype(np.int64)
    if kind == "text16":
        words = ["", "a", "ab", "abc", "b", "ba", "zzz", "hello", "hello world", "x" * 15, "\xff"]
        return datagen.text_slots([words[j] for j in rng.integers(0, len(words), n)])
    if kind == "text256":
        words = ["", "pear", "apple", "apples", "banana", "b" * 20, "b" * 19 + "c"]
        return datagen.text_slots([words[j] for j in rng.integers(0, len(words), n)], width=256)
    raise ValueError(kind)


KINDS = ["f32_uniform", "f32_zipf", "f32_equal", "f32_special", "i32", "i32_full", "i64", "date", "text16",
         "text256"]


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("desc", [False, True])
@pytest.mark.parametrize("n", [1, 100, 4097, 123_457])
def test_sort_matches_oracle(cuda, kind, desc, n):
    rng = np.random.default_rng(zlib.crc32(f"{kind}{n}".encode()))
    k = keys(kind, n, rng)
    t = A.DATETIME if kind == "date" else None
    got = gpu_perm(dev_col(k, t), descending=desc)
    want = oracle.sort_perm(k, desc=desc, type_=t)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("kind", ["f32_uniform", "i32", "i64", "text16"])
@pytest.mark.parametrize("nulls_first", [False, True])
@pytest.mark.parametrize("desc", [False, True])
def test_sort_nulls(cuda, kind, nulls_first, desc):
    rng = np.random.default_rng(7)
    n = 20_000
    k = keys(kind, n, rng)
    nl = rng.random(n) < 0.2
    got = gpu_perm(dev_col(k, None, nl), descending=desc, nulls_first=nulls_first)
    want = oracle.sort_perm(k, desc=desc, nulls=nl, nulls_first=nulls_first)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("bits", [4, 6, 8])
@pytest.mark.parametrize("kind", ["f32_uniform", "i64"])
@pytest.mark.parametrize("keep_trivial", [False, True])
def test_sort_digit_widths(cuda, bits, kind, keep_trivial):
    rng = np.random.default_rng(bits)
    k = keys(kind, 300_001, rng)
    cfg = ops.sort_config(bits, keep_trivial)
    got = gpu_perm(dev_col(k), descending=True, config=cfg)
    np.testing.assert_array_equal(got, oracle.sort_perm(k, desc=True))


def test_sort_segments_runs(cuda):
    rng = np.random.default_rng(11)
    sizes = [0, 1, 1000, 116_480, 5, 0, 70_000, 4096, 4097]
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint32)
    k = keys("f32_zipf", int(offs[-1]), rng)
    perm = ops.sort_segments(dev_col(k), [int(x) for x in offs], descending=True).cpu().numpy().view(np.uint32)
    want = oracle.sort_perm(k, desc=True, segments=offs)
    np.testing.assert_array_equal(perm, want)


def test_multi_key(cuda):
    rng = np.random.default_rng(12)
    n = 100_000
    k0 = rng.integers(0, 10, n).astype(np.int32)
    k1 = datagen.text_slots([["x", "y", "z"][j] for j in rng.integers(0, 3, n)])
    k2 = rng.uniform(0, 1, n).astype(np.float32)
    perm = ops.sort_indices_multi([dev_col(k0), dev_col(k1), dev_col(k2)], [True, False, True])
    want = oracle.sort_perm_multi([k0, k1, k2], [True, False, True])
    np.testing.assert_array_equal(perm.cpu().numpy().view(np.uint32), want)


def test_sort_batch_gathers_every_column(cuda):
    t = datagen.order_table(50_000, seed=1)
    b = ops.DeviceBatch([dev_col(t["key"]), dev_col(t["id"]), dev_col(t["txt"]), dev_col(t["d"], A.DATETIME)])
    out = ops.sort_batch(b, 0, descending=True)
    perm = oracle.sort_perm(t["key"], desc=True)
    for col, name in zip(out.columns, ["key", "id", "txt", "d"]):
        np.testing.assert_array_equal(col.data.cpu().numpy(), t[name][perm])


def test_large_sort_properties(cuda):
    """16M keys: the permutation is a bijection and the keys come out ordered
    (size-independent properties; exact parity is checked at smaller sizes)."""
    n = 16_000_000
    g = torch.Generator(device="cuda").manual_seed(5)
    k = (torch.rand(n, device="cuda", generator=g) * 2e6 - 1e6).to(torch.float32)
    col = ops.DeviceColumn(k, A.FLOAT32)
    perm = ops.sort_indices(col, descending=True).long()
    assert int(perm.min()) >= 0 and int(perm.max()) < n  # checked before any indexing by perm
    assert torch.equal(torch.bincount(perm, minlength=n), torch.ones(n, dtype=torch.int64, device="cuda"))
    s = k[perm]
    assert bool((s[:-1] >= s[1:]).all())
    # stability: among equal keys the row ids ascend
    eq = s[:-1] == s[1:]
    assert bool((perm[:-1][eq] < perm[1:][eq]).all())


@pytest.mark.parametrize("width", [64, 256])
@pytest.mark.parametrize("desc", [False, True])
@pytest.mark.parametrize("with_nulls", [False, True])
def test_long_text_keys_sort_in_chunks(cuda, width, desc, with_nulls):
    """Text keys with more significant bytes than one pass carries (32, or 28
    with a NULL word) sort as a chain of 32-byte chunk keys: values that agree
    on their first 32..200 bytes still order by the bytes after them, NULLs
    keep their input order."""
    rng = np.random.default_rng(width + 2 * desc + with_nulls)
    n = 50_000
    prefix = "p" * (width - 24)
    words = [prefix[: int(rng.integers(0, len(prefix) + 1))] + "".join(rng.choice(list("abc"), 6))
             for _ in range(n)]
    words = [w[: width - 1] for w in words]
    k = datagen.text_slots(words, width)
    nulls = (rng.random(n) < 0.1) if with_nulls else None
    col = dev_col(k, A.TEXT, nulls)
    perm = ops.sort_indices(col, descending=desc).cpu().numpy()
    want = oracle.sort_perm(k, desc=desc, nulls=nulls)
    np.testing.assert_array_equal(perm.astype(np.int64), want.astype(np.int64))
