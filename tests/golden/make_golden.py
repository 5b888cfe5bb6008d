"""Writes the golden fixtures of this directory from the reference's OWN
kernels: its src/kernels/*.cu, compiled where they lie in the reference tree
into oracle/_ref/libyqref.so by `make -C oracle ref` (needs a GPU to run).
Inputs are small and seeded; every fixture stores its inputs and the
reference's outputs, and tests/test_golden_cpu.py checks the oracle against
them on the CPU.

    python tests/golden/make_golden.py [--out DIR]
"""
import argparse
import ctypes as C
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from yallasql_b200 import datagen  # noqa: E402

REF_LIB = os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle", "_ref", "libyqref.so")


def d(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    L = C.CDLL(REF_LIB)
    vp, u32, i32 = C.c_void_p, C.c_uint32, C.c_int
    L.ref_reduce.argtypes = [vp, vp, u32, i32, vp]
    L.ref_merge_f32.argtypes = [vp, vp, u32, u32, u32, i32, vp, vp, vp, vp]
    L.ref_join_eq_i32.argtypes = [vp, u32, vp, u32, vp, vp]
    L.ref_cross_col_i32.argtypes = [vp, vp, u32, u32, i32, vp, vp]
    L.ref_mul_cast_f32.argtypes = [vp, vp, u32, vp]

    # reductions: SUM/MIN/MAX of float32, SUM/MIN/MAX/COUNT of int32, with null bytes
    rng = np.random.default_rng(101)
    n = 4096
    f = rng.normal(0, 100, n).astype(np.float32)
    i = rng.integers(-1000, 1000, n).astype(np.int32)
    nulls = (rng.random(n) < 0.1).astype(np.uint8)
    df, di, dn = d(f), d(i), d(nulls)
    res = []
    for kind, x in ((0, df), (1, df), (2, df), (3, di), (4, di), (5, di), (6, di)):
        buf = (C.c_double if kind == 0 else (C.c_float if kind in (1, 2) else C.c_int))()
        assert L.ref_reduce(x.data_ptr(), dn.data_ptr(), n, kind, C.addressof(buf)) == 0
        res.append(float(buf.value))
    np.savez(os.path.join(args.out, "reduce.npz"), f=f, i=i, nulls=nulls, out=np.array(res))

    # merge path of two sorted float runs with many ties (ascending and descending)
    for desc in (0, 1):
        rng = np.random.default_rng(200 + desc)
        a = np.sort(datagen.zipf_values(rng, 700, distinct=40))
        b = np.sort(datagen.zipf_values(rng, 500, distinct=40))
        if desc:
            a, b = a[::-1].copy(), b[::-1].copy()
        k = 900
        c_ = torch.empty(k, dtype=torch.float32, device="cuda")
        idx = torch.empty(k, dtype=torch.int32, device="cuda")
        fa = torch.empty(k, dtype=torch.uint8, device="cuda")
        last = torch.zeros(1, dtype=torch.int32, device="cuda")
        da, db = d(a), d(b)
        assert L.ref_merge_f32(da.data_ptr(), db.data_ptr(), len(a), len(b), k, desc, c_.data_ptr(), idx.data_ptr(),
                               fa.data_ptr(), last.data_ptr()) == 0
        np.savez(os.path.join(args.out, f"merge_{'desc' if desc else 'asc'}.npz"), a=a, b=b, k=k,
                 merged=c_.cpu().numpy(), from_a=fa.cpu().numpy(), last=last.item())

    # equi-join pairs of two int32 columns
    rng = np.random.default_rng(300)
    left = rng.integers(0, 60, 300).astype(np.int32)
    right = rng.integers(0, 60, 120).astype(np.int32)
    pairs = torch.empty(2 * 20_000, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    dl, dr = d(left), d(right)
    assert L.ref_join_eq_i32(dl.data_ptr(), 300, dr.data_ptr(), 120, pairs.data_ptr(), cnt.data_ptr()) == 0
    m = cnt.item()
    p = pairs[: 2 * m].cpu().numpy().view(np.uint32).reshape(m, 2)
    p = p[np.lexsort((p[:, 1], p[:, 0]))]
    np.savez(os.path.join(args.out, "join_eq.npz"), left=left, right=right, pairs=p)

    # price * CAST(discount AS FLOAT)
    t = datagen.sales_table(2000, seed=301)
    out = torch.empty(2000, dtype=torch.float32, device="cuda")
    dp, dd = d(t["price"]), d(t["discount"])
    assert L.ref_mul_cast_f32(dp.data_ptr(), dd.data_ptr(), 2000, out.data_ptr()) == 0
    np.savez(os.path.join(args.out, "mul_cast.npz"), price=t["price"], discount=t["discount"], out=out.cpu().numpy())
    print("golden fixtures written to", args.out)


if __name__ == "__main__":
    main()
