"""CSV scan on the CPU: the device code's tokenizer and conversions
(yallasql_b200/csrc/yq_csv.cuh, compiled for the host by g++) against glibc's
strtol/strtof/strptime/timegm (the calls behind the reference's std::stoi,
std::stof and getDateTime), the oracle against the reference's own csv-parser
reader (oracle/_ref/libcsvref.so) and against golden fixtures it wrote."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import oracle
from tests import csv_cases

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "csv_ref.npz")


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("csvshim") / "libcsvshim.so")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-o", out,
                           os.path.join(HERE, "csv_host_shim.cpp")])
    L = C.CDLL(out)
    L.hs_csv_scan.restype = C.c_int64
    L.hs_record_starts.restype = C.c_int64
    return L


def shim_convert(L, kind, strings):
    buf = b"".join(strings)
    offs = np.zeros(len(strings) + 1, np.uint64)
    offs[1:] = np.cumsum([len(s) for s in strings])
    out = np.zeros(len(strings), np.int64)
    st = np.zeros(len(strings), np.int32)
    L.hs_convert(C.c_int(kind), C.c_char_p(buf), offs.ctypes.data_as(C.c_void_p), C.c_uint64(len(strings)),
                 out.ctypes.data_as(C.c_void_p), st.ctypes.data_as(C.c_void_p))
    return out, st


def shim_scan(L, body, types, width=16):
    n = len(types)
    cap = body.count(b"\n") + body.count(b"\r") + 2
    datas, nulls = oracle._csv_outputs(types, width, cap)
    dp = (C.c_void_p * n)(*[d.ctypes.data for d in datas])
    npp = (C.c_void_p * n)(*[x.ctypes.data for x in nulls])
    ty = (C.c_int * n)(*types)
    wd = (C.c_int * n)(*[width if t == 3 else 0 for t in types])
    bad, fr, ff, fk = C.c_uint64(), C.c_int64(), C.c_int(), C.c_int()
    rows = L.hs_csv_scan(C.c_char_p(body), C.c_uint64(len(body)), n, ty, wd, dp, npp, C.c_uint64(cap),
                         C.byref(bad), C.byref(fr), C.byref(ff), C.byref(fk))
    assert rows >= 0, "record splitting: chunk summaries disagree with the plain state machine"
    return oracle._csv_result(rows, bad.value, fr.value, ff.value, fk.value, types, width, datas, nulls)


def same_scan(a, b):
    assert (a["rows"], a["bad"], a["first_row"], a["first_field"], a["first_kind"]) == \
        (b["rows"], b["bad"], b["first_row"], b["first_field"], b["first_kind"])
    for x, y in zip(a["cols"], b["cols"]):
        assert (x is None) == (y is None)
        if x is not None:
            assert np.array_equal(x[1], y[1])
            assert x[0].tobytes() == y[0].tobytes()  # bit-exact (floats, NaN payloads, text slots)


def float_strings(rng, n):
    from decimal import Decimal
    bits = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    f = bits.view(np.float32)
    out = [("%.9g" % x).encode() for x in f[: n // 2]] + [("%.6g" % x).encode() for x in f[n // 2:]]
    # exact midpoints between neighbouring floats and values just beside them
    for b in rng.integers(0, 0x7f7fffff, n // 20):
        lo, hi = Decimal(float(np.uint32(b).view(np.float32))), Decimal(float(np.uint32(b + 1).view(np.float32)))
        m = (lo + hi) / 2
        eps = Decimal(10) ** (m.adjusted() - 40)
        out += [format(m, "e").encode(), format(m + eps, "e").encode(), format(m - eps, "e").encode()]
    for e in range(-50, -34):
        out += [f"{m}e{e}".encode() for m in ("1", "1.4", "7.006", "1.17549435", "1.1754943", "5.877")]
    out += [s.encode() for s in ["3.4028235e38", "3.40282356e38", "3.40282357e38", "1e39", "0", "-0", ".5", ".",
                                 "+", "1e", "1e+", " \t12.5", "0x1p-149", "0x1.8p-149", "0x", "inf", "-Infinity",
                                 "nan", "-nan(5)", "nan(0x7fffff)", "nan(abc)", "1.5f", "9" * 120, '"12"']]
    alpha = list(b"0123456789.eE+- xXpPaAfFiInN()\t")
    out += [bytes(rng.choice(alpha, int(rng.integers(0, 12)))) for _ in range(n // 4)]
    return out


def test_float_conversion_matches_strtof(shim):
    s = float_strings(np.random.default_rng(11), 20000)
    a, sa = shim_convert(shim, 1, s)
    b, sb = oracle.convert_batch(1, s)
    bad = np.nonzero((a != b) | (sa != sb))[0]
    assert bad.size == 0, [(s[i], hex(a[i]), sa[i], hex(b[i]), sb[i]) for i in bad[:5]]


def test_int_conversion_matches_stoi(shim):
    rng = np.random.default_rng(12)
    s = [str(int(x)).encode() for x in rng.integers(-2**31, 2**31, 5000)]
    s += [x.encode() for x in ["2147483647", "2147483648", "-2147483648", "-2147483649", "9" * 25, " +7", "-", "",
                               "12abc", "\t\n3", "0x10", "1e3", "--1"]]
    s += [bytes(rng.choice(list(b"0123456789+- \tx"), int(rng.integers(0, 12)))) for _ in range(5000)]
    a, sa = shim_convert(shim, 0, s)
    b, sb = oracle.convert_batch(0, s)
    assert np.array_equal(sa, sb) and np.array_equal(a, b)


def test_datetime_conversion_matches_strptime_timegm(shim):
    rng = np.random.default_rng(13)
    s = []
    for _ in range(4000):
        y, mo, d, h, mi, se = (int(rng.integers(0, 10000)), int(rng.integers(1, 13)), int(rng.integers(1, 32)),
                               int(rng.integers(0, 24)), int(rng.integers(0, 60)), int(rng.integers(0, 62)))
        s += [f"{y:04d}-{mo:02d}-{d:02d} {h:02d}:{mi:02d}:{se:02d}".encode(), f"{y}-{mo}-{d} {h}:{mi}:{se}".encode()]
    alpha = list(b"0123456789-: \t\x0bx")
    for _ in range(8000):
        b = bytearray(s[int(rng.integers(0, len(s)))])
        for __ in range(int(rng.integers(1, 4))):
            p = int(rng.integers(0, len(b) + 1))
            op = int(rng.integers(0, 3))
            if op == 0 and b:
                del b[min(p, len(b) - 1)]
            elif op == 1:
                b.insert(p, int(rng.choice(alpha)))
            elif b:
                b[min(p, len(b) - 1)] = int(rng.choice(alpha))
        s.append(bytes(b))
    a, _ = shim_convert(shim, 2, s)
    b, _ = oracle.convert_batch(2, s)
    assert np.array_equal(a, b)


def quote_free_cases(rng):
    """Long quote-free texts (most 64-byte chunks take the kernels' newline-
    bitmask shortcut): the sales table, and CR/LF runs of every length at
    every offset across chunk boundaries."""
    from yallasql_b200 import datagen
    _, sales = datagen.sales_csv(3000, seed=3)
    out = [([0, 1, 0, 0, 3, 2], b"", sales.tobytes())]
    for _ in range(20):
        parts = []
        for _ in range(int(rng.integers(20, 200))):
            parts.append(",".join(str(int(x)) for x in rng.integers(0, 10**int(rng.integers(1, 9)), 2)))
            parts.append("".join(rng.choice(["\n", "\r", "\r\n", "\n\n"], int(rng.integers(1, 4)))))
        out.append(([0, 0], b"", "".join(parts).encode()))
    return out


def test_device_scan_semantics_match_oracle(shim):
    rng = np.random.default_rng(14)
    cases = csv_cases.edge_cases() + [csv_cases.random_csv(rng) for _ in range(300)] + quote_free_cases(rng)
    for types, header, body in cases:
        same_scan(shim_scan(shim, body, types), oracle.csv_scan(body, types))


@pytest.mark.skipif(not oracle.ref_csv_available(), reason="reference CSV reader not built (oracle/_ref)")
def test_oracle_matches_reference_reader():
    rng = np.random.default_rng(15)
    cases = csv_cases.edge_cases() + [csv_cases.random_csv(rng) for _ in range(200)]
    for types, header, body in cases:
        same_scan(oracle.csv_scan(body, types), oracle.ref_csv_scan(header, body, types))


@pytest.mark.skipif(not oracle.ref_csv_available(), reason="reference CSV reader not built (oracle/_ref)")
def test_sales_csv_with_the_references_format_guess():
    from yallasql_b200 import datagen
    header, body = datagen.sales_csv(5000, seed=0)
    types = [0, 1, 0, 0, 3, 2]
    same_scan(oracle.csv_scan(body.tobytes(), types), oracle.ref_csv_scan(header, body.tobytes(), types, guess=True))


def test_oracle_matches_golden():
    g = np.load(GOLDEN, allow_pickle=False)
    for i in range(int(g["count"])):
        body = g[f"body{i}"].tobytes()
        types = [int(t) for t in g[f"types{i}"]]
        got = oracle.csv_scan(body, types)
        meta = g[f"meta{i}"]
        assert (got["rows"], got["bad"], got["first_row"], got["first_field"], got["first_kind"]) == tuple(meta)
        for f, t in enumerate(types):
            if t < 0:
                continue
            assert got["cols"][f][0].tobytes() == g[f"vals{i}_{f}"].tobytes()
            assert np.array_equal(got["cols"][f][1], g[f"nulls{i}_{f}"])


def test_schema_follows_header_tags():
    from yallasql_b200 import _abi as A
    from yallasql_b200 import ops
    s = ops.csv_schema('id (N) (P),"price (N)",qty (N),d (D),t (T),plain\r', "1,2.5,3,2020-01-01 00:00:00,x,y")
    assert [(c.name, c.type, c.pk) for c in s] == [("id", A.INT32, True), ("price", A.FLOAT32, False),
                                                   ("qty", A.INT32, False), ("d", A.DATETIME, False),
                                                   ("t", A.TEXT, False), ("plain", A.TEXT, False)]
    with pytest.raises(ValueError):
        ops.csv_schema(" (N)", "1")


def test_writer_cells_match_the_reference_routines(shim):
    """Cell text of the device writer (host build) against the oracle's
    snprintf / gmtime_r + strftime, and the oracle's "%.4f" against
    std::to_chars(fixed, 4), the reference writer's own float routine."""
    rng = np.random.default_rng(16)

    def shim_cells(kind, vals):
        vals = np.asarray(vals, dtype=np.int64)
        out = C.create_string_buffer(64 * len(vals))
        ln = np.zeros(len(vals), np.int32)
        shim.hs_format(C.c_int(kind), vals.ctypes.data_as(C.c_void_p), C.c_uint64(len(vals)), out,
                       ln.ctypes.data_as(C.c_void_p))
        assert (ln >= 0).all(), "counting and writing passes disagree"
        return [out.raw[i * 64:i * 64 + ln[i]] for i in range(len(vals))]

    def oracle_cells(kind, vals, dtype):
        arr = np.asarray(vals).astype(dtype)
        text = oracle.csv_format([(kind, 0, arr, None)], len(arr))
        return text.split(b"\n")[:-1]

    bits = [int(b) for b in rng.integers(0, 2**32, 20000, dtype=np.uint64)]
    bits += [int(x) for x in (rng.integers(100, 100000, 5000) / 100.0).astype(np.float32).view(np.uint32)]
    bits += [int(np.float32(m / 2.0**k).view(np.uint32)) for k in range(1, 40) for m in (1, 3, 5, 7)]  # ties
    bits += [0, 0x80000000, 1, 0x7f7fffff, 0xff7fffff, 0x7f800000, 0xff800000, 0x7fc00000, 0xffc00000]
    assert shim_cells(1, bits) == oracle_cells(1, bits, np.uint32)
    shim.hs_to_chars_fixed4.restype = C.c_int32
    buf = C.create_string_buffer(64)
    want = oracle_cells(1, bits[:3000], np.uint32)
    for b, w in zip(bits[:3000], want):
        n = shim.hs_to_chars_fixed4(C.c_uint32(b), buf)
        assert buf.raw[:n] == w
    ints = [int(x) for x in rng.integers(-2**31, 2**31, 5000)] + [-2**31, 2**31 - 1, 0]
    assert shim_cells(0, ints) == oracle_cells(0, ints, np.int32)
    big = [int(x) for x in rng.integers(-2**63, 2**63 - 1, 5000, dtype=np.int64)] + [-2**63, 2**63 - 1]
    assert shim_cells(4, big) == oracle_cells(4, big, np.int64)
    secs = [int(x) for x in rng.integers(-62167219200 - 86400 * 366 * 50, 253402300800 + 86400 * 366 * 50, 5000)]
    secs += [int(x) for x in rng.integers(-2**40, 2**40, 2000)] + [0, -1, -62167219200, -62167219201, 253402300800]
    assert shim_cells(2, secs) == oracle_cells(2, secs, np.int64)


def test_generated_csv_matches_python_formatting():
    """The benchmark CSV generator's vectorised fields (variable-width ids and
    prices, "YYYY-MM-DD HH:MM:SS" dates) against Python's own formatting of
    the same values."""
    import datetime

    from yallasql_b200 import datagen
    rng = np.random.default_rng(17)
    secs = np.concatenate([rng.integers(-2_000_000_000, 4_000_000_000, 5000), [0, -1, 86399, 951782400]])
    got = datagen._date_text(secs)
    epoch = datetime.datetime(1970, 1, 1)
    for s, row in zip(secs, got):
        want = (epoch + datetime.timedelta(seconds=int(s))).strftime("%Y-%m-%d %H:%M:%S")
        assert bytes(row).decode() == want
    header, body = datagen.sales_csv(2000, seed=3)
    lines = bytes(body).decode().splitlines()
    assert len(lines) == 2000 and header.decode().count(",") == 5
    for i, line in enumerate(lines):
        f = line.split(",")
        assert int(f[0]) == i and len(f) == 6
        assert f[1] == f"{float(f[1]):.2f}" and 1.0 <= float(f[1]) < 1000.0
        assert 1 <= int(f[2]) <= 50 and 0 <= int(f[3]) <= 10 and f[4] in datagen.CATEGORIES
