"""Seeded CSV texts for the CSV scan tests: random tables with quoting,
escaped quotes, embedded delimiters/newlines, CRLF/CR line ends, blank lines,
empty (NULL) cells, ragged rows and cells the reference's conversions reject."""
from __future__ import annotations

import numpy as np

TYPE_CODES = [0, 1, 2, 3]  # INT, FLOAT, DATETIME, STRING (the reference's DataType order)


def _field(t: int, rng) -> str:
    k = rng.random()
    if k < 0.08:
        return ""
    if t == 0:
        v = str(int(rng.integers(-3000, 3000))) if k < 0.9 else str(rng.choice(
            ["abc", " 12", "99999999999", "+5", "-", "2147483648", "-2147483648", "7x"]))
    elif t == 1:
        v = ("%.4f" % rng.uniform(-1000, 1000)) if k < 0.85 else str(rng.choice(
            ["1e-40", "3e38", "x", ".5", " 2.5e3", "inf", "nan", "1e39", "0x1p3", "-0", "1.17549435e-38"]))
    elif t == 2:
        v = "%04d-%02d-%02d %02d:%02d:%02d" % (rng.integers(1990, 2030), rng.integers(1, 13), rng.integers(1, 32),
                                              rng.integers(0, 24), rng.integers(0, 60), rng.integers(0, 62))
        if k > 0.9:
            v = v[: int(rng.integers(0, len(v)))]
    else:
        v = "".join(rng.choice(list('abcdefgh xyz,"\n\r'), int(rng.integers(0, 22))))
    if any(c in v for c in '",\n\r') or rng.random() < 0.1:
        if rng.random() < 0.9:
            v = '"' + v.replace('"', '""') + '"'
    return v


def random_csv(rng, max_rows: int = 60) -> tuple[list[int], bytes, bytes]:
    """(field types with -1 for skipped fields, header line, body)."""
    nf = int(rng.integers(1, 7))
    types = [int(rng.choice(TYPE_CODES)) for _ in range(nf)]
    gen_types = list(types)
    if nf > 1 and rng.random() < 0.3:
        types[int(rng.integers(0, nf))] = -1
    header = (",".join(f"c{i}" for i in range(nf)) + "\n").encode()
    lines = []
    for _ in range(int(rng.integers(0, max_rows))):
        f = nf if rng.random() > 0.05 else int(rng.integers(1, nf + 2))
        lines.append(",".join(_field(gen_types[i % nf], rng) for i in range(f)))
    seps = []
    for _ in lines:
        x = rng.random()
        seps.append("\r\n" if x < 0.1 else "\n\n" if x < 0.15 else "\r" if x < 0.18 else "\n")
    body = "".join(l + s for l, s in zip(lines, seps))
    if body and rng.random() < 0.3:
        body = body.rstrip("\r\n")
    return types, header, body.encode()


def edge_cases() -> list[tuple[list[int], bytes, bytes]]:
    h1 = b"a\n"
    h3 = b"a,b,c\n"
    return [
        ([0], h1, b""),                                   # no rows
        ([0], h1, b"\n\n\r\n"),                           # only blank lines
        ([3], h1, b'"ab"'),                               # quoted field closed at the end of the text
        ([3], h1, b'"a,b\nc"'),                           # delimiter and newline inside quotes
        ([3], h1, b'"a""b"\n"x"y"z"\n"p""q"r"s"\n'),      # escaped and lone quotes
        ([3], h1, b'"unterminated\n,more'),               # quote never closed
        ([0, 1, 2], h3, b"1,2.5,2020-01-01 00:00:00\n,,\n3,abc,bad\n"),
        ([0, 1, 2], h3, b"1,2\n1,2,2020-01-01 00:00:00,4\n5,6.5,2021-02-03 04:05:06"),  # ragged rows dropped
        ([0, -1, 3], h3, b"7,skip,text\r\n8,skip,\r\n"),
        ([1], h1, b"1e-40\n3.4028236e38\n1.4e-45\n0x1p-149\nnan(5)\n-inf\n"),
        ([0], h1, b" 12\n+7\n-2147483648\n2147483648\n12abc\nabc\n"),
        ([3], h1, b"x" * 300 + b"\n" + b"\x00abc\n" + b"ab\x00cd\n"),  # long text, embedded NULs
    ]
