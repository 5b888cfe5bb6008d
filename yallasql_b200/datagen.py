"""Seeded synthetic tables with the shapes and distributions of the
benchmark workloads (the reference's own data files are not available; its
generator `create_dataset.py` only fixes the header-tag CSV convention).

Every generator uses numpy's PCG64 with the stated seed, so the same call
returns the same table on any host. Text columns are fixed 16-byte NUL-padded
slots (uint8 [rows, 16]); dates are int64 epoch seconds (UTC).
"""
from __future__ import annotations

import calendar

import numpy as np

TEXT_WIDTH = 16
DATE_LO = calendar.timegm((2015, 1, 1, 0, 0, 0))
DATE_HI = calendar.timegm((2021, 12, 31, 0, 0, 0))
CATEGORIES = [f"category_{i:03d}" for i in range(25)]  # 25 fixed 12-character strings
EXCLUDED_CATEGORY = CATEGORIES[7]


def text_slots(strings: list[str], width: int = TEXT_WIDTH) -> np.ndarray:
    out = np.zeros((len(strings), width), dtype=np.uint8)
    for i, s in enumerate(strings):
        b = s.encode()[: width - 1]
        out[i, : len(b)] = np.frombuffer(b, dtype=np.uint8)
    return out


def sales_table(rows: int = 1_000_000, seed: int = 0) -> dict:
    """Filter + aggregate table: id, price, qty, discount, category, updated_at."""
    rng = np.random.Generator(np.random.PCG64(seed))
    price = rng.uniform(1.0, 1000.0, rows).astype(np.float32)
    price = np.minimum(price, np.float32(np.nextafter(np.float32(1000.0), np.float32(0))))
    cat_idx = rng.integers(0, len(CATEGORIES), rows)
    return {
        "id": np.arange(rows, dtype=np.int64),
        "price": price,
        "qty": rng.integers(1, 51, rows, dtype=np.int32),
        "discount": rng.integers(0, 11, rows, dtype=np.int32),
        "category": text_slots(CATEGORIES)[cat_idx],
        "category_idx": cat_idx.astype(np.int32),
        "updated_at": rng.integers(DATE_LO, DATE_HI + 1, rows, dtype=np.int64),
    }


def zipf_values(rng, rows: int, distinct: int = 100_000, s: float = 1.1) -> np.ndarray:
    """Bounded Zipf(s) over `distinct` values drawn uniformly from [-1e6, 1e6)."""
    values = rng.uniform(-1e6, 1e6, distinct).astype(np.float32)
    w = 1.0 / np.arange(1, distinct + 1, dtype=np.float64) ** s
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    ranks = np.searchsorted(cdf, rng.random(rows), side="right")
    return values[np.minimum(ranks, distinct - 1)]


def order_table(rows: int = 64_000_000, seed: int = 1, dist: str = "uniform") -> dict:
    """ORDER BY table: key f32 (uniform | zipf | equal), id int64, txt 16-byte, d date."""
    rng = np.random.Generator(np.random.PCG64(seed))
    if dist == "uniform":
        key = rng.uniform(-1e6, 1e6, rows).astype(np.float32)
    elif dist == "zipf":
        key = zipf_values(rng, rows)
    elif dist == "equal":
        key = np.full(rows, 42.0, dtype=np.float32)
    else:
        raise ValueError(dist)
    txt = np.zeros((rows, TEXT_WIDTH), dtype=np.uint8)
    txt[:, :15] = rng.integers(97, 123, (rows, 15), dtype=np.uint8)
    return {
        "key": key,
        "id": np.arange(rows, dtype=np.int64),
        "txt": txt,
        "d": rng.integers(DATE_LO, DATE_HI + 1, rows, dtype=np.int64),
    }


def star_tables(fact_rows: int = 60_000_000, seed: int = 2) -> tuple[dict, dict]:
    """Fact lineorder-like table and the 2,556-row date dimension."""
    rng = np.random.Generator(np.random.PCG64(seed))
    fact = {
        "orderkey": np.arange(fact_rows, dtype=np.int64),
        "custkey": rng.integers(0, 300_000, fact_rows, dtype=np.int32),
        "partkey": rng.integers(0, 200_000, fact_rows, dtype=np.int32),
        "suppkey": rng.integers(0, 20_000, fact_rows, dtype=np.int32),
        "datekey": rng.integers(0, 2556, fact_rows, dtype=np.int32),
        "quantity": rng.integers(1, 51, fact_rows, dtype=np.int32),
        "extendedprice": rng.uniform(900.0, 105000.0, fact_rows).astype(np.float32),
        "discount": rng.integers(0, 11, fact_rows, dtype=np.int32),
    }
    dk = np.arange(2556, dtype=np.int32)
    dim = {
        "datekey": dk,
        "year": np.minimum(1992 + dk // 365, 1998).astype(np.int32),
        "month": (1 + (dk % 365) * 12 // 365).astype(np.int32),
    }
    return fact, dim


def cross_tables(rows: int = 20_000, seed: int = 2) -> tuple[np.ndarray, np.ndarray]:
    """Two int32 columns a.x, b.y uniform in [0, 1e6) for the cross product."""
    rng = np.random.Generator(np.random.PCG64(seed + 1000))
    return (rng.integers(0, 1_000_000, rows, dtype=np.int32),
            rng.integers(0, 1_000_000, rows, dtype=np.int32))


def batch_row_counts(total_rows: int, row_bytes: int, batch_bytes: int = 4 << 20, align: int = 256) -> list[int]:
    """Rows per out-of-core batch: floor(batch_bytes / row_bytes) rounded down to
    a multiple of 256 (the reference's calculateOptimalBatchSize, include/config.hpp:28-36)."""
    per = max(align, (batch_bytes // row_bytes) // align * align)
    counts = [per] * (total_rows // per)
    if total_rows % per:
        counts.append(total_rows % per)
    return counts


# ---------------------------------------------------------------- CSV text
def _digits(x: np.ndarray, width: int) -> tuple[np.ndarray, np.ndarray]:
    """Right-aligned decimal digits of non-negative integers in a (rows, width)
    byte array, and a mask of the significant ones (no leading zeros; 0 is "0")."""
    x = x.astype(np.int64)
    pw = 10 ** np.arange(width - 1, -1, -1, dtype=np.int64)
    d = (x[:, None] // pw[None, :]) % 10
    ndig = np.maximum(1, np.floor(np.log10(np.maximum(x, 1))).astype(np.int64) + 1)
    mask = np.arange(width)[None, :] >= (width - ndig)[:, None]
    return (d + 48).astype(np.uint8), mask


def _fixed(rows: int, text: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    return text, np.ones(text.shape, dtype=bool)


def csv_text(columns: list[tuple[np.ndarray, np.ndarray]]) -> np.ndarray:
    """Rows of comma-separated fields, each line ending in '\n', from per-field
    (bytes [rows, w], mask [rows, w]) pieces: a field is its masked bytes."""
    rows = columns[0][0].shape[0]
    parts, masks = [], []
    for i, (b, m) in enumerate(columns):
        parts.append(b)
        masks.append(m)
        sep = np.full((rows, 1), ord(",") if i + 1 < len(columns) else ord("\n"), dtype=np.uint8)
        parts.append(sep)
        masks.append(np.ones((rows, 1), dtype=bool))
    full = np.concatenate(parts, axis=1)
    mask = np.concatenate(masks, axis=1)
    return full[mask]


SALES_CSV_HEADER = "id (N) (P),price (N),qty (N),discount (N),category (T),updated_at (D)\n"


def sales_csv(rows: int = 1_000_000, seed: int = 0) -> tuple[bytes, np.ndarray]:
    """The filter+aggregate table as a CSV file in the reference's header-tag
    convention: (header line, body bytes). Prices are written with two
    decimals (cents uniform over [1.00, 999.99]), dates as
    "YYYY-MM-DD HH:MM:SS" (UTC), categories as their 12-character names."""
    rng = np.random.Generator(np.random.PCG64(seed))
    cents = rng.integers(100, 100_000, rows)
    qty = rng.integers(1, 51, rows)
    disc = rng.integers(0, 11, rows)
    cat = rng.integers(0, len(CATEGORIES), rows)
    secs = rng.integers(DATE_LO, DATE_HI + 86400, rows)
    chunks = []
    step = 1 << 21
    for lo in range(0, rows, step):
        hi = min(rows, lo + step)
        n = hi - lo
        ident = _digits(np.arange(lo, hi), 10)
        pint = _digits(cents[lo:hi] // 100, 3)
        frac = (_digits(cents[lo:hi] % 100 + 100, 3)[0][:, 1:], np.ones((n, 2), dtype=bool))
        dot = np.full((n, 1), ord("."), dtype=np.uint8)
        price = (np.concatenate([pint[0], dot, frac[0]], axis=1),
                 np.concatenate([pint[1], np.ones((n, 1), dtype=bool), frac[1]], axis=1))
        catb = np.frombuffer("".join(CATEGORIES).encode(), dtype=np.uint8).reshape(len(CATEGORIES), 12)[cat[lo:hi]]
        chunks.append(csv_text([ident, price, _digits(qty[lo:hi], 2), _digits(disc[lo:hi], 2),
                                _fixed(n, catb), _fixed(n, _date_text(secs[lo:hi]))]))
    return SALES_CSV_HEADER.encode(), np.concatenate(chunks)


def _date_text(secs: np.ndarray) -> np.ndarray:
    """"YYYY-MM-DD HH:MM:SS" bytes [rows, 19] of epoch seconds (UTC)."""
    days, rem = np.divmod(secs.astype(np.int64), 86400)
    # civil date from days since 1970-01-01 (proleptic Gregorian)
    z = days + 719468
    era = np.floor_divide(z, 146097)
    doe = z - era * 146097
    yoe = (doe - doe // 1460 + doe // 36524 - doe // 146096) // 365
    y = yoe + era * 400
    doy = doe - (365 * yoe + yoe // 4 - yoe // 100)
    mp = (5 * doy + 2) // 153
    d = doy - (153 * mp + 2) // 5 + 1
    m = np.where(mp < 10, mp + 3, mp - 9)
    y = y + (m <= 2)
    hh, rem = np.divmod(rem, 3600)
    mi, ss = np.divmod(rem, 60)
    out = np.empty((secs.shape[0], 19), dtype=np.uint8)
    for col, (v, w) in zip([0, 5, 8, 11, 14, 17], [(y, 4), (m, 2), (d, 2), (hh, 2), (mi, 2), (ss, 2)]):
        pw = 10 ** np.arange(w - 1, -1, -1)
        out[:, col:col + w] = ((v[:, None] // pw[None, :]) % 10 + 48).astype(np.uint8)
    out[:, 4] = out[:, 7] = ord("-")
    out[:, 10] = ord(" ")
    out[:, 13] = out[:, 16] = ord(":")
    return out
