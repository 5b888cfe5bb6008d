"""One launch sequence of each hot operator on a moderate case, for ncu captures.

    python -m yallasql_b200.profile_cases filter   # 32M-row sales table: WHERE + aggregate, then WHERE + projection
    python -m yallasql_b200.profile_cases join     # 30M-row fact table joined to the 2,556-row date table + SUM
    python -m yallasql_b200.profile_cases order    # 16M rows (key f32, id, 16-byte txt, date), 116,480-row runs
    python -m yallasql_b200.profile_cases cross    # 20K x 20K cross product with < (198M output pairs)
    python -m yallasql_b200.profile_cases csv      # 4M-row sales table as CSV text (~205 MB): index + parse + write
    python -m yallasql_b200.profile_cases group    # 16M sales rows GROUP BY discount: COUNT(*), SUM, AVG, MIN, MAX

An optional second argument sets the row count (rows per side for cross).

The inputs are larger than L2 (so DRAM counters mean something) and hold a few
GB of device memory at most; every case runs its operators once and exits.
"""
from __future__ import annotations

import sys

import numpy as np
import torch

from . import _abi as A
from . import datagen, ops
from .expr import Aggregate, And, Arith, Cast, ColumnRef, Compare, Constant, between


def _dev(a, t):
    return ops.DeviceColumn(torch.from_numpy(np.ascontiguousarray(a)).cuda(), t)


def filter_case(rows: int = 32_000_000) -> None:
    t = datagen.sales_table(rows, seed=0)
    b = ops.DeviceBatch([_dev(t["price"], A.FLOAT32), _dev(t["qty"], A.INT32), _dev(t["discount"], A.INT32),
                         _dev(t["category"], A.TEXT)])
    price, qty, disc, cat = (ColumnRef(0, A.FLOAT32), ColumnRef(1, A.INT32), ColumnRef(2, A.INT32),
                             ColumnRef(3, A.TEXT))
    pred = And(between(disc, Constant(1, A.INT32), Constant(3, A.INT32)), Compare(A.LT, qty, Constant(25, A.INT32)),
               Compare(A.NE, cat, Constant(datagen.EXCLUDED_CATEGORY, A.TEXT)))
    aggs = [Aggregate(A.AGG_SUM, Arith(A.MUL, price, Cast(disc, A.FLOAT32))), Aggregate(A.AGG_COUNT_STAR),
            Aggregate(A.AGG_MIN, price), Aggregate(A.AGG_MAX, price)]
    plan = ops.AggPlan([A.FLOAT32, A.INT32, A.INT32, A.TEXT], pred, aggs)
    plan.run(b, ops.AggState(aggs))
    sel = [3, 0, Arith(A.MUL, price, Cast(disc, A.FLOAT32))]
    ops.ProjectPlan([A.FLOAT32, A.INT32, A.INT32, A.TEXT], [4, 4, 4, 16], pred, sel).run(b, with_nulls=False)
    torch.cuda.synchronize()


def join_case(rows: int = 30_000_000) -> None:
    fact, dim = datagen.star_tables(rows, seed=2)
    fb = ops.DeviceBatch([_dev(fact["datekey"], A.INT32), _dev(fact["quantity"], A.INT32),
                          _dev(fact["discount"], A.INT32), _dev(fact["extendedprice"], A.FLOAT32)])
    db = ops.DeviceBatch([_dev(dim["datekey"], A.INT32), _dev(dim["year"], A.INT32), _dev(dim["month"], A.INT32)])
    aggs = [Aggregate(A.AGG_SUM, Arith(A.MUL, ColumnRef(3, A.FLOAT32), Cast(ColumnRef(2, A.INT32), A.FLOAT32)))]
    jp = ops.JoinAggPlan([A.INT32] * 3 + [A.FLOAT32], [A.INT32] * 3,
                         And(between(ColumnRef(2, A.INT32), Constant(1, A.INT32), Constant(3, A.INT32)),
                             Compare(A.LT, ColumnRef(1, A.INT32), Constant(25, A.INT32))), 0,
                         Compare(A.EQ, ColumnRef(1, A.INT32), Constant(1993, A.INT32)), 0, aggs)
    jp.run(fb, db, ops.AggState(aggs))
    torch.cuda.synchronize()


def order_case(rows: int = 16_000_000, run_rows: int = 116_480) -> None:
    t = datagen.order_table(rows, seed=1, dist="uniform")
    b = ops.DeviceBatch([_dev(t["key"], A.FLOAT32), _dev(t["id"], A.INT64), _dev(t["txt"], A.TEXT),
                         _dev(t["d"], A.DATETIME)])
    offs = list(range(0, rows, run_rows)) + [rows]
    job = ops.OrderByRuns(b, 0, offs)
    out = ops.DeviceBatch([ops.DeviceColumn.empty(c.type, rows, c.width if c.type == A.TEXT else None)
                           for c in b.columns])
    job.run(b, True, out)
    torch.cuda.synchronize()


def cross_case(rows: int = 20_000) -> None:
    x, y = datagen.cross_tables(rows, seed=2)
    ops.join_project(ops.DeviceBatch([_dev(x, A.INT32)]), ops.DeviceBatch([_dev(y, A.INT32)]), [(0, 0, A.LT)],
                     [(0, 0), (1, 0)])
    torch.cuda.synchronize()


def csv_case(rows: int = 4_000_000) -> None:
    _, body = datagen.sales_csv(rows, seed=0)
    text = torch.from_numpy(body).cuda()
    batch = ops.csv_scan(text, [A.INT32, A.FLOAT32, A.INT32, A.INT32, A.TEXT, A.DATETIME], text_width=16)
    ops.csv_format(batch)  # and back to text (the writer's two kernels)
    torch.cuda.synchronize()


def group_case(rows: int = 16_000_000) -> None:
    t = datagen.sales_table(rows, seed=0)
    b = ops.DeviceBatch([_dev(t["discount"], A.INT32), _dev(t["price"], A.FLOAT32), _dev(t["qty"], A.INT32)])
    ops.group_by(b, 0, [(A.AGG_COUNT_STAR, 0), (A.AGG_SUM, 1), (A.AGG_AVG, 2), (A.AGG_MIN, 1), (A.AGG_MAX, 1)],
                 capacity=64)
    torch.cuda.synchronize()


CASES = {"filter": filter_case, "join": join_case, "order": order_case, "cross": cross_case, "csv": csv_case,
         "group": group_case}

if __name__ == "__main__":
    which = sys.argv[1] if len(sys.argv) > 1 else "filter"
    if which not in CASES:
        raise SystemExit(f"unknown case {which!r}; one of {sorted(CASES)}")
    if len(sys.argv) > 2:
        CASES[which](int(sys.argv[2]))
    else:
        CASES[which]()
    print("ok")
