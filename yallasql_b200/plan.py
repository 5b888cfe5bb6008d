"""ctypes binding of the C++ operator layer (``include/yq_engine.h``).

A ``Plan`` assembles the reference's operator tree (scan -> filter ->
projection / aggregate / order / join / cross product) over HOST columns and
executes it with ``libyq_engine.so``: batches stream to the device through
pinned double-buffered copies, every operator runs the kernels of
``libyq_ops.so``, and the result comes back to host memory.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _abi as A
from .expr import Aggregate, ConstPool, Compiled, Expr, compile_expr

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libyq_engine.so")


class HostColumn(C.Structure):
    _fields_ = [("data", C.c_void_p), ("nulls", C.c_void_p), ("type", C.c_int32), ("width", C.c_int32)]


class PlanStats(C.Structure):
    _fields_ = [("batches", C.c_uint64), ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64),
                ("compute_ms", C.c_double), ("spilled_batches", C.c_uint64),
                ("disk_batches", C.c_uint64)]


_lib = None

PROTOTYPES = {
    "yq_plan_create": (C.c_void_p, [C.c_uint64]),
    "yq_plan_destroy": (None, [C.c_void_p]),
    "yq_plan_set_spill": (C.c_int, [C.c_void_p, C.c_uint64, C.c_char_p]),
    "yq_plan_scan": (C.c_int, [C.c_void_p, C.POINTER(HostColumn), C.c_int32, C.c_uint64, C.c_uint32]),
    "yq_plan_scan_csv": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_int32), C.c_int32,
                                   C.POINTER(C.c_int32), C.c_int32, C.c_int32, C.c_uint32]),
    "yq_plan_filter": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(A.Program), C.POINTER(A.Constants)]),
    "yq_plan_project": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(A.Projection), C.c_int32,
                                  C.POINTER(A.Constants)]),
    "yq_plan_aggregate": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(A.AggSpec), C.c_int32,
                                    C.POINTER(A.Constants)]),
    "yq_plan_order": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "yq_plan_order_multi": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                      C.POINTER(C.c_int32), C.c_int32]),
    "yq_plan_group_by": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(A.GroupAgg), C.c_int32]),
    "yq_plan_join": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(A.JoinCond), C.c_int32]),
    "yq_plan_join_or": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(A.JoinCond), C.POINTER(C.c_int32),
                                  C.c_int32]),
    "yq_plan_cross": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "yq_plan_execute": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)]),
    "yq_result_rows": (C.c_uint64, [C.c_void_p]),
    "yq_result_ncols": (C.c_int32, [C.c_void_p]),
    "yq_result_column": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(HostColumn)]),
    "yq_result_destroy": (None, [C.c_void_p]),
    "yq_plan_stats_read": (C.c_int, [C.c_void_p, C.POINTER(PlanStats)]),
}


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libyq_engine.so not built at {LIB_PATH}")
        A.load()  # libyq_ops.so first (the engine links it by rpath)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


NP_TYPE = {np.dtype(np.int32): A.INT32, np.dtype(np.float32): A.FLOAT32, np.dtype(np.int64): A.INT64,
           np.dtype(np.float64): A.FLOAT64, np.dtype(np.uint8): A.BOOL}
NP_OF = {A.INT32: np.int32, A.FLOAT32: np.float32, A.INT64: np.int64, A.DATETIME: np.int64, A.FLOAT64: np.float64,
         A.BOOL: np.uint8}


def _node(st: int, what: str) -> int:
    if st < 0:
        raise A.YQError(-st, what, A.load())
    return st


class Plan:
    """One query: build nodes, then execute once."""

    def __init__(self, gpu_budget: int = 0, host_budget: int = 0, cache_dir: str | None = None):
        """gpu_budget: device bytes before batches spill to pinned host memory
        (0 = 1 GiB); host_budget with cache_dir: host bytes before spilled
        batches move on to files in cache_dir (0 = no file tier)."""
        self.h = lib().yq_plan_create(gpu_budget)
        if not self.h:
            raise A.YQError(A.ERR_CUDA, "yq_plan_create")
        if host_budget:
            st = lib().yq_plan_set_spill(self.h, host_budget, (cache_dir or "").encode())
            if st:
                raise A.YQError(st, "yq_plan_set_spill")
        self._keep = []
        self.types: dict[int, list[int]] = {}

    def __del__(self):
        if getattr(self, "h", None):
            lib().yq_plan_destroy(self.h)
            self.h = None

    def scan(self, cols: list, types: list[int] | None = None, nulls: list | None = None, batch_rows: int = 0):
        """Host columns: numpy arrays (text as uint8 [rows, width]) or pinned
        torch CPU tensors."""
        arr = (HostColumn * len(cols))()
        ts = []
        for i, c in enumerate(cols):
            if hasattr(c, "data_ptr"):  # torch tensor (pinned host memory)
                ptr, shape, esize = c.data_ptr(), tuple(c.shape), c.element_size()
                t = types[i]
                width = shape[1] if t == A.TEXT else esize
                rows = shape[0]
            else:
                c = np.ascontiguousarray(c)
                ptr, rows = c.ctypes.data, c.shape[0]
                t = types[i] if types else (A.TEXT if c.ndim == 2 else NP_TYPE[c.dtype])
                width = c.shape[1] if c.ndim == 2 else c.itemsize
            self._keep.append(c)
            nl = None
            if nulls is not None and nulls[i] is not None:
                nl = np.ascontiguousarray(nulls[i].astype(np.uint8))
                self._keep.append(nl)
            arr[i] = HostColumn(ptr, None if nl is None else nl.ctypes.data, t, width)
            ts.append(t)
        self._keep.append(arr)
        n = _node(lib().yq_plan_scan(self.h, arr, len(cols), rows, batch_rows), "yq_plan_scan")
        self.types[n] = ts
        return n

    def scan_csv(self, data: bytes, project: list[str] | None = None, text_width: int = 256, batch_rows: int = 0):
        """A CSV file (header line included) as the plan's table: schema from
        the header tags on the host, the body converted on the device batch by
        batch (GetOperator's place in the tree). Returns the node id; the
        output columns are the projected fields in `project` order."""
        from .ops import csv_schema
        if data.startswith(b"\xef\xbb\xbf"):
            data = data[3:]
        nl = data.find(b"\n")
        header = data[: nl if nl >= 0 else len(data)].decode("utf-8", "replace")
        body = data[nl + 1:] if nl >= 0 else b""
        nl2 = body.find(b"\n")
        schema = csv_schema(header, body[: nl2 if nl2 >= 0 else len(body)].decode("utf-8", "replace"))
        names = [c.name for c in schema]
        fields = list(range(len(schema))) if project is None else [names.index(p) for p in project]
        buf = np.frombuffer(body, dtype=np.uint8).copy() if body else np.zeros(1, np.uint8)
        types = (C.c_int32 * len(schema))(*[c.type for c in schema])
        proj = (C.c_int32 * len(fields))(*fields)
        self._keep += [buf, types, proj]
        n = _node(lib().yq_plan_scan_csv(self.h, buf.ctypes.data, len(body), types, len(schema), proj, len(fields),
                                         text_width, batch_rows), "yq_plan_scan_csv")
        self.types[n] = [schema[f].type for f in fields]
        return n

    def filter(self, child: int, pred: Expr):
        pool = ConstPool()
        prog = Compiled(compile_expr(pred, pool, self.types[child]))
        k, kk = pool.to_c()
        self._keep += [prog, k, kk]
        n = _node(lib().yq_plan_filter(self.h, child, C.byref(prog.prog), C.byref(k)), "yq_plan_filter")
        self.types[n] = self.types[child]
        return n

    def project(self, child: int, select: list):
        pool = ConstPool()
        proj = (A.Projection * len(select))()
        ts = []
        for i, s in enumerate(select):
            if isinstance(s, int):
                proj[i].column = s
                proj[i].out_type = self.types[child][s]
                ts.append(self.types[child][s])
            else:
                p = Compiled(compile_expr(s, pool, self.types[child]))
                self._keep.append(p)
                proj[i].column = -1
                proj[i].out_type = s.type
                proj[i].program = p.prog
                ts.append(s.type)
        k, kk = pool.to_c()
        self._keep += [proj, k, kk]
        n = _node(lib().yq_plan_project(self.h, child, proj, len(select), C.byref(k)), "yq_plan_project")
        self.types[n] = ts
        return n

    def aggregate(self, child: int, aggs: list[Aggregate]):
        pool = ConstPool()
        specs = (A.AggSpec * len(aggs))()
        for i, a in enumerate(aggs):
            p = Compiled(compile_expr(a.arg, pool, self.types[child]) if a.arg is not None else [])
            self._keep.append(p)
            specs[i].kind = a.kind
            specs[i].input_type = a.input_type
            specs[i].input = p.prog
        k, kk = pool.to_c()
        self._keep += [specs, k, kk]
        n = _node(lib().yq_plan_aggregate(self.h, child, specs, len(aggs), C.byref(k)), "yq_plan_aggregate")
        self.types[n] = []
        return n

    def order(self, child: int, key: int, descending=False, nulls_first=False):
        n = _node(lib().yq_plan_order(self.h, child, key, int(descending), int(nulls_first)), "yq_plan_order")
        self.types[n] = self.types[child]
        return n

    def order_multi(self, child: int, keys: list[int], descending: list[bool], nulls_first: list[bool] | None = None):
        """ORDER BY several keys, most significant first."""
        k = (C.c_int32 * len(keys))(*keys)
        d = (C.c_int32 * len(keys))(*[int(x) for x in descending])
        nf = (C.c_int32 * len(keys))(*[int(x) for x in (nulls_first or [False] * len(keys))])
        self._keep += [k, d, nf]
        n = _node(lib().yq_plan_order_multi(self.h, child, k, d, nf, len(keys)), "yq_plan_order_multi")
        self.types[n] = self.types[child]
        return n

    def group_by(self, child: int, key: int, aggs: list[tuple[int, int]]):
        """SELECT key, aggs GROUP BY key; aggs are (yq_agg_kind, input column)."""
        from .ops import group_by_out_type
        arr = (A.GroupAgg * max(1, len(aggs)))(*[A.GroupAgg(k, c) for k, c in aggs])
        self._keep.append(arr)
        n = _node(lib().yq_plan_group_by(self.h, child, key, arr, len(aggs)), "yq_plan_group_by")
        ct = self.types[child]
        self.types[n] = [ct[key]] + [group_by_out_type(k, A.INT64 if k == A.AGG_COUNT_STAR else ct[c]) for k, c in aggs]
        return n

    def join(self, left: int, right: int, conds: list, disjunct: list | None = None):
        """Inner join on conds [(left_col, right_col, cmp)], ANDed; with
        `disjunct` (a group per condition) an OR of the groups' ANDs."""
        arr = (A.JoinCond * len(conds))(*[A.JoinCond(l, r, c) for l, r, c in conds])
        self._keep.append(arr)
        if disjunct is None:
            n = _node(lib().yq_plan_join(self.h, left, right, arr, len(conds)), "yq_plan_join")
        else:
            dj = (C.c_int32 * len(conds))(*disjunct)
            self._keep.append(dj)
            n = _node(lib().yq_plan_join_or(self.h, left, right, arr, dj, len(conds)), "yq_plan_join_or")
        self.types[n] = self.types[left] + self.types[right]
        return n

    def cross(self, left: int, right: int):
        n = _node(lib().yq_plan_cross(self.h, left, right), "yq_plan_cross")
        self.types[n] = self.types[left] + self.types[right]
        return n

    def execute(self, root: int) -> list:
        """Returns [(values ndarray, nulls ndarray|None)] per result column (copies)."""
        res = C.c_void_p()
        A.check(lib().yq_plan_execute(self.h, root, C.byref(res)), "yq_plan_execute")
        try:
            rows = lib().yq_result_rows(res)
            out = []
            for c in range(lib().yq_result_ncols(res)):
                hc = HostColumn()
                A.check(lib().yq_result_column(res, c, C.byref(hc)), "yq_result_column")
                if hc.type == A.TEXT:
                    buf = (C.c_uint8 * (rows * hc.width)).from_address(hc.data)
                    v = np.frombuffer(buf, dtype=np.uint8).reshape(rows, hc.width).copy()
                else:
                    dt = np.dtype(NP_OF[hc.type])
                    buf = (C.c_uint8 * (rows * dt.itemsize)).from_address(hc.data) if rows else None
                    v = np.frombuffer(buf, dtype=dt).copy() if rows else np.zeros(0, dt)
                nl = None
                if hc.nulls:
                    nb = (C.c_uint8 * rows).from_address(hc.nulls) if rows else None
                    nl = np.frombuffer(nb, dtype=np.uint8).astype(bool) if rows else np.zeros(0, bool)
                out.append((v, nl))
            return out
        finally:
            lib().yq_result_destroy(res)

    def stats(self) -> PlanStats:
        s = PlanStats()
        A.check(lib().yq_plan_stats_read(self.h, C.byref(s)), "yq_plan_stats_read")
        return s
