"""C-ABI boundary checks that need no GPU: the library loads, exports every
symbol the public headers declare, and rejects bad arguments before any
device work (the reference exits the process on errors instead,
include/utils/macros.hpp:6-22)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from yallasql_b200 import _abi as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header: str) -> list[str]:
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(yq_[a-z0-9_]+)\s*\(", text)))


def exported(lib_path: str) -> set[str]:
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], stdout=subprocess.PIPE, text=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_loads(yq):
    assert yq.yq_abi_version() == 1


def test_every_declared_symbol_is_exported(yq):
    names = declared_functions("yq_ops.h")
    assert len(names) > 30
    missing = sorted(set(names) - exported(A.LIB_PATH))
    assert not missing, f"declared in yq_ops.h but not exported: {missing}"


def test_engine_library_exports_its_header(yq):
    from yallasql_b200 import build, plan
    if not os.path.exists(plan.LIB_PATH):
        build.build_engine()
    names = declared_functions("yq_engine.h")
    assert len(names) >= 14
    missing = sorted(set(names) - exported(plan.LIB_PATH))
    assert not missing, f"declared in yq_engine.h but not exported: {missing}"
    assert set(names) <= set(plan.PROTOTYPES)
    plan.lib()  # loads (with libyq_ops.so) without touching a GPU


def test_prototypes_cover_header(yq):
    names = set(declared_functions("yq_ops.h"))
    assert names <= set(A.PROTOTYPES), sorted(names - set(A.PROTOTYPES))


def test_status_strings(yq):
    for s in range(7):
        assert yq.yq_status_string(s)
    assert yq.yq_status_string(A.ERR_CAPACITY) == b"output capacity exceeded"


def _batch(types_widths, rows=10):
    cols = (A.Column * len(types_widths))()
    for i, (t, w) in enumerate(types_widths):
        cols[i] = A.Column(0x1000 * (i + 1), None, t, w)  # never dereferenced: validation fails first
    return A.Batch(cols, len(types_widths), rows), cols


def _prog(insns):
    arr = (A.Insn * len(insns))(*[A.Insn(*i) for i in insns])
    return A.Program(arr, len(insns)), arr


@pytest.mark.parametrize("insns", [
    [(A.OP_AND, 0, 0, 0, 0)],                                   # stack underflow
    [(A.OP_COL, A.INT32, 5, 0, 0)],                             # column out of range
    [(A.OP_COL, A.INT32, 0, 0, 0), (A.OP_COL, A.FLOAT32, 1, 0, 0),
     (A.OP_ARITH, A.INT32, A.ADD, 0, 0)],                       # operand types differ
    [(A.OP_COL, A.INT32, 0, 0, 0)],                             # predicate is not BOOL
    [(A.OP_CMP_COL_CONST, A.INT32, A.LT, 0, 9)],                # constant out of range
    [(A.OP_COL, A.INT32, 0, 0, 0)] * 5,                         # deeper than the register stack
    [(99, 0, 0, 0, 0)],                                         # unknown opcode
])
def test_bad_programs_rejected_before_launch(yq, insns):
    b, keep = _batch([(A.INT32, 4), (A.FLOAT32, 4)])
    p, pk = _prog(insns)
    st = yq.yq_filter_project(C.byref(b), C.byref(p), None, None, 0, None, 0, None, None, None, 0, None)
    assert st in (A.ERR_INVALID_ARG, A.ERR_UNSUPPORTED)


@pytest.mark.parametrize("tw", [(A.INT32, 8), (A.FLOAT64, 4), (A.TEXT, 6), (A.TEXT, 512), (9, 4)])
def test_bad_columns_rejected(yq, tw):
    b, keep = _batch([tw])
    p, pk = _prog([(A.OP_CONST, A.BOOL, 0, 0, 0)])
    st = yq.yq_filter_project(C.byref(b), C.byref(p), None, None, 0, None, 0, None, None, None, 0, None)
    assert st == A.ERR_INVALID_ARG


def test_bad_sort_arguments(yq):
    col = A.Column(0x1000, None, A.FLOAT32, 4)
    cfg = A.SortConfig(5, 0, 0, 0)  # digit width must be 4, 6 or 8
    assert yq.yq_sort_indices(C.byref(col), 10, 0, 0, 0x2000, C.byref(cfg), None, 0, None) == A.ERR_INVALID_ARG
    bad = A.Column(0x1000, None, A.TEXT, 7)
    assert yq.yq_sort_indices(C.byref(bad), 10, 0, 0, 0x2000, None, None, 0, None) == A.ERR_INVALID_ARG
    assert yq.yq_sort_indices(None, 10, 0, 0, 0x2000, None, None, 0, None) == A.ERR_INVALID_ARG
    assert yq.yq_sort_indices(C.byref(col), 1 << 30, 0, 0, 0x2000, None, None, 0, None) == A.ERR_UNSUPPORTED


def test_workspace_sizes_are_host_only(yq):
    assert yq.yq_filter_project_workspace_size(1_000_000) > 977 * 8
    col = A.Column(0x1000, None, A.FLOAT32, 4)
    assert yq.yq_sort_workspace_size(C.byref(col), 1_000_000) >= 4 * 1_000_000 * 5
    assert yq.yq_agg_state_bytes(4) >= 4 * 24


def test_bad_or_join_arguments(yq):
    """OR-of-AND join conditions: groups numbered 0..G-1 with every group
    used; rejected before any device work otherwise."""
    lb, lk = _batch([(A.INT32, 4), (A.INT32, 4)])
    rb, rk = _batch([(A.INT32, 4), (A.INT32, 4)])
    conds = (A.JoinCond * 2)(A.JoinCond(0, 0, A.EQ), A.JoinCond(1, 1, A.LT))
    cnt = C.c_uint64()
    for groups in ([0, 2], [1, 1], [0, 9], [-1, 0]):
        g = (C.c_int32 * 2)(*groups)
        st = yq.yq_join_pairs_or(C.byref(lb), C.byref(rb), conds, C.cast(g, C.c_void_p), 2, 0x3000, 0x4000, 100,
                                 C.byref(cnt), None, 0, None)
        assert st == A.ERR_INVALID_ARG, groups
    assert yq.yq_join_pairs_or(C.byref(lb), C.byref(rb), conds, None, 2, 0x3000, 0x4000, 100, C.byref(cnt), None, 0,
                               None) == A.ERR_INVALID_ARG
    g = (C.c_int32 * 2)(0, 1)
    assert yq.yq_join_pairs_or(C.byref(lb), C.byref(rb), conds, C.cast(g, C.c_void_p), 0, 0x3000, 0x4000, 100,
                               C.byref(cnt), None, 0, None) == A.ERR_INVALID_ARG


def test_bad_tuning_arguments(yq):
    col = A.Column(0x1000, None, A.FLOAT32, 4)
    for block in (96, 1024, -1):
        cfg = A.SortConfig(8, 0, block, 0)
        assert yq.yq_sort_indices(C.byref(col), 10, 0, 0, 0x2000, C.byref(cfg), None, 0, None) == A.ERR_INVALID_ARG
    b, keep = _batch([(A.FLOAT32, 4), (A.INT64, 8)])
    offs = (C.c_uint32 * 3)(0, 5, 10)
    for items in (3, 12, 32):
        assert yq.yq_order_by_tiled(C.byref(b), 0, 0, 0, offs, 2, C.byref(b), items, None, 0, None) == \
            A.ERR_INVALID_ARG


def test_join_workspace_covers_counting(yq):
    """With a right side long enough for the up-front match counts, the join
    workspace also holds the right key's sort and one count per left row."""
    small = yq.yq_join_workspace_size(50_000, 1_000)
    big = yq.yq_join_workspace_size(50_000, 100_000)
    assert big >= small + 4 * 50_000 + 12 * 100_000
