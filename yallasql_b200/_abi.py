"""ctypes declarations for the C ABI in ``include/yq_ops.h``.

The shared library is the in-tree ``libyq_ops.so``; importing this module
never falls back to anything else: a missing library is an ImportError.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libyq_ops.so")

# yq_status
OK, ERR_INVALID_ARG, ERR_UNSUPPORTED, ERR_CAPACITY, ERR_TIMEOUT, ERR_CUDA, ERR_ALLOC = range(7)

# yq_type (0..3 equal the reference's DataType)
INT32, FLOAT32, DATETIME, TEXT, INT64, FLOAT64, BOOL = range(7)
TYPE_NAMES = {INT32: "int32", FLOAT32: "float32", DATETIME: "datetime", TEXT: "text", INT64: "int64",
              FLOAT64: "float64", BOOL: "bool"}
# yq_cmp
LT, LE, GT, GE, EQ, NE = range(6)
# yq_arith
ADD, SUB, MUL, DIV, MOD = range(5)
# yq_opcode
OP_COL, OP_CONST, OP_NULL, OP_CAST, OP_ARITH, OP_CMP, OP_CMP_COL_CONST, OP_CMP_COL_COL = range(1, 9)
OP_AND, OP_OR, OP_NOT, OP_IS_NULL, OP_IS_NOT_NULL = range(9, 14)
OP_ARITH_COL, OP_ARITH_CONST, OP_AND_CMP_COL_CONST = 20, 21, 22
# yq_agg_kind
AGG_COUNT_STAR, AGG_COUNT, AGG_SUM, AGG_AVG, AGG_MIN, AGG_MAX = range(6)

MAX_PROGRAM_INSNS = 48
MAX_BATCH_COLUMNS = 16
MAX_CONSTANTS = 32
MAX_TEXT_CONSTANTS = 4
MAX_TEXT_WIDTH = 256
MAX_AGGREGATES = 8
MAX_PROJECTIONS = 12


class Column(C.Structure):
    _fields_ = [("data", C.c_void_p), ("nulls", C.c_void_p), ("type", C.c_int32), ("width", C.c_int32)]


class Batch(C.Structure):
    _fields_ = [("columns", C.POINTER(Column)), ("ncols", C.c_int32), ("rows", C.c_uint32)]


class Insn(C.Structure):
    _fields_ = [("op", C.c_uint8), ("type", C.c_uint8), ("a", C.c_uint8), ("b", C.c_uint8), ("imm", C.c_int32)]


class Program(C.Structure):
    _fields_ = [("code", C.POINTER(Insn)), ("len", C.c_int32)]


class Constants(C.Structure):
    _fields_ = [("values", C.POINTER(C.c_int64)), ("count", C.c_int32), ("text", C.c_char_p),
                ("text_count", C.c_int32), ("text_width", C.c_int32)]


class AggSpec(C.Structure):
    _fields_ = [("kind", C.c_int32), ("input_type", C.c_int32), ("input", Program)]


class AggResult(C.Structure):
    _fields_ = [("i", C.c_int64), ("f", C.c_double), ("count", C.c_int64), ("is_null", C.c_int32),
                ("kind", C.c_int32)]


class Projection(C.Structure):
    _fields_ = [("column", C.c_int32), ("out_type", C.c_int32), ("program", Program)]


class SortConfig(C.Structure):
    _fields_ = [("digit_bits", C.c_int32), ("items_per_thread", C.c_int32), ("block_threads", C.c_int32),
                ("keep_trivial", C.c_int32)]


class JoinCond(C.Structure):
    _fields_ = [("left_col", C.c_int32), ("right_col", C.c_int32), ("cmp", C.c_int32)]


class JoinOutput(C.Structure):
    _fields_ = [("side", C.c_int32), ("column", C.c_int32)]


class Operand(C.Structure):
    _fields_ = [("data", C.c_void_p), ("type", C.c_int32), ("width", C.c_int32), ("is_scalar", C.c_int32)]


class GroupAgg(C.Structure):
    _fields_ = [("kind", C.c_int32), ("column", C.c_int32)]


class CsvError(C.Structure):
    _fields_ = [("bad_cells", C.c_uint64), ("first_row", C.c_uint32), ("first_field", C.c_int32),
                ("kind", C.c_int32)]


CSV_MAX_FIELDS = 64

P = C.POINTER
vp, sz, u32, i32, u64 = C.c_void_p, C.c_size_t, C.c_uint32, C.c_int32, C.c_uint64

# name -> (restype, argtypes). Every symbol declared in include/yq_ops.h.
PROTOTYPES = {
    "yq_status_string": (C.c_char_p, [C.c_int]),
    "yq_last_cuda_error": (C.c_int, []),
    "yq_abi_version": (C.c_int, []),
    "yq_agg_state_bytes": (sz, [i32]),
    "yq_agg_state_init": (C.c_int, [vp, P(AggSpec), i32, vp]),
    "yq_filter_aggregate_workspace_size": (sz, [u32, i32]),
    "yq_filter_aggregate": (C.c_int, [P(Batch), P(Program), P(Constants), P(AggSpec), i32, vp, vp, sz, vp]),
    "yq_agg_state_read": (C.c_int, [vp, P(AggSpec), i32, P(AggResult), vp]),
    "yq_filter_project_workspace_size": (sz, [u32]),
    "yq_filter_project": (C.c_int, [P(Batch), P(Program), P(Constants), P(Projection), i32, P(Column), u32,
                                    P(u32), P(u32), vp, sz, vp]),
    "yq_filter_project_noalloc": (C.c_int, [P(Batch), P(Program), P(Constants), P(Projection), i32, P(Column), u32,
                                            P(u32), P(u32), vp]),
    "yq_sort_workspace_size": (sz, [P(Column), u32]),
    "yq_sort_indices": (C.c_int, [P(Column), u32, i32, i32, vp, P(SortConfig), vp, sz, vp]),
    "yq_sort_indices_multi": (C.c_int, [P(Column), P(i32), P(i32), i32, u32, vp, P(SortConfig), vp, sz, vp]),
    "yq_sort_segments_workspace_size": (sz, [P(Column), u32, P(u32), i32]),
    "yq_sort_segments": (C.c_int, [P(Column), u32, P(u32), i32, i32, i32, vp, P(SortConfig), vp, sz, vp]),
    "yq_gather": (C.c_int, [P(Column), i32, vp, u32, P(Column), vp]),
    "yq_merge_workspace_size": (sz, [u32, i32]),
    "yq_merge_pass": (C.c_int, [P(Column), i32, i32, i32, i32, P(u32), i32, P(Column), vp, sz, vp]),
    "yq_order_by_workspace_size": (sz, [P(Column), u32, P(u32), i32]),
    "yq_order_by_batch_workspace_size": (sz, [P(Batch), i32, P(u32), i32]),
    "yq_agg_states_init": (C.c_int, [vp, i32, P(AggSpec), i32, vp]),
    "yq_agg_states_read": (C.c_int, [vp, i32, P(AggSpec), i32, P(AggResult), vp]),
    "yq_filter_aggregate_segments_workspace_size": (sz, [u32, i32]),
    "yq_filter_aggregate_segments": (C.c_int, [P(Batch), P(u32), i32, P(Program), P(Constants), P(AggSpec), i32,
                                                vp, vp, sz, vp]),
    "yq_filter_aggregate_ranges_workspace_size": (sz, [P(u32), P(u32), i32]),
    "yq_filter_aggregate_ranges": (C.c_int, [P(Batch), P(u32), P(u32), i32, P(Program), P(Constants), P(AggSpec),
                                              i32, vp, vp, sz, vp]),
    "yq_order_by_segments_workspace_size": (sz, [P(Column), u32, P(u32), i32]),
    "yq_order_by_segments": (C.c_int, [P(Batch), i32, i32, i32, P(u32), i32, P(Batch), P(SortConfig), vp, sz, vp]),
    "yq_order_by_segments_perm": (C.c_int, [P(Batch), i32, i32, i32, P(u32), i32, P(Batch), vp, P(SortConfig), vp,
                                            sz, vp]),
    "yq_sort_autotune": (C.c_int, [P(Column), u32, P(u32), i32, i32, P(SortConfig), vp]),
    "yq_order_by_tiled": (C.c_int, [P(Batch), i32, i32, i32, P(u32), i32, P(Batch), i32, vp, sz, vp]),
    "yq_order_by_autotune": (C.c_int, [P(Batch), i32, i32, i32, P(u32), i32, P(SortConfig), P(i32), vp]),
    "yq_order_by": (C.c_int, [P(Batch), i32, i32, i32, P(u32), i32, P(Batch), vp, sz, vp]),
    "yq_join_workspace_size": (sz, [u32, u32]),
    "yq_join_pairs": (C.c_int, [P(Batch), P(Batch), P(JoinCond), i32, vp, vp, u64, P(u64), vp, sz, vp]),
    "yq_join_project": (C.c_int, [P(Batch), P(Batch), P(JoinCond), i32, P(JoinOutput), i32, P(Column), u64,
                                  P(u64), vp, sz, vp]),
    "yq_join_pairs_or": (C.c_int, [P(Batch), P(Batch), P(JoinCond), vp, i32, vp, vp, u64, P(u64), vp, sz, vp]),
    "yq_join_project_or": (C.c_int, [P(Batch), P(Batch), P(JoinCond), vp, i32, P(JoinOutput), i32, P(Column), u64,
                                     P(u64), vp, sz, vp]),
    "yq_join_aggregate_workspace_size": (sz, [u32, u32, i32]),
    "yq_join_dim_table_size": (sz, [u32]),
    "yq_join_dim_table_build": (C.c_int, [P(Batch), P(Program), i32, P(Constants), vp, sz, P(u32), vp]),
    "yq_join_aggregate_prepared_workspace_size": (sz, [i32]),
    "yq_join_aggregate_prepared": (C.c_int, [P(Batch), P(Program), i32, vp, u32, u32, i32, P(Constants),
                                             P(AggSpec), i32, vp, vp, sz, vp]),
    "yq_join_aggregate": (C.c_int, [P(Batch), P(Program), i32, P(Batch), P(Program), i32, P(Constants),
                                    P(AggSpec), i32, vp, vp, sz, vp]),
    "yq_compare": (C.c_int, [Operand, Operand, i32, i32, vp, u32, vp]),
    "yq_logic": (C.c_int, [Operand, Operand, i32, vp, u32, vp]),
    "yq_binary": (C.c_int, [Operand, Operand, i32, vp, u32, vp]),
    "yq_cast": (C.c_int, [vp, i32, vp, i32, u32, vp]),
    "yq_prefix_sum_workspace_size": (sz, [u32]),
    "yq_prefix_sum_mask": (C.c_int, [vp, vp, u32, vp, sz, vp]),
    "yq_debug_lookback_stall": (C.c_int, [u32, vp, sz, vp]),
    "yq_prefix_sum_u32": (C.c_int, [vp, vp, u32, vp, sz, vp]),
    "yq_move_rows_filter": (C.c_int, [P(Column), vp, vp, u32, P(Column), vp]),
    "yq_move_rows_join": (C.c_int, [P(Column), vp, u32, i32, P(Column), vp]),
    "yq_move_rows_merge": (C.c_int, [P(Column), P(Column), vp, vp, i32, u32, P(Column), vp]),
    "yq_reduce": (C.c_int, [vp, i32, vp, u32, i32, vp, vp]),
    "yq_key_transform": (C.c_int, [vp, i32, vp, u32, i32, vp]),
    "yq_merge_path": (C.c_int, [vp, vp, i32, i32, i32, u32, u32, u32, vp, vp, vp, vp, vp]),
    "yq_cross_product_col": (C.c_int, [P(Column), u32, u32, i32, P(Column), vp]),
    "yq_group_by_workspace_size": (sz, [P(Column), u32, i32, u32]),
    "yq_group_by": (C.c_int, [P(Batch), i32, P(GroupAgg), i32, P(Column), u32, P(u32), vp, sz, vp]),
    "yq_csv_index_workspace_size": (sz, [u64]),
    "yq_csv_index": (C.c_int, [vp, u64, vp, u64, P(u64), vp, sz, vp]),
    "yq_csv_parse_workspace_size": (sz, [u32]),
    "yq_csv_parse": (C.c_int, [vp, u64, vp, u32, P(i32), i32, P(Column), i32, P(u32), P(CsvError), vp, sz, vp]),
    "yq_csv_format_workspace_size": (sz, [u32]),
    "yq_csv_format": (C.c_int, [P(Batch), vp, u64, P(u64), vp, sz, vp]),
    "yq_device_sm_count": (C.c_int, []),
    "yq_launch_count": (u64, []),
    "yq_profile_enable": (C.c_int, [i32]),
    "yq_jit_enable": (C.c_int, [i32]),
    "yq_jit_stats": (C.c_int, [P(i32), P(i32), P(i32), P(C.c_double), C.c_char_p, sz]),
    "yq_profile_read": (C.c_int, [C.c_char_p, sz, i32]),
}


class YQError(RuntimeError):
    def __init__(self, status: int, where: str, lib=None):
        msg = f"{where}: status {status}"
        if lib is not None:
            try:
                msg += f" ({lib.yq_status_string(status).decode()})"
                if status == ERR_CUDA:
                    msg += f", cudaError {lib.yq_last_cuda_error()}"
            except Exception:  # pragma: no cover - formatting only
                pass
        super().__init__(msg)
        self.status = status


_lib = None


def load(path: str | None = None, required_symbols: bool = False):
    """Load libyq_ops.so (in-tree). Raises ImportError when absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(f"libyq_ops.so not built at {p}; run `python -m yallasql_b200.build`")
    lib = C.CDLL(p)
    missing = []
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            missing.append(name)
            continue
        fn.restype = res
        fn.argtypes = args
    if missing and required_symbols:
        raise ImportError("libyq_ops.so lacks symbols: " + ", ".join(missing))
    lib._yq_missing = missing
    if path is None:
        _lib = lib
    return lib


def check(status: int, where: str) -> None:
    if status != OK:
        raise YQError(status, where, _lib)
