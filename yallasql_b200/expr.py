"""Expression trees and their compilation to the kernels' postfix programs.

The node classes mirror the reference's ``our::Expression`` hierarchy
(include/engine/operators/expressions/*.hpp):

=====================  ==================================================
``ColumnRef``          BoundRefExpression (bound_ref.hpp:7-45)
``Constant``           BoundValueExpression (bound_value.hpp:8-70)
``Cast``               CastExpression (cast.hpp:9-92)
``Arith``              BoundFuncExpression + - * / % (bound_func.hpp:25-169)
``Compare``            ComparisonExpression (filters/comparison.hpp:32-217)
``And`` / ``Or``       ConjuntionExpression (filters/conjunction.hpp:34-115)
``Not`` / ``IsNull``   OPERATOR_NOT / IS [NOT] NULL (expression.cpp:41-42)
``Aggregate``          AggregateExpression (aggregate.hpp:20-284)
=====================  ==================================================

Instead of one kernel launch and one materialised column per node, a tree
compiles to a postfix program (``yq_insn`` array) that the fused kernels run
per row in registers. Types follow what the planner inserted: an ``Arith``
or ``Compare`` needs both sides of the same type (wrap the other side in a
``Cast``, as DuckDB's binder does).
"""
from __future__ import annotations

import calendar
import ctypes as C
import struct
import time
from dataclasses import dataclass, field

from . import _abi as A

NUMERIC = (A.INT32, A.FLOAT32, A.INT64, A.DATETIME, A.FLOAT64)
WIDTH = {A.INT32: 4, A.FLOAT32: 4, A.INT64: 8, A.DATETIME: 8, A.FLOAT64: 8, A.BOOL: 1}
_FLIP = {A.LT: A.GT, A.LE: A.GE, A.GT: A.LT, A.GE: A.LE, A.EQ: A.EQ, A.NE: A.NE}


def parse_datetime(s: str) -> int:
    """Epoch seconds (UTC) of 'YYYY-MM-DD HH:MM:SS', 0 when it does not parse.

    Same contract as the reference's getDateTime (strptime + timegm,
    include/enums/data_type_utils.hpp:24-44)."""
    try:
        return int(calendar.timegm(time.strptime(s, "%Y-%m-%d %H:%M:%S")))
    except (ValueError, TypeError):
        return 0


class Expr:
    type: int

    def __and__(self, o):
        return And(self, o)

    def __or__(self, o):
        return Or(self, o)


@dataclass
class ColumnRef(Expr):
    index: int
    type: int


@dataclass
class Constant(Expr):
    value: object
    type: int

    def word(self) -> int:
        """Raw 64-bit constant-pool word for a numeric constant."""
        t = self.type
        if t in (A.INT32, A.INT64, A.BOOL):
            return int(self.value)
        if t == A.DATETIME:
            return parse_datetime(self.value) if isinstance(self.value, str) else int(self.value)
        if t == A.FLOAT32:
            return struct.unpack("<I", struct.pack("<f", float(self.value)))[0]
        if t == A.FLOAT64:
            return struct.unpack("<q", struct.pack("<d", float(self.value)))[0]
        raise TypeError("text constants live in the text pool")


@dataclass
class Cast(Expr):
    child: Expr
    to: int

    @property
    def type(self) -> int:
        return self.to


@dataclass
class Arith(Expr):
    op: int
    lhs: Expr
    rhs: Expr

    @property
    def type(self) -> int:
        return self.lhs.type


@dataclass
class Compare(Expr):
    op: int
    lhs: Expr
    rhs: Expr
    type: int = A.BOOL


class And(Expr):
    type = A.BOOL

    def __init__(self, *children: Expr):
        flat = []
        for c in children:
            flat.extend(c.children if isinstance(c, And) else [c])
        self.children = flat

    def __repr__(self):
        return "And(" + ", ".join(map(repr, self.children)) + ")"


class Or(Expr):
    type = A.BOOL

    def __init__(self, *children: Expr):
        flat = []
        for c in children:
            flat.extend(c.children if isinstance(c, Or) else [c])
        self.children = flat

    def __repr__(self):
        return "Or(" + ", ".join(map(repr, self.children)) + ")"


@dataclass
class Not(Expr):
    child: Expr
    type: int = A.BOOL


@dataclass
class IsNull(Expr):
    child: Expr
    negate: bool = False
    type: int = A.BOOL


@dataclass
class Aggregate:
    kind: int
    arg: Expr | None = None

    @property
    def input_type(self) -> int:
        return self.arg.type if self.arg is not None else A.INT64


def between(x: Expr, lo: Expr, hi: Expr) -> Expr:
    """x BETWEEN lo AND hi, lowered to x >= lo AND x <= hi (the reference has
    no COMPARE_BETWEEN case, expression.cpp:6-50)."""
    return And(Compare(A.GE, x, lo), Compare(A.LE, x, hi))


# ---------------------------------------------------------------- compiler
@dataclass
class ConstPool:
    words: list = field(default_factory=list)
    texts: list = field(default_factory=list)
    text_width: int = 0

    def num(self, c: Constant) -> int:
        w = c.word()
        key = (c.type, w)
        for i, (t, v) in enumerate(self.words):
            if (t, v) == key:
                return i
        if len(self.words) >= A.MAX_CONSTANTS:
            raise ValueError("too many constants")
        self.words.append(key)
        return len(self.words) - 1

    def text(self, s) -> int:
        b = s.encode() if isinstance(s, str) else bytes(s)
        if b in self.texts:
            return self.texts.index(b)
        if len(self.texts) >= A.MAX_TEXT_CONSTANTS:
            raise ValueError("too many text constants")
        self.texts.append(b)
        self.text_width = max(self.text_width, (len(b) + 4) // 4 * 4)
        return len(self.texts) - 1

    def to_c(self):
        """Returns (Constants struct, keepalive)."""
        vals = (C.c_int64 * max(1, len(self.words)))(*[C.c_int64(v).value for _, v in self.words])
        w = max(4, self.text_width)
        tb = b"".join(t.ljust(w, b"\0")[:w] for t in self.texts)
        k = A.Constants()
        k.values = vals
        k.count = len(self.words)
        k.text = tb if self.texts else None
        k.text_count = len(self.texts)
        k.text_width = w if self.texts else 0
        return k, (vals, tb)


def _insn(op, type_=0, a=0, b=0, imm=0):
    return (op, type_, a, b, imm)


def _cmp_operand_col(e: Expr):
    """A ColumnRef, possibly under a Cast: (column index, compare type)."""
    if isinstance(e, ColumnRef):
        return e.index, e.type
    if isinstance(e, Cast) and isinstance(e.child, ColumnRef):
        return e.child.index, e.to
    return None


def compile_expr(e: Expr, pool: ConstPool, col_types: list[int]) -> list[tuple]:
    """Postfix code for expression `e` (list of insn tuples)."""
    out: list[tuple] = []

    def emit(x: Expr):
        if isinstance(x, ColumnRef):
            out.append(_insn(A.OP_COL, x.type, x.index))
        elif isinstance(x, Constant):
            if x.value is None:
                out.append(_insn(A.OP_NULL, x.type))
            else:
                out.append(_insn(A.OP_CONST, x.type, imm=pool.num(x)))
        elif isinstance(x, Cast):
            emit(x.child)
            if x.child.type != x.to:
                out.append(_insn(A.OP_CAST, x.child.type, x.to))
        elif isinstance(x, Arith):
            if x.lhs.type != x.rhs.type:
                raise TypeError(f"arith operands differ: {x}")
            emit(x.lhs)
            emit(x.rhs)
            out.append(_insn(A.OP_ARITH, x.lhs.type, x.op))
        elif isinstance(x, Compare):
            lhs, rhs, op = x.lhs, x.rhs, x.op
            if isinstance(lhs, Constant) and not isinstance(rhs, Constant):
                lhs, rhs, op = rhs, lhs, _FLIP[op]
            lc = _cmp_operand_col(lhs)
            if lhs.type == A.TEXT or rhs.type == A.TEXT:
                if not isinstance(lhs, ColumnRef):
                    raise TypeError("text comparisons need a text column on one side")
                if isinstance(rhs, Constant):
                    out.append(_insn(A.OP_CMP_COL_CONST, A.TEXT, op, lhs.index, pool.text(rhs.value)))
                elif isinstance(rhs, ColumnRef):
                    out.append(_insn(A.OP_CMP_COL_COL, A.TEXT, op, lhs.index, rhs.index))
                else:
                    raise TypeError("unsupported text comparison")
                return
            if lhs.type != rhs.type:
                raise TypeError(f"compare operands differ: {x}")
            rc = _cmp_operand_col(rhs)
            if lc is not None and isinstance(rhs, Constant) and rhs.value is not None:
                out.append(_insn(A.OP_CMP_COL_CONST, lc[1], op, lc[0], pool.num(rhs)))
            elif lc is not None and rc is not None:
                out.append(_insn(A.OP_CMP_COL_COL, lc[1], op, lc[0], rc[0]))
            else:
                emit(lhs)
                emit(rhs)
                out.append(_insn(A.OP_CMP, lhs.type, op))
        elif isinstance(x, (And, Or)):
            op = A.OP_AND if isinstance(x, And) else A.OP_OR
            emit(x.children[0])
            for c in x.children[1:]:
                emit(c)
                out.append(_insn(op))
        elif isinstance(x, Not):
            emit(x.child)
            out.append(_insn(A.OP_NOT))
        elif isinstance(x, IsNull):
            emit(x.child)
            out.append(_insn(A.OP_IS_NOT_NULL if x.negate else A.OP_IS_NULL))
        else:
            raise TypeError(f"cannot compile {x!r}")

    emit(e)
    return out


class Compiled:
    """A program in C form plus the buffers it points into."""

    def __init__(self, code: list[tuple]):
        self.n = len(code)
        self.arr = (A.Insn * max(1, self.n))(*[A.Insn(*c) for c in code])
        self.prog = A.Program(self.arr, self.n)


def program(e: Expr | None, pool: ConstPool, col_types: list[int]) -> Compiled:
    return Compiled(compile_expr(e, pool, col_types) if e is not None else [])
