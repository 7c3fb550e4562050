"""Operator configuration types, mirroring the reference's Rust types.

Reference definitions (native/prism-executor/src):
  hash_join.rs:48-64        JoinType, HashJoinConfig
  hash_aggregate.rs:79-101  AggFunc, AggExpr, HashAggConfig
  filter_project.rs:22-62   Predicate, ScalarValue
  filter_project.rs:186-213 ArithmeticOp, ScalarExpr

Each tree is flattened to the post-order POD arrays of include/prism_gpu.h by
``encode()``; the returned object keeps every ctypes buffer alive.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

from . import _abi


class JoinType(enum.IntEnum):
    Inner = 0
    Left = 1
    Right = 2
    Full = 3
    LeftSemi = 4
    LeftAnti = 5


@dataclass
class HashJoinConfig:
    join_type: JoinType
    build_keys: List[int]
    probe_keys: List[int]

    def encode(self):
        pk = _abi.int_array(self.probe_keys)
        bk = _abi.int_array(self.build_keys)
        cfg = _abi.prism_join_config(int(self.join_type), len(self.probe_keys), pk, bk)
        cfg._keep = (pk, bk)
        return cfg


class SortDirection(enum.IntEnum):
    """SortDirection (sort.rs:13-17)."""
    Asc = 0
    Desc = 1


class NullOrdering(enum.IntEnum):
    """NullOrdering (sort.rs:20-24)."""
    NullsFirst = 0
    NullsLast = 1


@dataclass
class SortKey:
    """SortKey (sort.rs:27-32)."""
    column: int
    direction: SortDirection = SortDirection.Asc
    nulls: NullOrdering = NullOrdering.NullsLast


def encode_sort_keys(keys):
    arr = (_abi.prism_sort_key * max(1, len(keys)))()
    for i, k in enumerate(keys):
        arr[i].column = k.column
        arr[i].descending = 1 if k.direction == SortDirection.Desc else 0
        arr[i].nulls_first = 1 if k.nulls == NullOrdering.NullsFirst else 0
    return arr


class AggFunc(enum.IntEnum):
    Sum = 0
    Count = 1
    Avg = 2
    Min = 3
    Max = 4
    CountDistinct = 5


@dataclass
class AggExpr:
    column: int
    func: AggFunc
    output_name: str


@dataclass
class HashAggConfig:
    group_by: List[int]
    aggregates: List[AggExpr]

    def encode(self):
        gb = _abi.int_array(self.group_by)
        names = [a.output_name.encode() for a in self.aggregates]
        aggs = (_abi.prism_agg_expr * max(1, len(self.aggregates)))()
        for i, a in enumerate(self.aggregates):
            aggs[i].column = a.column
            aggs[i].func = int(a.func)
            aggs[i].output_name = names[i]
        cfg = _abi.prism_agg_config(len(self.group_by), gb, len(self.aggregates), aggs)
        cfg._keep = (gb, aggs, names)
        return cfg


# ----------------------------------------------------------- ScalarValue ----

SCALAR_INT32, SCALAR_INT64, SCALAR_FLOAT64, SCALAR_UTF8, SCALAR_BOOLEAN, SCALAR_DATE32 = range(6)


@dataclass(frozen=True)
class ScalarValue:
    kind: int
    value: object

    @staticmethod
    def Int32(v: int) -> "ScalarValue":
        return ScalarValue(SCALAR_INT32, int(v))

    @staticmethod
    def Int64(v: int) -> "ScalarValue":
        return ScalarValue(SCALAR_INT64, int(v))

    @staticmethod
    def Float64(v: float) -> "ScalarValue":
        return ScalarValue(SCALAR_FLOAT64, float(v))

    @staticmethod
    def Utf8(v: str) -> "ScalarValue":
        return ScalarValue(SCALAR_UTF8, str(v))

    @staticmethod
    def Boolean(v: bool) -> "ScalarValue":
        return ScalarValue(SCALAR_BOOLEAN, bool(v))

    @staticmethod
    def Date32(v: int) -> "ScalarValue":
        return ScalarValue(SCALAR_DATE32, int(v))

    def fill(self, s: _abi.prism_scalar, keep: list):
        s.type = self.kind
        if self.kind == SCALAR_FLOAT64:
            s.f64 = self.value
        elif self.kind == SCALAR_UTF8:
            b = self.value.encode("utf-8")
            keep.append(b)
            s.str = b
            s.str_len = len(b)
        elif self.kind == SCALAR_BOOLEAN:
            s.i64 = 1 if self.value else 0
        else:
            s.i64 = self.value


# ------------------------------------------------------------- Predicate ----

PRED_OPS = {
    "Literal": 0, "Eq": 1, "Ne": 2, "Lt": 3, "Le": 4, "Gt": 5, "Ge": 6,
    "IsNull": 7, "IsNotNull": 8, "And": 9, "Or": 10, "Not": 11, "Like": 12, "ILike": 13,
}


@dataclass(frozen=True)
class Predicate:
    op: str
    column: int = -1
    value: object = None  # ScalarValue, bool (Literal) or str (Like pattern)
    children: Tuple["Predicate", ...] = ()

    @staticmethod
    def Literal(v: bool):
        return Predicate("Literal", value=bool(v))

    @staticmethod
    def Eq(c, v):
        return Predicate("Eq", c, v)

    @staticmethod
    def Ne(c, v):
        return Predicate("Ne", c, v)

    @staticmethod
    def Lt(c, v):
        return Predicate("Lt", c, v)

    @staticmethod
    def Le(c, v):
        return Predicate("Le", c, v)

    @staticmethod
    def Gt(c, v):
        return Predicate("Gt", c, v)

    @staticmethod
    def Ge(c, v):
        return Predicate("Ge", c, v)

    @staticmethod
    def IsNull(c):
        return Predicate("IsNull", c)

    @staticmethod
    def IsNotNull(c):
        return Predicate("IsNotNull", c)

    @staticmethod
    def And(a, b):
        return Predicate("And", children=(a, b))

    @staticmethod
    def Or(a, b):
        return Predicate("Or", children=(a, b))

    @staticmethod
    def Not(a):
        return Predicate("Not", children=(a,))

    @staticmethod
    def Like(c, pattern: str):
        return Predicate("Like", c, pattern)

    @staticmethod
    def ILike(c, pattern: str):
        return Predicate("ILike", c, pattern)

    def columns(self) -> set:
        out = set()
        if self.op not in ("Literal", "And", "Or", "Not"):
            out.add(self.column)
        for ch in self.children:
            out |= ch.columns()
        return out

    def post_order(self) -> List["Predicate"]:
        out: List[Predicate] = []
        for ch in self.children:
            out.extend(ch.post_order())
        out.append(self)
        return out

    def fill_nodes(self, arr, start: int, keep: list) -> int:
        nodes = self.post_order()
        for i, p in enumerate(nodes):
            n = arr[start + i]
            n.op = PRED_OPS[p.op]
            n.column = p.column
            if p.op == "Literal":
                n.value.type = SCALAR_BOOLEAN
                n.value.i64 = 1 if p.value else 0
            elif p.op in ("Like", "ILike"):
                b = p.value.encode("utf-8")
                keep.append(b)
                n.value.type = SCALAR_UTF8
                n.value.str = b
                n.value.str_len = len(b)
            elif isinstance(p.value, ScalarValue):
                p.value.fill(n.value, keep)
        return len(nodes)

    def encode(self):
        nodes = self.post_order()
        arr = (_abi.prism_pred_node * len(nodes))()
        keep: list = []
        self.fill_nodes(arr, 0, keep)
        pred = _abi.prism_predicate(arr, len(nodes))
        pred._keep = (arr, keep)
        return pred


# ------------------------------------------------------------ ScalarExpr ----


class ArithmeticOp(enum.IntEnum):
    Add = 2
    Subtract = 3
    Multiply = 4
    Divide = 5


EXPR_COLUMN, EXPR_LITERAL, EXPR_NEG, EXPR_IF_THEN = 0, 1, 6, 7

ARITH_F64 = 0
ARITH_EXACT = 1


@dataclass(frozen=True)
class ScalarExpr:
    kind: str
    column: int = -1
    literal: Optional[ScalarValue] = None
    op: Optional[ArithmeticOp] = None
    children: Tuple["ScalarExpr", ...] = ()
    clauses: Tuple[Tuple[Predicate, "ScalarExpr"], ...] = ()
    else_expr: Optional["ScalarExpr"] = None

    @staticmethod
    def ColumnRef(i: int):
        return ScalarExpr("ColumnRef", column=i)

    @staticmethod
    def Literal(v: ScalarValue):
        return ScalarExpr("Literal", literal=v)

    @staticmethod
    def BinaryOp(op: ArithmeticOp, left: "ScalarExpr", right: "ScalarExpr"):
        return ScalarExpr("BinaryOp", op=op, children=(left, right))

    @staticmethod
    def Negate(x: "ScalarExpr"):
        return ScalarExpr("Negate", children=(x,))

    @staticmethod
    def IfThen(clauses: Sequence[Tuple[Predicate, "ScalarExpr"]], else_expr: Optional["ScalarExpr"] = None):
        return ScalarExpr("IfThen", clauses=tuple(clauses), else_expr=else_expr)

    def columns(self) -> set:
        out = set()
        if self.kind == "ColumnRef":
            out.add(self.column)
        for ch in self.children:
            out |= ch.columns()
        for p, e in self.clauses:
            out |= p.columns() | e.columns()
        if self.else_expr is not None:
            out |= self.else_expr.columns()
        return out

    def encode(self):
        nodes: list = []
        preds: list = []  # (Predicate) in pool order
        clause_list: list = []

        def walk(e: ScalarExpr):
            if e.kind == "ColumnRef":
                nodes.append(("col", e))
            elif e.kind == "Literal":
                nodes.append(("lit", e))
            elif e.kind == "BinaryOp":
                walk(e.children[0])
                walk(e.children[1])
                nodes.append(("bin", e))
            elif e.kind == "Negate":
                walk(e.children[0])
                nodes.append(("neg", e))
            elif e.kind == "IfThen":
                for _, then in e.clauses:
                    walk(then)
                if e.else_expr is not None:
                    walk(e.else_expr)
                begin = len(clause_list)
                for p, _ in e.clauses:
                    clause_list.append(p)
                nodes.append(("if", e, begin))
            else:
                raise ValueError(e.kind)

        walk(self)
        keep: list = []
        narr = (_abi.prism_expr_node * len(nodes))()
        # predicate pool
        pred_sizes = [len(p.post_order()) for p in clause_list]
        parr = (_abi.prism_pred_node * max(1, sum(pred_sizes)))()
        carr = (_abi.prism_expr_clause * max(1, len(clause_list)))()
        pos = 0
        for i, p in enumerate(clause_list):
            carr[i].pred_begin = pos
            carr[i].pred_len = p.fill_nodes(parr, pos, keep)
            pos += carr[i].pred_len
        for i, item in enumerate(nodes):
            n = narr[i]
            kind, e = item[0], item[1]
            if kind == "col":
                n.op = EXPR_COLUMN
                n.column = e.column
            elif kind == "lit":
                n.op = EXPR_LITERAL
                e.literal.fill(n.literal, keep)
            elif kind == "bin":
                n.op = int(e.op)
            elif kind == "neg":
                n.op = EXPR_NEG
            else:
                n.op = EXPR_IF_THEN
                n.n_clauses = len(e.clauses)
                n.has_else = 1 if e.else_expr is not None else 0
                n.clause_begin = item[2]
        ex = _abi.prism_expr(narr, len(nodes), parr, sum(pred_sizes), carr, len(clause_list))
        ex._keep = (narr, parr, carr, keep)
        return ex


def encode_exprs(exprs: Sequence[ScalarExpr]):
    encoded = [e.encode() for e in exprs]
    arr = (_abi.prism_expr * max(1, len(encoded)))(*encoded)
    arr._keep = encoded
    return arr
