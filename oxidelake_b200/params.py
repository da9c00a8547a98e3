"""Plan vocabulary, mirrored from crates/oxidelake-core/src/params.rs.

``Predicate`` is an AND-tree of ``column <op> literal`` comparisons
(params.rs:60-113); ``AggregateSpec`` a group key and ``(function, column)``
pairs (params.rs:142-147); ``DistanceMetric`` L2 or cosine
(params.rs:151-166).  Widened beyond the reference by Int32 literals, AVG and
COUNT(*), which the north-star queries need.
"""
from __future__ import annotations

import enum
from dataclasses import dataclass, field
from typing import List, Tuple, Union


class Comparison(enum.IntEnum):
    """params.rs:12-36; the values are the ABI's oxb_cmp."""

    Eq = 0
    Lt = 1
    LtEq = 2
    Gt = 3
    GtEq = 4

    def symbol(self) -> str:
        return {0: "=", 1: "<", 2: "<=", 3: ">", 4: ">="}[int(self)]


class LiteralType(enum.IntEnum):
    Int64 = 1
    Float64 = 2
    Int32 = 3


@dataclass(frozen=True)
class Literal:
    """params.rs:40-55 (Int64 / Float64), plus Int32."""

    type: LiteralType
    value: Union[int, float]

    @staticmethod
    def int64(v: int) -> "Literal":
        return Literal(LiteralType.Int64, int(v))

    @staticmethod
    def float64(v: float) -> "Literal":
        return Literal(LiteralType.Float64, float(v))

    @staticmethod
    def int32(v: int) -> "Literal":
        if not -(2**31) <= int(v) < 2**31:
            raise ValueError("Int32 literal out of range")
        return Literal(LiteralType.Int32, int(v))


@dataclass(frozen=True)
class Compare:
    column: int
    op: Comparison
    literal: Literal


@dataclass(frozen=True)
class And:
    left: "Predicate"
    right: "Predicate"


Predicate = Union[Compare, And]


def compare(column: int, op: Comparison, literal: Literal) -> Compare:
    """Predicate::compare (params.rs:76)."""
    return Compare(column, Comparison(op), literal)


def and_(left: Predicate, right: Predicate) -> And:
    """Predicate::and (params.rs:85)."""
    return And(left, right)


def leaves(p: Predicate | None) -> List[Compare]:
    """The comparison leaves in evaluation order (Predicate::columns order,
    params.rs:90-104).  A WHERE keeps a row only when every leaf is true, so
    the AND-tree flattens exactly."""
    if p is None:
        return []
    if isinstance(p, Compare):
        return [p]
    return leaves(p.left) + leaves(p.right)


def columns(p: Predicate) -> List[int]:
    return [lf.column for lf in leaves(p)]


def leaf_count(p: Predicate) -> int:
    return len(leaves(p))


class AggregateFunction(enum.IntEnum):
    """params.rs:117-138 (Sum, Count, Min, Max) plus Avg and CountStar; the
    values are the ABI's oxb_agg_func."""

    Sum = 0
    Count = 1
    Min = 2
    Max = 3
    Avg = 4
    CountStar = 5

    def sql_name(self) -> str:
        return {0: "SUM", 1: "COUNT", 2: "MIN", 3: "MAX", 4: "AVG", 5: "COUNT"}[int(self)]


@dataclass
class AggregateSpec:
    """params.rs:142-147."""

    group_by: int
    aggregates: List[Tuple[AggregateFunction, int]] = field(default_factory=list)


class DistanceMetric(enum.IntEnum):
    """params.rs:151-166."""

    L2 = 0
    Cosine = 1

    def metric_name(self) -> str:
        return "l2" if self == DistanceMetric.L2 else "cosine"
