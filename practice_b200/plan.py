"""Star-join plan builder: the reference's optimised operator tree for the hot
path, written as the S-expression the C++ code generator reads.

The reference builds the tree with its SQL translator and optimiser, then the
push-model visitor derives build parameters and the aggregate layout.  This
module restates the derivations the generated code depends on:

* join build parameters -- ``JITOperatorVisitor::computeBuildInfo``
  (src/core/visitor.cpp:3864-4016): PART/SUPPLIER/CUSTOMER hash tables have
  ``len`` = table size and key minimum 0, DDATE has len 61131 and key minimum
  19920101, any other dimension uses its key column's catalog range; the
  payload is the first dimension column the aggregate (then a later filter)
  needs, which makes the join a PHT_2, otherwise PHT_1;
* result nullability -- ``resultColumnNullableForExpr`` (:128-170) and
  ``resultColumnNullableForAggregateOutput`` (:172-185);
* fast sparse output -- ``aggregateFastSparseOutputEligible`` (:2192-2213)
  and ``requires_dense_result`` set by ORDER BY / HAVING (:1937-1946, :1905).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Iterable

# ---------------------------------------------------------------- expressions


class E:
    """Expression node: op is one of the plan grammar's heads."""

    __slots__ = ("op", "kids", "name", "val")

    def __init__(self, op: str, *kids: "E", name: str | None = None, val: int | None = None):
        self.op, self.kids, self.name, self.val = op, kids, name, val

    def sexpr(self) -> str:
        if self.op == "col":
            return f"(col {self.name})"
        if self.op == "int":
            return f"(int {self.val})"
        if self.op in ("null", "star"):
            return f"({self.op})"
        return "(" + self.op + "".join(" " + k.sexpr() for k in self.kids) + ")"

    def columns(self) -> list[str]:
        out: list[str] = []
        if self.op == "col":
            out.append(self.name)
        for k in self.kids:
            for c in k.columns():
                if c not in out:
                    out.append(c)
        return out

    # arithmetic sugar
    def __add__(self, o): return E("add", self, _e(o))
    def __sub__(self, o): return E("sub", self, _e(o))
    def __mul__(self, o): return E("mul", self, _e(o))
    def __truediv__(self, o): return E("div", self, _e(o))
    def __radd__(self, o): return E("add", _e(o), self)
    def __rsub__(self, o): return E("sub", _e(o), self)
    def __rmul__(self, o): return E("mul", _e(o), self)

    # comparison helpers (== is kept for Python identity semantics)
    def eq(self, o): return E("eq", self, _e(o))
    def ne(self, o): return E("ne", self, _e(o))
    def lt(self, o): return E("lt", self, _e(o))
    def le(self, o): return E("le", self, _e(o))
    def gt(self, o): return E("gt", self, _e(o))
    def ge(self, o): return E("ge", self, _e(o))
    def between(self, lo, hi): return and_(self.ge(lo), self.le(hi))
    def is_null(self): return E("isnull", self)
    def not_null(self): return E("notnull", self)

    def __repr__(self) -> str:
        return self.sexpr()


def _e(x) -> E:
    if isinstance(x, E):
        return x
    if isinstance(x, bool):
        return E("int", val=int(x))
    if isinstance(x, int):
        return E("int", val=x)
    if x is None:
        return E("null")
    raise TypeError(f"cannot make an expression of {x!r}")


def col(name: str) -> E: return E("col", name=name)
def lit(v: int) -> E: return E("int", val=int(v))
def null() -> E: return E("null")
def star() -> E: return E("star")
def not_(a) -> E: return E("not", _e(a))
def case(cond, then, other) -> E: return E("case", _e(cond), _e(then), _e(other))


def and_(*xs) -> E:
    xs = [_e(x) for x in xs]
    out = xs[0]
    for x in xs[1:]:
        out = E("and", out, x)
    return out


def or_(*xs) -> E:
    xs = [_e(x) for x in xs]
    out = xs[0]
    for x in xs[1:]:
        out = E("or", out, x)
    return out


# ---------------------------------------------------------------------- plan


@dataclass
class Table:
    name: str
    cols: list[str]
    rows: int
    fact: bool = False
    key_col: str | None = None  # dimension key column (for generic build ranges)
    key_min: int = 0
    key_max: int = 0
    key_unique: bool = True     # catalog: the key column holds each value at most once
    # catalog statistics of attribute columns: column -> (min, distinct values)
    stats: dict = field(default_factory=dict)


@dataclass
class Join:
    dim: str
    pk: str
    fk: str
    length: int
    keymin: int
    filter: E | None = None
    payload: str | None = None
    more_fks: tuple[str, ...] = ()   # further fact keys of an OR-join
    multi: bool = False              # multi-value hash table (non-unique build key)
    gathers: tuple[str, ...] = ()    # MHT: build columns read through the row id
    prange: tuple[int, int] | None = None  # catalog (min, cardinality) of the payload's values

    @property
    def fks(self) -> tuple[str, ...]:
        return (self.fk,) + tuple(self.more_fks)

    @property
    def expands(self) -> bool:
        return self.multi or len(self.more_fks) > 0


@dataclass
class Group:
    expr: E
    min: int
    card: int
    nullable: bool = False


@dataclass
class Agg:
    fn: str  # count | sum | min | max | avg
    arg: E


@dataclass
class Plan:
    tables: list[Table]
    nullable: set[str]
    steps: list[tuple[str, object]] = field(default_factory=list)
    groups: list[Group] = field(default_factory=list)
    aggs: list[Agg] = field(default_factory=list)
    order_by: list[tuple[int, bool]] = field(default_factory=list)  # (visible col, descending)
    sparse: bool = False
    name: str = "query"

    @property
    def fact(self) -> Table:
        return next(t for t in self.tables if t.fact)

    # A built plan is not changed in place; assigning any field drops what was
    # derived from it (its text, its shape), so a query submitted again costs
    # no re-rendering.
    def __setattr__(self, name, value):
        object.__setattr__(self, name, value)
        if name != "_memo":
            object.__setattr__(self, "_memo", {})

    def memo(self, key: str, fn):
        m = self.__dict__.setdefault("_memo", {})
        if key not in m:
            m[key] = fn()
        return m[key]

    def text(self) -> str:
        return self.memo("text", self._render)

    def _render(self) -> str:
        out = ["(query"]
        for t in self.tables:
            out.append(f"  (table {t.name}{' fact' if t.fact else ''} (cols {' '.join(t.cols)}))")
        if self.nullable:
            out.append(f"  (nullable {' '.join(sorted(self.nullable))})")
        for kind, s in self.steps:
            if kind == "filter":
                out.append(f"  (filter {s.sexpr()})")
            else:
                j: Join = s
                parts = [f"(join {j.dim} (pk {j.pk}) (fk {' '.join(j.fks)}) (len {j.length}) (keymin {j.keymin})"]
                if j.multi:
                    parts.append(" (multi 1)")
                if j.filter is not None:
                    parts.append(f" (filter {j.filter.sexpr()})")
                if j.multi and j.gathers:
                    parts.append(f" (payload {' '.join(j.gathers)})")
                elif j.payload:
                    parts.append(f" (payload {j.payload})")
                    if j.prange:
                        parts.append(f" (prange {j.prange[0]} {j.prange[1]})")
                out.append("  " + "".join(parts) + ")")
        agg = ["  (aggregate"]
        for g in self.groups:
            agg.append(f"    (group {g.expr.sexpr()} (min {g.min}) (card {g.card}) (nullable {int(g.nullable)}))")
        for a in self.aggs:
            agg.append(f"    ({a.fn} {a.arg.sexpr()})")
        agg.append(f"    (sparse {int(self.sparse)}))")
        out.append("\n".join(agg))
        out.append(")")
        return "\n".join(out) + "\n"

    # result layout (AggregateNode::visibleTupleSize / storageTupleSize, include/core/operators.h:303-321)
    @property
    def visible_ts(self) -> int:
        return len(self.groups) + len(self.aggs)

    @property
    def storage_ts(self) -> int:
        s = len(self.groups) + len(self.aggs) + sum(1 for a in self.aggs if a.fn == "avg")
        return s if s else 1

    @property
    def group_slots(self) -> int:
        n = 1
        for g in self.groups:
            n *= g.card + (1 if g.nullable else 0)
        return n

    def columns_read(self) -> list[str]:
        """Distinct fact columns the scan reads (the roofline's algorithmic bytes)."""
        fact = set(self.fact.cols)
        seen: list[str] = []

        def add(cs: Iterable[str]):
            for c in cs:
                if c in fact and c not in seen:
                    seen.append(c)

        for kind, s in self.steps:
            if kind == "filter":
                add(s.columns())
            else:
                add(list(s.fks))
        for g in self.groups:
            add(g.expr.columns())
        for a in self.aggs:
            add(a.arg.columns())
        return seen


# ----------------------------------------------------------- derivations


def expr_nullable(e: E | None, nullable: set[str]) -> bool:
    """resultColumnNullableForExpr (src/core/visitor.cpp:128-170)."""
    if e is None:
        return True
    if e.op == "null":
        return True
    if e.op in ("star", "int", "isnull", "notnull"):
        return False
    if e.op == "col":
        return e.name in nullable
    if e.op == "not":
        return expr_nullable(e.kids[0], nullable)
    if e.op == "case":
        return expr_nullable(e.kids[1], nullable) or expr_nullable(e.kids[2], nullable)
    return any(expr_nullable(k, nullable) for k in e.kids)


def build_params(dim: Table) -> tuple[int, int]:
    """(len, keymin) of a dimension's perfect hash table (computeBuildInfo)."""
    if dim.name in ("PART", "SUPPLIER", "CUSTOMER"):
        return dim.rows, 0
    if dim.name == "DDATE":
        return 61131, 19920101
    if dim.key_col is not None:
        return dim.key_max - dim.key_min + 1, dim.key_min
    return dim.rows, 0


def choose_payload(dim: Table, pk: str, agg_cols: list[str], later_filter_cols: list[str]) -> str | None:
    for cols in (agg_cols, later_filter_cols):
        for c in cols:
            if c in dim.cols and c != pk:
                return c
    return None


def sparse_eligible(plan: Plan) -> bool:
    """aggregateFastSparseOutputEligible && !requires_dense_result."""
    if plan.order_by:
        return False
    if any(a.fn == "avg" for a in plan.aggs):
        return False
    for g in plan.groups:
        if g.nullable:
            return False
    for a in plan.aggs:
        if a.fn != "count" and expr_nullable(a.arg, plan.nullable):
            return False
    if not all(a.fn in ("count", "sum") for a in plan.aggs):
        return False
    if not plan.groups:
        return True
    for g in plan.groups:
        if g.expr.op == "col" and g.min != 0:
            return True
    return any(a.fn == "count" for a in plan.aggs)


class PlanBuilder:
    """Builds a Plan in the order the visitor walks it: fact scan, then filters
    and joins upward, then the aggregate."""

    def __init__(self, tables: dict[str, Table], fact: str, nullable: Iterable[str] = (), name: str = "query"):
        self.all_tables = tables
        self.fact = tables[fact]
        self.nullable = set(nullable)
        self.name = name
        self._steps: list[tuple[str, object]] = []
        self._pending_joins: list[tuple[int, str, str, str, E | None, str | None]] = []

    def filter(self, pred: E) -> "PlanBuilder":
        self._steps.append(("filter", pred))
        return self

    def join(self, dim: str, fk: str | tuple[str, ...], pk: str | None = None, where: E | None = None,
             payload: str | None = None) -> "PlanBuilder":
        """Joins a dimension.  `fk` may name several fact keys: the SQL form
        `(fk1 = pk OR fk2 = pk)`, probed once per distinct key
        (visitor.cpp:4587-4640).  A dimension whose key the catalog marks
        non-unique becomes a multi-value hash table (:3947-3968)."""
        d = self.all_tables[dim]
        pk = pk or d.key_col or d.cols[0]
        self._pending_joins.append((len(self._steps), dim, pk, fk, where, payload))
        self._steps.append(("join", None))
        return self

    def aggregate(self, groups: list[tuple[E, int, int]] | list[Group], aggs: list[tuple[str, E]],
                  order_by: list[tuple[int, bool]] | None = None) -> Plan:
        gl: list[Group] = []
        for g in groups:
            if isinstance(g, Group):
                gl.append(g)
            else:
                e, mn, card = g
                gl.append(Group(e, mn, card, expr_nullable(e, self.nullable) if e.op == "col" else False))
        al = [Agg(fn, arg) for fn, arg in aggs]
        agg_cols: list[str] = []
        for a in al:
            for c in a.arg.columns():
                if c not in agg_cols:
                    agg_cols.append(c)
        for g in gl:
            for c in g.expr.columns():
                if c not in agg_cols:
                    agg_cols.append(c)
        steps = list(self._steps)
        used_tables = [self.fact]
        for idx, dim, pk, fk, where, payload in self._pending_joins:
            d = self.all_tables[dim]
            later_filter_cols: list[str] = []
            for kind, s in steps[idx + 1:]:
                if kind == "filter":
                    later_filter_cols += s.columns()
            fks = (fk,) if isinstance(fk, str) else tuple(fk)
            length, keymin = build_params(d)
            if not d.key_unique:
                # MHT: the payload is the build row id, so every dimension column
                # used above the join is read through it.
                gathers = tuple(c for c in dict.fromkeys(agg_cols + later_filter_cols) if c in d.cols)
                steps[idx] = ("join", Join(dim, pk, fks[0], length, keymin, where, None, fks[1:], True, gathers))
            else:
                if payload is None:
                    payload = choose_payload(d, pk, agg_cols, later_filter_cols)
                prange = d.stats.get(payload) if payload else None
                steps[idx] = ("join", Join(dim, pk, fks[0], length, keymin, where, payload, fks[1:],
                                           prange=tuple(prange) if prange else None))
            used_tables.append(d)
        plan = Plan(tables=used_tables, nullable=set(self.nullable), steps=steps, groups=gl, aggs=al,
                    order_by=list(order_by or []), name=self.name)
        plan.sparse = sparse_eligible(plan)
        return plan
