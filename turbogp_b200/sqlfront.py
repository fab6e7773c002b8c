"""The SQL the wire front-end accepts, lowered onto the engine's operators.

The subset is the shape of the analytic statements this backend executes
(the reference's interpreter handles them in ``build_mask`` /
``execute_grouped`` / ``hash_join_with_keys``, src/engine/query_interpreter/
expr.rs:419, aggregate.rs:507, join.rs:544):

    SELECT item [, item]...
    FROM table [, table]
    [WHERE cond [AND cond]...]
    [GROUP BY column [, column]...]
    [ORDER BY position [ASC | DESC] LIMIT n]

* ``item``: a column of the GROUP BY list, ``COUNT(*)``, or ``SUM | AVG |
  MIN | MAX | COUNT (arith)`` with ``arith`` a product of factors, each a
  column, an integer, or an affine ``(k - column)``, ``(k + column)``,
  ``(column - k)``, ``(column + k)``; an optional ``AS name``.
* ``cond``: ``column op integer`` (op: = <> != < <= > >=), ``column [NOT]
  BETWEEN integer AND integer``, or, with two tables, the equi-join
  condition ``a.column = b.column``. Conditions on the second table filter the
  join's build side (``apply_single_table_filters``, join.rs:79-100).
* Columns may be qualified (``t.c``); unqualified names resolve to the one
  table that has them.

Anything else raises ``SqlError`` with the SQLSTATE the reference's server
returns for it (42601 syntax error, 42703 unknown column, 42P01 unknown table,
0A000 unsupported).
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field

from .engine import Agg, Col, Pred, avg, build_col, col, count_col, count_star, lit, max_, min_, sum_


class SqlError(Exception):
    def __init__(self, sqlstate: str, message: str):
        super().__init__(message)
        self.sqlstate = sqlstate


_TOKEN = re.compile(r"\s*(?:(?P<num>\d+)|(?P<id>[A-Za-z_][A-Za-z_0-9]*)|(?P<op><>|!=|<=|>=|[=<>(),.*+\-;]))")
_KEYWORDS = {"select", "from", "where", "and", "group", "by", "order", "limit", "asc", "desc", "between", "not",
             "as", "sum", "avg", "min", "max", "count", "or"}


def tokenize(sql: str) -> list[tuple[str, str]]:
    out, pos = [], 0
    sql = sql.strip()
    while pos < len(sql):
        m = _TOKEN.match(sql, pos)
        if not m or m.end() == pos:
            raise SqlError("42601", f"syntax error at or near {sql[pos:pos + 10]!r}")
        pos = m.end()
        if m.group("num") is not None:
            out.append(("num", m.group("num")))
        elif m.group("id") is not None:
            w = m.group("id")
            out.append(("kw", w.lower()) if w.lower() in _KEYWORDS else ("id", w))
        else:
            out.append(("op", m.group("op")))
    while out and out[-1] == ("op", ";"):
        out.pop()
    return out


@dataclass
class TableInfo:
    """What the front-end knows of a registered table: its column names and
    comparison types ('int' | 'date' | 'float')."""
    name: str
    columns: list[str]
    coltypes: dict = field(default_factory=dict)


@dataclass
class SelectItem:
    kind: str            # "key" | "agg"
    index: int           # position among the GROUP BY keys or the aggregates
    name: str


@dataclass
class QuerySpec:
    """A parsed statement, lowered: the probe table, its WHERE, the join
    (build table, build key, probe key, build WHERE), GROUP BY keys,
    aggregates, the output columns, ORDER BY / LIMIT, and ``shape``: the
    statement with the probe-side WHERE literals blanked (statements of one
    shape share a prepared query, rebound to each one's WHERE)."""
    table: str
    where: Pred | None
    group_by: tuple
    aggs: list[Agg]
    items: list[SelectItem]
    join: tuple | None = None          # (build table, build key, probe key, build where)
    order: tuple | None = None         # (aggregate index, descending)
    limit: int | None = None
    shape: str = ""


class _Parser:
    def __init__(self, tokens, catalog: dict[str, TableInfo]):
        self.t, self.i, self.catalog = tokens, 0, catalog
        self.tables: list[TableInfo] = []
        self.shape: list[str] = []

    # -- token helpers ------------------------------------------------------
    def peek(self, k: int = 0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else ("eof", "")

    def take(self):
        tok = self.peek()
        self.i += 1
        return tok

    def accept(self, kind, val=None) -> bool:
        tok = self.peek()
        if tok[0] == kind and (val is None or tok[1] == val):
            self.i += 1
            return True
        return False

    def expect(self, kind, val=None):
        tok = self.take()
        if tok[0] != kind or (val is not None and tok[1] != val):
            raise SqlError("42601", f"syntax error at or near {tok[1]!r}" if tok[0] != "eof" else
                           "syntax error at end of input")
        return tok

    def number(self) -> int:
        neg = self.accept("op", "-")
        v = int(self.expect("num")[1])
        return -v if neg else v

    # -- names ----------------------------------------------------------------
    def colref(self) -> tuple[int, str]:
        """(table position, column name) of a possibly qualified column."""
        name = self.expect("id")[1]
        if self.accept("op", "."):
            tname, cname = name, self.expect("id")[1]
            for k, ti in enumerate(self.tables):
                if ti.name == tname:
                    if cname not in ti.columns:
                        raise SqlError("42703", f'column "{tname}.{cname}" does not exist')
                    return k, cname
            raise SqlError("42P01", f'missing FROM-clause entry for table "{tname}"')
        owners = [k for k, ti in enumerate(self.tables) if name in ti.columns]
        if not owners:
            raise SqlError("42703", f'column "{name}" does not exist')
        if len(owners) > 1:
            raise SqlError("42702", f'column reference "{name}" is ambiguous')
        return owners[0], name

    def column(self, ref) -> Col:
        k, name = ref
        return col(name) if k == 0 else build_col(name)

    # -- expressions ----------------------------------------------------------
    def factor(self):
        if self.peek()[0] == "num" or (self.peek() == ("op", "-") and self.peek(1)[0] == "num"):
            return lit(self.number())
        if self.accept("op", "("):
            if self.peek()[0] == "num" or (self.peek() == ("op", "-") and self.peek(1)[0] == "num"):
                k = self.number()
                op = self.take()
                c = self.column(self.colref())
                self.expect("op", ")")
                if op == ("op", "-"):
                    return k - c
                if op == ("op", "+"):
                    return c + k
                raise SqlError("0A000", "only (k - column) and (k + column) forms are supported")
            e = self.arith()
            if self.accept("op", "-"):
                e = e - self.number()
            elif self.accept("op", "+"):
                e = e + self.number()
            self.expect("op", ")")
            return e
        return self.column(self.colref())

    def arith(self):
        e = self.factor()
        while self.accept("op", "*"):
            e = e * self.factor()
        return e

    # -- clauses --------------------------------------------------------------
    def select_list(self):
        raw = []
        while True:
            if self.peek()[0] == "kw" and self.peek()[1] in ("sum", "avg", "min", "max", "count"):
                fn = self.take()[1]
                self.expect("op", "(")
                if fn == "count" and self.accept("op", "*"):
                    agg, label = ("count*", None), "count"
                else:
                    agg, label = (fn, self.arith()), fn
                self.expect("op", ")")
                raw.append(("agg", agg, label))
            else:
                ref = self.colref_deferred()
                raw.append(("col", ref, ref[1]))
            if self.accept("kw", "as"):
                name = self.expect("id")[1]
                raw[-1] = (raw[-1][0], raw[-1][1], name)
            if not self.accept("op", ","):
                return raw

    def colref_deferred(self):
        """A select-list column before FROM is parsed: (qualifier or None, name)."""
        name = self.expect("id")[1]
        if self.accept("op", "."):
            return name, self.expect("id")[1]
        return None, name

    def resolve_deferred(self, q, name):
        for k, ti in enumerate(self.tables):
            if (q is None or ti.name == q) and name in ti.columns:
                return k, name
        raise SqlError("42703", f'column "{name}" does not exist')


def parse(sql: str, catalog: dict[str, TableInfo]) -> QuerySpec:
    """Parses one statement against the catalog of registered tables."""
    tokens = tokenize(sql)
    p = _Parser(tokens, catalog)
    p.expect("kw", "select")
    # The select list refers to tables named later: parse FROM first.
    depth, j = 0, p.i
    while j < len(tokens) and not (tokens[j] == ("kw", "from") and depth == 0):
        depth += {("op", "("): 1, ("op", ")"): -1}.get(tokens[j], 0)
        j += 1
    if j == len(tokens):
        raise SqlError("42601", "syntax error: missing FROM")
    select_start = p.i
    p.i = j + 1
    for k in range(2):
        name = p.expect("id")[1]
        if name not in catalog:
            raise SqlError("42P01", f'relation "{name}" does not exist')
        p.tables.append(catalog[name])
        if not p.accept("op", ","):
            break
    if p.peek() == ("op", ","):
        raise SqlError("0A000", "at most two tables (one equi-join)")
    after_from = p.i
    p.i = select_start
    raw = p.select_list()
    if p.i != j:
        raise SqlError("42601", f"syntax error at or near {p.peek()[1]!r}")
    p.i = after_from

    probe_leaves, build_leaves, join_eq = [], [], None
    shape = []
    if p.accept("kw", "where"):
        while True:
            ref = p.colref()
            negate = p.accept("kw", "not")
            if negate and p.peek() != ("kw", "between"):
                raise SqlError("42601", f"syntax error at or near {p.peek()[1]!r}")
            if p.accept("kw", "between"):
                a = p.number()
                p.expect("kw", "and")
                b = p.number()
                c = Col(ref[1])
                leaf = c.not_between(a, b) if negate else c.between(a, b)
                (probe_leaves if ref[0] == 0 else build_leaves).append(leaf)
                tag = "notbetween" if negate else "between"
                shape.append(f"{ref}:{tag}:{'?' if ref[0] == 0 else (a, b)}")
            else:
                op = p.take()
                if op[0] != "op" or op[1] not in ("=", "<>", "!=", "<", "<=", ">", ">="):
                    raise SqlError("42601", f"syntax error at or near {op[1]!r}")
                if p.peek()[0] == "id":
                    other = p.colref()
                    if op[1] != "=" or other[0] == ref[0] or join_eq is not None:
                        raise SqlError("0A000", "only one equi-join condition between the two tables")
                    join_eq = (ref, other) if ref[0] == 0 else (other, ref)
                    shape.append(f"join:{join_eq}")
                else:
                    v = p.number()
                    c = Col(ref[1])
                    leaf = {"=": c == v, "<>": c != v, "!=": c != v, "<": c < v, "<=": c <= v, ">": c > v,
                            ">=": c >= v}[op[1]]
                    (probe_leaves if ref[0] == 0 else build_leaves).append(leaf)
                    shape.append(f"{ref}:{op[1]}:{'?' if ref[0] == 0 else v}")
            if not p.accept("kw", "and"):
                break
        if p.peek() == ("kw", "or"):
            raise SqlError("0A000", "OR in WHERE is not supported by the wire front-end")

    group = []
    if p.accept("kw", "group"):
        p.expect("kw", "by")
        while True:
            group.append(p.colref())
            if not p.accept("op", ","):
                break
    order = None
    limit = None
    if p.accept("kw", "order"):
        p.expect("kw", "by")
        order_pos = p.number()
        desc = p.accept("kw", "desc")
        if not desc:
            p.accept("kw", "asc")
        p.expect("kw", "limit")
        limit = p.number()
        order = (order_pos, desc)
    if p.peek()[0] != "eof":
        raise SqlError("42601", f"syntax error at or near {p.peek()[1]!r}")

    if len(p.tables) == 2 and join_eq is None:
        raise SqlError("0A000", "two tables need an equi-join condition")
    if build_leaves and len(p.tables) < 2:
        raise SqlError("42601", "conditions on a second table without a join")

    keys = tuple(p.column(g) for g in group)
    key_ids = {(g[0], g[1]): i for i, g in enumerate(group)}
    aggs, items = [], []
    for kind, what, label in raw:
        if kind == "col":
            ref = p.resolve_deferred(*what)
            if ref not in key_ids:
                raise SqlError("42803", f'column "{ref[1]}" must appear in the GROUP BY clause')
            items.append(SelectItem("key", key_ids[ref], label))
        else:
            fn, term = what
            a = {"count*": lambda t: count_star(), "sum": sum_, "avg": avg, "min": min_, "max": max_,
                 "count": count_col}[fn](term)
            items.append(SelectItem("agg", len(aggs), label))
            aggs.append(a)
    if not aggs:
        raise SqlError("0A000", "a statement without aggregates")
    order_spec = None
    if order is not None:
        pos, desc = order
        if not (1 <= pos <= len(items)) or items[pos - 1].kind != "agg":
            raise SqlError("0A000", "ORDER BY takes the position of an aggregate in the select list")
        order_spec = (items[pos - 1].index, desc)

    def conj(leaves):
        w = None
        for leaf in leaves:
            w = leaf if w is None else w & leaf
        return w

    join = None
    if join_eq is not None:
        probe_ref, build_ref = join_eq
        join = (p.tables[1].name, build_ref[1], probe_ref[1], conj(build_leaves))
    spec = QuerySpec(table=p.tables[0].name, where=conj(probe_leaves), group_by=keys, aggs=aggs, items=items,
                     join=join, order=order_spec, limit=limit)
    # The shape: the statement with the probe-side literals blanked.
    spec.shape = repr((spec.table, [t.name for t in p.tables], shape, group,
                       [(r[0], repr(r[1]) if r[0] == "col" else (r[1][0], _term_sig(r[1][1]))) for r in raw],
                       order_spec, limit))
    return spec


def _term_sig(term) -> str:
    if term is None:
        return "*"
    return repr([(f.column, f.mul, f.add, f.side) for f in term.factors])


def format_rows(spec: QuerySpec, out) -> tuple[list[str], list[tuple]]:
    """Column names and text rows of a result in select-list order: group key
    values, exact integer aggregates, AVG as the f64 quotient (the reference
    returns AVG as a float, aggregate.rs:1416-1424)."""
    from . import _capi as A
    names = [it.name for it in spec.items]
    rows = []
    for k, vals in zip(out.keys, out.values):
        row = []
        for it in spec.items:
            if it.kind == "key":
                row.append(str(k[it.index]))
            else:
                v = vals[it.index]
                row.append(repr(float(v.as_f64)) if spec.aggs[it.index].func == A.AGG_AVG else str(v.value))
        rows.append(tuple(row))
    return names, rows
