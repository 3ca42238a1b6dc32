"""SQL front end with the interface of VoxelVM's voxel_sql (reference
bindings/voxel_sql.py), executed on the B200 backend.

    import voxel_sql as vsql          # with voxel_b200/frontend on sys.path
    vsql.execute("SELECT SUM(price) FROM trades WHERE price > 500", data={"trades": prices})

The reference parses with pglast; this module has its own parser for the
statements the reference's compiler handles (SELECT with aggregates over one
table, WHERE comparisons joined by AND / OR, GROUP BY, ORDER BY, LIMIT,
subqueries and CSV paths in FROM) and gives them the reference's meaning
(voxel_sql.py:48-316):

* without GROUP BY the statement becomes a voxel_query: every WHERE
  comparison (>, >=, <, <=, =) becomes a filter on the table's column and, as
  in the query builder, only the last one applies; aggregates emit their
  loops (AVG emits SUM then COUNT, whose second loop never ends: VoxelError);
  ORDER BY returns the sort indices, LIMIT k the k largest values;
* with GROUP BY, WHERE is a row mask (all comparisons ANDed, whatever the
  boolean operator, and `=` meaning |x - v| < 1e-10), the group keys are the
  named data column (else row numbers), and the result is
  {"groups": <distinct keys>, "function": <aggregate name>}.

WHERE masks run on the GPU (VectorFilter kernels, bitmap AND), the group-by on
the GPU HashAggregator, the rest through voxel_query.
"""
from __future__ import annotations

import csv as _csv
import os as _os
import re as _re

import numpy as np

import voxel_query as _vq
from voxel_b200 import capi as _capi

_F64 = 0
_OPS = {">": 4, ">=": 5, "<": 2, "<=": 3}


# ---------------------------------------------------------------------------
# parsing
# ---------------------------------------------------------------------------
_TOKEN = _re.compile(r"""\s*(?:
    (?P<num>\d+\.\d*(?:[eE][-+]?\d+)?|\.\d+(?:[eE][-+]?\d+)?|\d+(?:[eE][-+]?\d+)?)
  | (?P<str>'(?:[^']|'')*')
  | (?P<qid>"(?:[^"]|"")*")
  | (?P<op><>|!=|>=|<=|[=<>(),*;.+-])
  | (?P<id>[A-Za-z_][A-Za-z_0-9$]*)
)""", _re.VERBOSE)

_KEYWORDS = {"select", "from", "where", "group", "by", "order", "limit", "and", "or", "not", "asc", "desc", "as",
             "insert", "delete", "update", "into", "values"}


def _tokenize(sql: str):
    toks, pos = [], 0
    sql = sql.strip()
    while pos < len(sql):
        m = _TOKEN.match(sql, pos)
        if not m or m.end() == pos:
            if sql[pos:].strip() == "":
                break
            raise ValueError(f"SQL syntax error near {sql[pos:pos + 20]!r}")
        pos = m.end()
        kind = m.lastgroup
        text = m.group(kind)
        if kind == "id" and text.lower() in _KEYWORDS:
            toks.append(("kw", text.lower()))
        else:
            toks.append((kind, text))
    return toks


class _Parser:
    def __init__(self, sql: str):
        self.t = _tokenize(sql)
        self.i = 0

    def peek(self, k=0):
        return self.t[self.i + k] if self.i + k < len(self.t) else (None, None)

    def take(self):
        tok = self.peek()
        self.i += 1
        return tok

    def accept(self, kind, text=None):
        k, v = self.peek()
        if k == kind and (text is None or v == text):
            self.i += 1
            return v
        return None

    def expect(self, kind, text=None):
        v = self.accept(kind, text)
        if v is None:
            raise ValueError(f"SQL syntax error: expected {text or kind}, got {self.peek()[1]!r}")
        return v

    def statement(self):
        k, v = self.peek()
        if k is None:
            raise ValueError("Empty SQL statement")
        if k == "kw" and v == "insert":
            raise NotImplementedError("INSERT not yet supported")
        if k == "kw" and v == "delete":
            raise NotImplementedError("DELETE not yet supported")
        if not (k == "kw" and v == "select"):
            raise NotImplementedError(f"Statement type {v} not supported")
        s = self.select()
        self.accept("op", ";")
        return s

    def select(self):
        self.expect("kw", "select")
        targets = [self.target()]
        while self.accept("op", ","):
            targets.append(self.target())
        sel = {"targets": targets, "from": None, "where": None, "group": None, "sort": None, "limit": None}
        if self.accept("kw", "from"):
            sel["from"] = self.from_item()
        if self.accept("kw", "where"):
            sel["where"] = self.bool_expr()
        if self.accept("kw", "group"):
            self.expect("kw", "by")
            cols = [self.column_name()]
            while self.accept("op", ","):
                cols.append(self.column_name())
            sel["group"] = cols
        if self.accept("kw", "order"):
            self.expect("kw", "by")
            self.operand()
            asc = True
            if self.accept("kw", "desc"):
                asc = False
            else:
                self.accept("kw", "asc")
            while self.accept("op", ","):
                self.operand()
                self.accept("kw", "asc") or self.accept("kw", "desc")
            sel["sort"] = asc
        if self.accept("kw", "limit"):
            sel["limit"] = self.operand()
        return sel

    def target(self):
        if self.accept("op", "*"):
            t = ("star",)
        else:
            t = self.operand()
        if self.accept("kw", "as"):
            self.take()
        elif self.peek()[0] == "id":
            self.take()  # a bare alias
        return t

    def from_item(self):
        if self.accept("op", "("):
            sub = self.select()
            self.expect("op", ")")
            self.accept("kw", "as")
            if self.peek()[0] == "id":
                self.take()
            return ("subquery", sub)
        k, v = self.take()
        if k == "str":
            name = v[1:-1].replace("''", "'")
        elif k == "qid":
            name = v[1:-1].replace('""', '"')
        elif k == "id":
            name = v
            while self.accept("op", "."):
                name = self.take()[1]  # schema-qualified: the relation name
        else:
            raise ValueError(f"Cannot resolve table: {v}")
        if self.peek()[0] == "id":
            self.take()  # alias
        return ("table", name)

    def column_name(self):
        k, v = self.take()
        if k == "id":
            while self.accept("op", "."):
                v = self.take()[1]
            return v
        if k == "qid":
            return v[1:-1]
        if k == "num":
            return None
        raise ValueError(f"SQL syntax error near {v!r}")

    def bool_expr(self):
        left = self.bool_term()
        args = [left]
        while self.accept("kw", "or"):
            args.append(self.bool_term())
        return ("bool", "or", args) if len(args) > 1 else left

    def bool_term(self):
        args = [self.bool_factor()]
        while self.accept("kw", "and"):
            args.append(self.bool_factor())
        return ("bool", "and", args) if len(args) > 1 else args[0]

    def bool_factor(self):
        if self.accept("kw", "not"):
            return ("bool", "not", [self.bool_factor()])
        if self.peek() == ("op", "(") and not self._is_subselect():
            self.take()
            e = self.bool_expr()
            self.expect("op", ")")
            return e
        left = self.operand()
        k, v = self.peek()
        if k == "op" and v in (">", ">=", "<", "<=", "=", "<>", "!="):
            self.take()
            right = self.operand()
            return ("cmp", "<>" if v == "!=" else v, left, right)
        return ("other", left)

    def _is_subselect(self):
        return self.peek(1) == ("kw", "select")

    def operand(self):
        k, v = self.peek()
        if k == "op" and v in ("-", "+"):
            self.take()
            o = self.operand()
            if o[0] == "const" and isinstance(o[1], float):
                return ("const", -o[1] if v == "-" else o[1])
            return o
        if k == "num":
            self.take()
            return ("const", float(v))
        if k == "str":
            self.take()
            return ("const", v[1:-1].replace("''", "'"))
        if k == "id" and self.peek(1) == ("op", "("):
            name = self.take()[1].lower()
            self.take()
            arg = None
            if self.accept("op", "*"):
                arg = ("star",)
            elif not self.accept("op", ")"):
                arg = self.operand()
                while self.accept("op", ","):
                    self.operand()
            else:
                return ("func", name, None)
            self.expect("op", ")")
            return ("func", name, arg)
        if k == "id" and v.lower() == "null":
            self.take()
            return ("const", None)
        if k in ("id", "qid"):
            return ("col", self.column_name())
        if k == "op" and v == "(":
            self.take()
            o = self.operand()
            self.expect("op", ")")
            return o
        raise ValueError(f"SQL syntax error near {v!r}")


# ---------------------------------------------------------------------------
# execution
# ---------------------------------------------------------------------------
def _f64_bits(x: float) -> int:
    return int(np.array([x], np.float64).view(np.uint64)[0])


class SqlCompiler:
    """Compiles the parsed statement onto VoxelVM queries and operators."""

    def __init__(self, data_sources=None):
        self._data = data_sources or {}
        self._columns = {}

    def execute(self, sql: str):
        stmt = _Parser(sql).statement()
        return self._compile_select(stmt)

    def _compile_select(self, sel):
        if sel["from"] is None:
            raise ValueError("FROM clause required")
        table = self._resolve_table(sel["from"])
        targets = sel["targets"]
        if sel["group"] is not None:
            return self._execute_group_by(table, sel["where"], sel["group"], targets)
        q = _vq.from_numpy(table)
        if sel["where"] is not None:
            self._compile_where(q, sel["where"])
        for t in targets:
            if t[0] == "func":
                self._compile_func(q, t[1])
        if sel["sort"] is not None:
            q.sort(ascending=sel["sort"])
        if sel["limit"] is not None:
            k = self._eval_const(sel["limit"])
            if k:
                q.topk(int(k), largest=True)
        return q.run()

    # WHERE as voxel_query filters (voxel_sql.py:217-239)
    def _compile_where(self, q, node):
        if node[0] == "cmp":
            _, op, left, right = node
            if self._column_of(left) is None:
                return
            val = self._eval_const(right)
            if op == ">":
                q.filter_gt(val)
            elif op == ">=":
                q.filter_ge(val)
            elif op == "<":
                q.filter_lt(val)
            elif op == "<=":
                q.filter_le(val)
            elif op == "=":
                q.filter_eq(val)
        elif node[0] == "bool":
            for arg in node[2]:
                self._compile_where(q, arg)

    def _compile_func(self, q, name):
        if name == "sum":
            q.sum()
        elif name == "count":
            q.count()
        elif name == "avg":
            q.sum()
            q.count()
        elif name == "min":
            q.min()
        elif name == "max":
            q.max()

    # GROUP BY (voxel_sql.py:87-148): a GPU row mask, GPU HashAggregator
    def _execute_group_by(self, table, where, group_cols, targets):
        table = np.ascontiguousarray(table, dtype=np.float64)
        offsets = None
        if where is not None:
            mask = self._where_mask(table, where)
            offsets = np.flatnonzero(mask)
            filtered = table[offsets]
        else:
            filtered = table
        agg_func = "sum"
        if targets and targets[0][0] == "func":
            agg_func = targets[0][1] or "sum"
        name = group_cols[0] if group_cols else None
        if name is not None and name in self._data:
            raw = np.asarray(self._data[name])
            keys = np.array(raw[offsets] if offsets is not None else raw, dtype=np.uint32)
        else:
            keys = np.arange(len(filtered), dtype=np.uint32)
        L = _capi.lib()
        agg = L.voxel_agg_create()
        try:
            L.voxel_agg_init(agg, max(128, int(len(keys) / 10) + 1))
            vals = np.ascontiguousarray(filtered, dtype=np.float64)
            L.voxel_agg_accumulate(agg, keys.ctypes.data, vals.ctypes.data, min(keys.size, vals.size))
            ngroups = int(L.voxel_agg_group_count(agg))
        finally:
            L.voxel_agg_destroy(agg)
        return {"groups": ngroups, "function": agg_func}

    def _where_mask(self, table, node):
        """Rows passing the WHERE clause: comparisons evaluated by the GPU's
        VectorFilter kernels, every boolean node taken as AND of its arguments
        (voxel_sql.py:118-146)."""
        n = table.size
        words = max((n + 63) // 64, 1)
        L = _capi.lib()

        def bitmap(nd):
            bm = np.zeros(words, np.uint64)
            if nd[0] == "cmp":
                _, op, _left, right = nd
                val = self._eval_const(right)
                if op in _OPS and isinstance(val, float):
                    L.voxel_vfilter(_F64, _OPS[op], table.ctypes.data, n, _f64_bits(val), 0, bm.ctypes.data)
                    return bm
                if op == "=" and isinstance(val, float):
                    # |x - v| < 1e-10 as the open interval around v
                    lo = np.nextafter(val - 1e-10, np.inf)
                    hi = np.nextafter(val + 1e-10, -np.inf)
                    L.voxel_vfilter(_F64, 6, table.ctypes.data, n, _f64_bits(lo), _f64_bits(hi), bm.ctypes.data)
                    return bm
            elif nd[0] == "bool":
                parts = [bitmap(a) for a in nd[2]]
                ptrs = (np.ctypeslib.ctypes.c_void_p * len(parts))(*[p.ctypes.data for p in parts])
                L.voxel_bitmap_and(ptrs, len(parts), n, bm.ctypes.data)
                return bm
            bm[:] = np.uint64(0xFFFFFFFFFFFFFFFF)
            if n % 64:
                bm[-1] = np.uint64((1 << (n % 64)) - 1)
            return bm

        bm = bitmap(node)
        return np.unpackbits(bm.view(np.uint8), bitorder="little")[:n].astype(bool)

    def _resolve_table(self, item):
        kind, val = item
        if kind == "subquery":
            return self._compile_select(val)
        name = val
        if name in self._data:
            v = self._data[name]
            return v.astype(np.float64) if isinstance(v, np.ndarray) else v
        path = name.strip("'\"")
        if _os.path.exists(path):
            return self._load_csv(path)
        if name in self._columns:
            return self._columns[name]
        raise ValueError(f"Cannot resolve table: {name}")

    @staticmethod
    def _load_csv(path):
        return load_csv(path, 0)

    @staticmethod
    def _column_of(node):
        if node[0] == "col":
            return node[1]
        if node[0] == "const":
            return node[1]
        return None

    @staticmethod
    def _eval_const(node):
        if node is None:
            return None
        if node[0] == "const":
            return node[1]
        return None


def execute(sql: str, data=None):
    """Execute SQL against VoxelVM on the GPU.  data: a dict of table / column
    name -> numpy array, or one array (the table "t").  Returns a float for
    aggregates, a dict for GROUP BY."""
    compiler = SqlCompiler(data if isinstance(data, dict) else {"t": data})
    return compiler.execute(sql)


def load_csv(path, column=0):
    """One CSV column (after the header row) as f64; unparsable cells skipped."""
    rows = []
    with open(path, "r") as f:
        reader = _csv.reader(f)
        next(reader, None)
        for row in reader:
            if row and column < len(row):
                try:
                    rows.append(float(row[column]))
                except ValueError:
                    pass
    return np.array(rows, dtype=np.float64)
