"""CPU oracle for the GPU operator path — TEST INFRASTRUCTURE ONLY.

A restatement of the reference's CPU semantics
(crates/oxidelake-device/src/cpu/kernels.rs) in C (oracle.c, built by
oracle/Makefile) with this ctypes wrapper over Arrow record batches.  Only
tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py use it,
as the checker or as the timed stand-in for the reference's CPU path; the
product never imports it.

Parity pins: tests/test_oracle_golden.py checks this oracle against every
golden vector the reference's own tests hold for the path
(tests/golden/reference_vectors.json, made by tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path
from typing import Optional, Sequence, Tuple

import numpy as np
import pyarrow as pa

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboxb_oracle.so"

INT64, FLOAT64, INT32, FLOAT32, VECTOR_F32 = 1, 2, 3, 4, 5
SUM, COUNT, MIN, MAX, AVG, COUNT_STAR = 0, 1, 2, 3, 4, 5
L2, COSINE = 0, 1


class OracleError(Exception):
    def __init__(self, code: int, what: str):
        kind = {-1: "unsupported", -3: "execution", -4: "plan"}.get(code, "error")
        super().__init__(f"{kind}: {what}")
        self.code = code

    def is_unsupported(self) -> bool:
        return self.code == -1


class _Col(C.Structure):
    _fields_ = [("type", C.c_int32), ("dim", C.c_int32), ("length", C.c_int64), ("values", C.c_void_p), ("validity", C.c_void_p)]


class _Lit(C.Union):
    _fields_ = [("i", C.c_int64), ("f", C.c_double)]


class _Leaf(C.Structure):
    _fields_ = [("column", C.c_int32), ("op", C.c_int32), ("lit_type", C.c_int32), ("reserved", C.c_int32), ("lit", _Lit)]


class _Spec(C.Structure):
    _fields_ = [("group_by", C.c_int32), ("naggregates", C.c_int32), ("funcs", C.c_int32 * 16), ("columns", C.c_int32 * 16)]


class _JAQuery(C.Structure):
    _fields_ = [
        ("probe_key", C.c_int32),
        ("build_key", C.c_int32),
        ("group_side", C.c_int32),
        ("group_column", C.c_int32),
        ("naggregates", C.c_int32),
        ("funcs", C.c_int32 * 16),
        ("sides", C.c_int32 * 16),
        ("columns", C.c_int32 * 16),
    ]


def build() -> Path:
    """Compiles the oracle with its Makefile (gcc) when it is missing or stale."""
    src = [HERE / "oracle.c", HERE / "oracle.h"]
    if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < max(p.stat().st_mtime for p in src):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        l = C.CDLL(str(LIB_PATH))
        P, I32, I64, U32 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint32
        sig = {
            "orc_total_order_key": (I64, [C.c_double]),
            "orc_from_total_order_key": (C.c_double, [I64]),
            "orc_filter_order_key": (I64, [C.c_double]),
            "orc_slot_hash": (U32, [I64, U32]),
            "orc_l2": (C.c_float, [P, P, I64]),
            "orc_cosine": (C.c_float, [P, P, I64]),
            "orc_filter": (I64, [P, I32, P, I32, P]),
            "orc_join_build": (I32, [P, C.POINTER(P)]),
            "orc_join_free": (None, [P]),
            "orc_join_distinct": (I64, [P]),
            "orc_join_nrows": (I64, [P]),
            "orc_join_export": (None, [P, P, P, P, P]),
            "orc_join_probe": (I64, [P, P, P, P]),
            "orc_join_pairs": (I32, [P, P, P, I64, C.c_uint64, C.c_uint64, P, P]),
            "orc_agg_new": (I32, [P, I32, P, C.POINTER(P)]),
            "orc_agg_update": (I32, [P, P, I32, P, I32]),
            "orc_agg_merge": (I32, [P, P, I32]),
            "orc_agg_groups": (I64, [P]),
            "orc_agg_finish": (None, [P, P, P, P, P]),
            "orc_agg_free": (None, [P]),
            "orc_aggregate_parallel": (I32, [P, I32, P, P, I32, I32, C.POINTER(P)]),
            "orc_join_aggregate": (I32, [P, I32, P, I32, P, I32, P, I32, C.POINTER(P)]),
            "orc_vector_distance": (I32, [P, P, I32, P, P]),
            "orc_vector_topk": (I32, [P, I32, I32, P, I32, P, I32, I32, I32, I32, P, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


# ---------------------------------------------------------------- columns

def _bits(buf, offset: int, length: int) -> np.ndarray:
    raw = np.frombuffer(buf, dtype=np.uint8)
    bits = np.unpackbits(raw, bitorder="little")[offset : offset + length]
    return np.packbits(bits, bitorder="little")


class _Cols:
    """Arrow columns as oracle descriptors (buffers kept alive)."""

    def __init__(self, batch: pa.RecordBatch | Sequence[pa.Array]):
        arrays = [batch.column(i) for i in range(batch.num_columns)] if isinstance(batch, pa.RecordBatch) else list(batch)
        self.keep = []
        self.arr = (_Col * max(1, len(arrays)))()
        for i, a in enumerate(arrays):
            if isinstance(a, pa.ChunkedArray):
                a = a.combine_chunks()
            n = len(a)
            t = a.type
            dim = 1
            if pa.types.is_int64(t):
                code, vals = INT64, np.asarray(a.fill_null(0).to_numpy(zero_copy_only=False), dtype=np.int64)
            elif pa.types.is_float64(t):
                code, vals = FLOAT64, np.asarray(a.fill_null(0.0).to_numpy(zero_copy_only=False), dtype=np.float64)
            elif pa.types.is_int32(t):
                code, vals = INT32, np.asarray(a.fill_null(0).to_numpy(zero_copy_only=False), dtype=np.int32)
            elif pa.types.is_float32(t):
                code, vals = FLOAT32, np.asarray(a.fill_null(0.0).to_numpy(zero_copy_only=False), dtype=np.float32)
            elif pa.types.is_fixed_size_list(t):
                code, dim = VECTOR_F32, t.list_size
                child = a.values
                start = (a.offset + 0) * dim
                cbuf = child.buffers()[1]
                vals = np.frombuffer(cbuf, dtype=np.float32, count=n * dim, offset=(child.offset + start) * 4).copy() if n else np.zeros(0, np.float32)
            else:
                code, vals = 0, np.zeros(max(1, n), np.uint8)  # not readable by the oracle
            vals = np.ascontiguousarray(vals)
            valid = None
            if a.null_count > 0:
                valid = np.packbits(np.asarray(a.is_valid().to_numpy(zero_copy_only=False), dtype=bool), bitorder="little")
            self.keep.append((vals, valid))
            self.arr[i].type = code
            self.arr[i].dim = dim
            self.arr[i].length = n
            self.arr[i].values = vals.ctypes.data if n else None
            self.arr[i].validity = valid.ctypes.data if valid is not None else None
        self.n = len(arrays)

    def ptr(self):
        return C.cast(self.arr, C.c_void_p)


def _leaves(leaves) -> Tuple[object, int]:
    lst = list(leaves or [])
    arr = (_Leaf * max(1, len(lst)))()
    for i, lf in enumerate(lst):
        if isinstance(lf, tuple):
            col, op, lt, val = lf
        else:
            col, op, lt, val = lf.column, int(lf.op), int(lf.literal.type), lf.literal.value
        arr[i].column = col
        arr[i].op = int(op)
        arr[i].lit_type = int(lt)
        if int(lt) == FLOAT64:
            arr[i].lit.f = float(val)
        else:
            arr[i].lit.i = int(val)
    return arr, len(lst)


def _check(rc: int, what: str) -> None:
    if rc < 0:
        raise OracleError(rc, what)


# ---------------------------------------------------------------- scalars

def total_order_key(x: float) -> int:
    return lib().orc_total_order_key(x)


def from_total_order_key(k: int) -> float:
    return lib().orc_from_total_order_key(k)


def slot_hash(key: int, capacity: int) -> int:
    return lib().orc_slot_hash(key, capacity)


def l2(a, b) -> np.float32:
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    return np.float32(lib().orc_l2(a.ctypes.data, b.ctypes.data, len(a)))


def cosine(a, b) -> np.float32:
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    return np.float32(lib().orc_cosine(a.ctypes.data, b.ctypes.data, len(a)))


# ---------------------------------------------------------------- filter

def filter_rows(batch: pa.RecordBatch, leaves) -> np.ndarray:
    """evaluate_predicate + filter, cpu/kernels.rs:99-152: selected row ids."""
    cols = _Cols(batch)
    lv, nl = _leaves(leaves)
    out = np.zeros(max(1, batch.num_rows), dtype=np.uint32)
    k = lib().orc_filter(cols.ptr(), cols.n, lv, nl, out.ctypes.data)
    _check(k, "filter")
    return out[:k].copy()


def filter_project(batch: pa.RecordBatch, leaves, projection: Sequence[int]) -> pa.RecordBatch:
    rows = filter_rows(batch, leaves)
    return batch.select(list(projection)).take(pa.array(rows, type=pa.uint32()))


# ---------------------------------------------------------------- join

class JoinTable:
    """JoinTable, cpu/kernels.rs:185-266."""

    def __init__(self, build: pa.RecordBatch, key: int):
        self._cols = _Cols([build.column(key)])
        h = C.c_void_p()
        _check(lib().orc_join_build(self._cols.ptr(), C.byref(h)), "join build")
        self.h = h.value
        self.build = build

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_join_free(self.h)
            self.h = None

    def distinct_keys(self) -> int:
        return lib().orc_join_distinct(self.h)

    def rows(self) -> int:
        return lib().orc_join_nrows(self.h)

    def runs(self):
        """(keys, starts, counts, rows): JoinTable::runs + row_indices."""
        d, r = self.distinct_keys(), self.rows()
        keys = np.zeros(max(1, d), np.int64)
        starts = np.zeros(max(1, d), np.uint32)
        counts = np.zeros(max(1, d), np.uint32)
        rows = np.zeros(max(1, r), np.uint32)
        lib().orc_join_export(self.h, keys.ctypes.data, starts.ctypes.data, counts.ctypes.data, rows.ctypes.data)
        return keys[:d], starts[:d], counts[:d], rows[:r]


class JoinMatches:
    """JoinMatches, cpu/kernels.rs:303-407."""

    def __init__(self, left: pa.RecordBatch, key: int, table: JoinTable):
        cols = _Cols([left.column(key)])
        n = left.num_rows
        self.offsets = np.zeros(n + 1, np.uint64)
        self.starts = np.zeros(max(1, n), np.uint32)
        total = lib().orc_join_probe(table.h, cols.ptr(), self.offsets.ctypes.data, self.starts.ctypes.data)
        self.total = int(total)
        self.table = table
        self.n = n

    def __len__(self) -> int:
        return self.total

    def pairs(self, first: int, rows: int):
        if first < 0 or rows < 0 or first + rows > self.total:
            raise OracleError(-3, f"matches {first}..+{rows} are outside a probe with {self.total} matches")
        left = np.zeros(max(1, rows), np.uint32)
        right = np.zeros(max(1, rows), np.uint32)
        rc = lib().orc_join_pairs(
            self.table.h, self.offsets.ctypes.data, self.starts.ctypes.data, self.n, first, rows, left.ctypes.data, right.ctypes.data
        )
        _check(rc, "join pairs")
        return left[:rows], right[:rows]


def hash_join_gather(left, right, table, matches, first, rows, projection=None) -> pa.RecordBatch:
    """hash_join_gather, cpu/kernels.rs:414-472."""
    li, ri = matches.pairs(first, rows)
    fields = list(left.schema) + list(right.schema)
    width = left.num_columns
    sel = list(projection) if projection is not None else list(range(len(fields)))
    arrays = []
    for i in sel:
        if i < width:
            arrays.append(left.column(i).take(pa.array(li, type=pa.uint32())))
        else:
            arrays.append(right.column(i - width).take(pa.array(ri, type=pa.uint32())))
    return pa.RecordBatch.from_arrays(arrays, schema=pa.schema([fields[i] for i in sel]))


def hash_join(left, right, left_key, right_key, projection=None) -> pa.RecordBatch:
    t = JoinTable(right, right_key)
    m = JoinMatches(left, left_key, t)
    return hash_join_gather(left, right, t, m, 0, len(m), projection)


# ---------------------------------------------------------------- aggregate

def _out_type(func: int, dt: pa.DataType) -> pa.DataType:
    if func in (COUNT, COUNT_STAR):
        return pa.int64()
    if func == SUM:
        return pa.float64() if pa.types.is_float64(dt) else pa.int64()
    if func == AVG:
        return pa.float64()
    return dt


def _name(func: int, col: str) -> str:
    if func == COUNT_STAR:
        return "COUNT(*)"
    return f"{['SUM', 'COUNT', 'MIN', 'MAX', 'AVG'][func]}({col})"


class GroupedAggregator:
    """GroupedAggregator, cpu/kernels.rs:669-811."""

    def __init__(self, schema: pa.Schema, group_by: int, aggregates: Sequence[Tuple[int, int]]):
        self.schema = schema
        self.group_by = group_by
        self.aggs = [(int(f), int(c)) for f, c in aggregates]
        # a zero-row batch of the schema gives the oracle the types
        empty = pa.RecordBatch.from_arrays([pa.array([], type=f.type) for f in schema], schema=schema)
        cols = _Cols(empty)
        spec = _Spec()
        spec.group_by = group_by
        spec.naggregates = len(self.aggs)
        for j, (f, c) in enumerate(self.aggs):
            spec.funcs[j] = f
            spec.columns[j] = c
        h = C.c_void_p()
        _check(lib().orc_agg_new(cols.ptr(), cols.n, C.byref(spec), C.byref(h)), "aggregate")
        self.h = h.value

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_agg_free(self.h)
            self.h = None

    def update(self, batch: pa.RecordBatch, leaves=None) -> None:
        cols = _Cols(batch)
        lv, nl = _leaves(leaves)
        _check(lib().orc_agg_update(self.h, cols.ptr(), cols.n, lv, nl), "aggregate update")

    def merge(self, partial: pa.RecordBatch) -> None:
        cols = _Cols(partial)
        _check(lib().orc_agg_merge(self.h, cols.ptr(), cols.n), "aggregate merge")

    def groups(self) -> int:
        return lib().orc_agg_groups(self.h)

    def output_schema(self) -> pa.Schema:
        key = self.schema.field(self.group_by)
        fields = [pa.field(key.name, key.type, True)]
        for f, c in self.aggs:
            if f == COUNT_STAR:
                fields.append(pa.field("COUNT(*)", pa.int64(), True))
            else:
                fld = self.schema.field(c)
                fields.append(pa.field(_name(f, fld.name), _out_type(f, fld.type), True))
        return pa.schema(fields)

    def finish(self) -> pa.RecordBatch:
        return _finish(self.h, self.output_schema(), [f for f, _ in self.aggs])


def _finish(h, schema: pa.Schema, funcs) -> pa.RecordBatch:
    G = lib().orc_agg_groups(h)
    n = len(funcs)
    keys = np.zeros(max(1, G), np.int64)
    kvalid = np.zeros(max(1, G), np.uint8)
    vals = np.zeros(max(1, n * G), np.int64)
    valid = np.zeros(max(1, n * G), np.uint8)
    lib().orc_agg_finish(h, keys.ctypes.data, kvalid.ctypes.data, vals.ctypes.data, valid.ctypes.data)
    arrays = []
    kt = schema.field(0).type
    arrays.append(pa.array(keys[:G].astype(np.int32 if pa.types.is_int32(kt) else np.int64), type=kt, mask=kvalid[:G] == 0))
    for j, f in enumerate(funcs):
        t = schema.field(1 + j).type
        v = vals[j * G : (j + 1) * G]
        m = valid[j * G : (j + 1) * G] == 0
        if pa.types.is_float64(t):
            arr = pa.array(v.view(np.float64), type=t, mask=m)
        elif pa.types.is_int32(t):
            arr = pa.array(v.astype(np.int32), type=t, mask=m)
        else:
            arr = pa.array(v, type=t, mask=m)
        arrays.append(arr)
    return pa.RecordBatch.from_arrays(arrays, schema=schema)


def aggregate(batch: pa.RecordBatch, group_by: int, aggregates, leaves=None, threads: int = 1) -> pa.RecordBatch:
    """aggregate, cpu/kernels.rs:814-818 (with an optional WHERE first).
    threads > 1 splits the groups over threads by key hash, each folding its
    groups' rows in row order: the same bits as one thread, sooner."""
    g = GroupedAggregator(batch.schema, group_by, aggregates)
    if threads <= 1:
        g.update(batch, leaves)
        return g.finish()
    cols = _Cols(batch)
    lv, nl = _leaves(leaves)
    spec = _Spec()
    spec.group_by = group_by
    spec.naggregates = len(g.aggs)
    for j, (f, c) in enumerate(g.aggs):
        spec.funcs[j] = f
        spec.columns[j] = c
    h = C.c_void_p()
    _check(lib().orc_aggregate_parallel(cols.ptr(), cols.n, C.byref(spec), lv, nl, int(threads), C.byref(h)), "aggregate")
    try:
        return _finish(h.value, g.output_schema(), [f for f, _ in g.aggs])
    finally:
        lib().orc_agg_free(h.value)


def join_aggregate(
    probe: pa.RecordBatch,
    build: pa.RecordBatch,
    probe_key: int,
    build_key: int,
    leaves,
    group: Tuple[int, int],
    aggregates: Sequence[Tuple[int, int, int]],
    threads: int = 1,
) -> pa.RecordBatch:
    """probe JOIN build ... WHERE ... GROUP BY, as the reference's CPU path
    computes it (threads > 1: partitioned, partials merged in order)."""
    pc, bc = _Cols(probe), _Cols(build)
    lv, nl = _leaves(leaves)
    q = _JAQuery()
    q.probe_key, q.build_key = probe_key, build_key
    q.group_side, q.group_column = group
    q.naggregates = len(aggregates)
    for j, (f, side, col) in enumerate(aggregates):
        q.funcs[j], q.sides[j], q.columns[j] = int(f), int(side), int(col)
    h = C.c_void_p()
    _check(lib().orc_join_aggregate(pc.ptr(), pc.n, bc.ptr(), bc.n, lv, nl, C.byref(q), threads, C.byref(h)), "join aggregate")
    try:
        schemas = (probe.schema, build.schema)
        key = schemas[group[0]].field(group[1])
        fields = [pa.field(key.name, key.type, True)]
        for f, side, col in aggregates:
            if int(f) == COUNT_STAR:
                fields.append(pa.field("COUNT(*)", pa.int64(), True))
            else:
                fld = schemas[side].field(col)
                fields.append(pa.field(_name(int(f), fld.name), _out_type(int(f), fld.type), True))
        return _finish(h.value, pa.schema(fields), [int(f) for f, _, _ in aggregates])
    finally:
        lib().orc_agg_free(h.value)


# ---------------------------------------------------------------- vectors

def vector_distance(batch: pa.RecordBatch, column: int, query, metric: int) -> pa.Array:
    """vector_distance, cpu/kernels.rs:841-906: a Float32 column."""
    cols = _Cols([batch.column(column)])
    q = np.ascontiguousarray(query, dtype=np.float32)
    n = batch.num_rows
    out = np.zeros(max(1, n), np.float32)
    ok = np.zeros(max(1, n), np.uint8)
    _check(lib().orc_vector_distance(cols.ptr(), q.ctypes.data, int(metric), out.ctypes.data, ok.ctypes.data), "vector distance")
    return pa.array(out[:n], type=pa.float32(), mask=ok[:n] == 0)


def vector_topk(batch: pa.RecordBatch, column: int, queries: np.ndarray, k: int, metric: int, leaves=None, threads: int = 1):
    """ORDER BY distance, id LIMIT k per query: (ids int64 [Q, k], dist f32 [Q, k])."""
    cols = _Cols(batch)
    lv, nl = _leaves(leaves)
    q = np.ascontiguousarray(queries, dtype=np.float32)
    nq = q.shape[0]
    ids = np.zeros((max(1, nq), max(1, k)), np.int64)
    dist = np.zeros((max(1, nq), max(1, k)), np.float32)
    rc = lib().orc_vector_topk(cols.ptr(), cols.n, column, lv, nl, q.ctypes.data, nq, k, int(metric), threads, ids.ctypes.data, dist.ctypes.data)
    _check(rc, "vector topk")
    return ids[:nq, :k], dist[:nq, :k]


def cpu_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
