"""CudaBackend: the reference's object-safe GpuBackend trait over liboxb200.

Method for method crates/oxidelake-device/src/backend.rs:44-198, arguments
as crates/oxidelake-device/src/args.rs:10-86, handles as
crates/oxidelake-device/src/handles.rs (DeviceBatch, DeviceJoinTable,
DeviceJoinMatches), errors as crates/oxidelake-core/src/error.rs.  Every
operator runs on the device through the C ABI; none falls back to the CPU.
Host data crosses as Arrow (pyarrow) record batches in the transfer format
of columns.py.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np
import pyarrow as pa

from . import _abi, columns
from .errors import Plan, Unsupported
from .params import AggregateFunction, AggregateSpec, DistanceMetric, Predicate, leaves

_L = _abi.lib


def _release(fn: str, handle) -> None:
    """Frees a handle from a finaliser.  At interpreter exit the module state
    may already be gone; the process then returns every resource itself."""
    try:
        getattr(_L(), fn)(handle)
    except Exception:
        pass


@dataclass
class MemoryInfo:
    """backend.rs:18-33."""

    total_bytes: int
    free_bytes: int
    pinned_supported: bool

    def used_bytes(self) -> int:
        return max(0, self.total_bytes - self.free_bytes)


class DeviceStream:
    """An execution stream (backend.rs:62)."""

    def __init__(self, backend: "CudaBackend", handle: int):
        self._backend = backend
        self.handle = handle

    def cuda_handle(self) -> int:
        return _L().oxb_stream_cuda_handle(self.handle) or 0

    def __del__(self):
        h, self.handle = getattr(self, "handle", None), None
        if h:
            _release("oxb_stream_destroy", h)


class DeviceBuffer:
    def __init__(self, handle: int):
        self.handle = handle

    def device_ptr(self) -> int:
        return _L().oxb_buffer_device_ptr(self.handle)

    def __len__(self) -> int:
        return _L().oxb_buffer_len(self.handle)

    def __del__(self):
        h, self.handle = getattr(self, "handle", None), None
        if h:
            _release("oxb_buffer_free", h)


class HostBuffer:
    def __init__(self, handle: int):
        self.handle = handle

    def is_pinned(self) -> bool:
        return bool(_L().oxb_host_buffer_is_pinned(self.handle))

    def view(self) -> np.ndarray:
        n = _L().oxb_host_buffer_len(self.handle)
        ptr = _L().oxb_host_buffer_ptr(self.handle)
        return np.ctypeslib.as_array((C.c_uint8 * n).from_address(ptr)) if n else np.zeros(0, np.uint8)

    def __del__(self):
        h, self.handle = getattr(self, "handle", None), None
        if h:
            _release("oxb_host_buffer_free", h)


class DeviceBatch:
    """handles.rs:130: a batch resident on the device, with its Arrow schema."""

    def __init__(self, handle: int, schema: pa.Schema, keep=None):
        self.handle = handle
        self.schema = schema
        self._keep = keep  # host or device memory the batch borrows

    def num_rows(self) -> int:
        return _L().oxb_batch_num_rows(self.handle)

    def num_columns(self) -> int:
        return _L().oxb_batch_num_columns(self.handle)

    def column(self, i: int) -> _abi.Column:
        c = _abi.Column()
        _abi.check(_L().oxb_batch_column(self.handle, i, C.byref(c)))
        return c

    def free(self) -> None:
        h, self.handle = getattr(self, "handle", None), None
        if h:
            _release("oxb_batch_free", h)

    def __del__(self):
        self.free()


class DeviceJoinTable:
    """handles.rs:224: a prepared build side."""

    def __init__(self, handle: int, build: DeviceBatch):
        self.handle = handle
        self.build = build

    def distinct_keys(self) -> int:
        return _L().oxb_join_table_distinct_keys(self.handle)

    def rows(self) -> int:
        return _L().oxb_join_table_rows(self.handle)

    def __del__(self):
        h, self.handle = getattr(self, "handle", None), None
        if h:
            _release("oxb_join_table_free", h)


class VectorIndex:
    """The BF16 copy of a vector column that vector_topk scans."""

    def __init__(self, handle: int, input: "DeviceBatch"):
        self.handle = handle
        self._input = input

    def __del__(self):
        h, self.handle = getattr(self, "handle", None), None
        if h:
            _release("oxb_vector_index_free", h)


class DeviceJoinMatches:
    """handles.rs:303: one probe batch's matches."""

    def __init__(self, handle: int, table: DeviceJoinTable):
        self.handle = handle
        self.table = table

    def __len__(self) -> int:
        return int(_L().oxb_join_matches_len(self.handle))

    def len(self) -> int:
        return len(self)

    def probe_rows(self) -> int:
        return _L().oxb_join_matches_probe_rows(self.handle)

    def __del__(self):
        h, self.handle = getattr(self, "handle", None), None
        if h:
            _release("oxb_join_matches_free", h)


def _leaf_array(pred: Optional[Predicate]) -> Tuple[Optional[C.Array], int]:
    lfs = leaves(pred)
    if not lfs:
        return None, 0
    arr = (_abi.Leaf * len(lfs))()
    for i, lf in enumerate(lfs):
        arr[i].column = lf.column
        arr[i].op = int(lf.op)
        arr[i].lit_type = int(lf.literal.type)
        if lf.literal.type == 2:
            arr[i].lit.f = float(lf.literal.value)
        else:
            arr[i].lit.i = int(lf.literal.value)
    return arr, len(lfs)


def _i32_array(vals: Sequence[int]):
    arr = (C.c_int32 * max(1, len(vals)))(*vals)
    return arr


def aggregate_output_schema(schema: pa.Schema, spec: AggregateSpec) -> pa.Schema:
    """crates/oxidelake-compute/src/exec/aggregate.rs:35-66: the key, then
    `FUNC(column)` per aggregate; SUM(Int*) -> Int64, SUM(Float64) ->
    Float64, COUNT -> Int64, MIN/MAX keep the type, AVG -> Float64."""
    key = schema.field(spec.group_by)
    fields = [pa.field(key.name, key.type, True)]
    for func, idx in spec.aggregates:
        func = AggregateFunction(func)
        if func == AggregateFunction.CountStar:
            fields.append(pa.field("COUNT(*)", pa.int64(), True))
            continue
        f = schema.field(idx)
        if func == AggregateFunction.Count:
            t = pa.int64()
        elif func == AggregateFunction.Sum:
            t = pa.float64() if pa.types.is_float64(f.type) else pa.int64()
        elif func == AggregateFunction.Avg:
            t = pa.float64()
        else:
            t = f.type
        fields.append(pa.field(f"{func.sql_name()}({f.name})", t, True))
    return pa.schema(fields)


class CudaBackend:
    """crates/oxidelake-device/src/cuda/mod.rs:247 (CudaBackend) behind the
    GpuBackend trait, on liboxb200 instead of NVRTC-compiled kernels."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _abi.check(_L().oxb_backend_create(device, C.byref(h)))
        self.handle = h.value
        self._default_stream: Optional[DeviceStream] = None

    def __del__(self):
        h, self.handle = getattr(self, "handle", None), None
        self._default_stream = None
        if h:
            _release("oxb_backend_destroy", h)

    # --- identity and memory (backend.rs:45-59) ---------------------------
    def kind(self) -> str:
        return _L().oxb_backend_kind(self.handle).decode()

    def device_id(self) -> int:
        return _L().oxb_backend_device_id(self.handle)

    def memory_info(self) -> MemoryInfo:
        m = _abi.MemoryInfo()
        _abi.check(_L().oxb_memory_info_get(self.handle, C.byref(m)))
        return MemoryInfo(m.total_bytes, m.free_bytes, bool(m.pinned_supported))

    def alloc_device(self, nbytes: int) -> DeviceBuffer:
        h = C.c_void_p()
        _abi.check(_L().oxb_alloc_device(self.handle, nbytes, C.byref(h)))
        return DeviceBuffer(h.value)

    def alloc_pinned_host(self, nbytes: int) -> HostBuffer:
        h = C.c_void_p()
        _abi.check(_L().oxb_alloc_pinned_host(self.handle, nbytes, C.byref(h)))
        return HostBuffer(h.value)

    # --- streams and transfers (backend.rs:62-81) -------------------------
    def create_stream(self) -> DeviceStream:
        h = C.c_void_p()
        _abi.check(_L().oxb_stream_create(self.handle, C.byref(h)))
        return DeviceStream(self, h.value)

    def wrap_stream(self, cuda_stream: int) -> DeviceStream:
        h = C.c_void_p()
        _abi.check(_L().oxb_stream_wrap(self.handle, C.c_void_p(cuda_stream), C.byref(h)))
        return DeviceStream(self, h.value)

    def default_stream(self) -> DeviceStream:
        if self._default_stream is None:
            self._default_stream = self.create_stream()
        return self._default_stream

    def copy_h2d(self, stream: DeviceStream, src: HostBuffer, dst: DeviceBuffer) -> None:
        _abi.check(_L().oxb_copy_h2d(self.handle, stream.handle, src.handle, dst.handle))

    def copy_d2h(self, stream: DeviceStream, src: DeviceBuffer, dst: HostBuffer) -> None:
        _abi.check(_L().oxb_copy_d2h(self.handle, stream.handle, src.handle, dst.handle))

    def synchronize(self, stream: DeviceStream) -> None:
        _abi.check(_L().oxb_stream_synchronize(self.handle, stream.handle))

    # --- batches (backend.rs:84-95) -----------------------------------------
    def upload(self, stream: DeviceStream, batch: pa.RecordBatch) -> DeviceBatch:
        cols = [columns.extract(batch.column(i)) for i in range(batch.num_columns)]
        desc = (_abi.Column * max(1, len(cols)))(*[c.descriptor() for c in cols])
        h = C.c_void_p()
        _abi.check(_L().oxb_upload(self.handle, stream.handle, desc, len(cols), batch.num_rows, C.byref(h)))
        self.synchronize(stream)  # the host buffers may go once the copies are done
        return DeviceBatch(h.value, batch.schema)

    def upload_arrow(self, stream: DeviceStream, batch: pa.RecordBatch) -> DeviceBatch:
        """upload through the Arrow C data interface (oxb_import_arrow): the
        batch is exported as a struct array and its buffers are read in
        place, offsets included.  On an error the exported structs are
        released here and the error raised."""
        arr, sch = _abi.ArrowArray(), _abi.ArrowSchema()
        batch._export_to_c(C.addressof(arr), C.addressof(sch))
        h = C.c_void_p()
        st = _L().oxb_import_arrow(self.handle, stream.handle, C.byref(arr), C.byref(sch), C.byref(h))
        if st != 0:
            for x in (arr, sch):
                if x.release:
                    x.release(C.byref(x))
            _abi.check(st)
        return DeviceBatch(h.value, batch.schema)

    def download_arrow(self, stream: DeviceStream, batch: DeviceBatch) -> pa.RecordBatch:
        """download through the Arrow C data interface (oxb_export_arrow),
        imported by pyarrow without a copy."""
        names = [f.name.encode() for f in batch.schema]
        carr = (C.c_char_p * max(1, len(names)))(*names)
        arr, sch = _abi.ArrowArray(), _abi.ArrowSchema()
        _abi.check(_L().oxb_export_arrow(self.handle, stream.handle, batch.handle, carr, C.byref(arr), C.byref(sch)))
        out = pa.RecordBatch._import_from_c(C.addressof(arr), C.addressof(sch))
        return out.cast(batch.schema) if out.schema != batch.schema else out

    def batch_from_device(self, schema: pa.Schema, descs: List[_abi.Column], rows: int, keep=None) -> DeviceBatch:
        """A batch over columns already in device memory (no copy)."""
        arr = (_abi.Column * max(1, len(descs)))(*descs)
        h = C.c_void_p()
        _abi.check(_L().oxb_batch_from_device(self.handle, arr, len(descs), rows, C.byref(h)))
        return DeviceBatch(h.value, schema, keep=keep)

    def download(self, stream: DeviceStream, batch: DeviceBatch) -> pa.RecordBatch:
        """backend.rs:91-95: every column into host memory, one call and one
        stream synchronization (oxb_download)."""
        ncols = len(batch.schema)
        vals, bits, lens = [], [], []
        for i in range(ncols):
            c = batch.column(i)
            n = c.length
            lens.append(n)
            vals.append(np.empty(n * (c.dim if c.type == _abi.TYPE_VECTOR_F32 else 1), dtype=columns.numpy_dtype(c.type)))
            bits.append(np.empty((n + 7) // 8, dtype=np.uint8))
        k = max(1, ncols)
        vp = (C.c_void_p * k)(*[v.ctypes.data if v.size else None for v in vals])
        bp = (C.c_void_p * k)(*[b.ctypes.data if b.size else None for b in bits])
        has = (C.c_int32 * k)()
        _abi.check(_L().oxb_download(self.handle, stream.handle, batch.handle, ncols, vp, bp, has))
        arrays = []
        for i, field in enumerate(batch.schema):
            n = lens[i]
            arrays.append(columns.rebuild(field.type, vals[i], bits[i] if has[i] and n else None, n))
        return pa.RecordBatch.from_arrays(arrays, schema=batch.schema)

    def download_column(self, stream: DeviceStream, batch: DeviceBatch, i: int) -> pa.Array:
        """One column (oxb_download_column)."""
        c = batch.column(i)
        n = c.length
        values = np.empty(n * (c.dim if c.type == _abi.TYPE_VECTOR_F32 else 1), dtype=columns.numpy_dtype(c.type))
        validity = np.empty((n + 7) // 8, dtype=np.uint8)
        has = C.c_int32(0)
        _abi.check(_L().oxb_download_column(self.handle, stream.handle, batch.handle, i,
                                            values.ctypes.data if n else None, validity.ctypes.data if n else None,
                                            C.byref(has)))
        return columns.rebuild(batch.schema.field(i).type, values, validity if has.value and n else None, n)

    # --- operators ----------------------------------------------------------
    def filter_project(
        self, stream: DeviceStream, input: DeviceBatch, predicate: Optional[Predicate], projection: Sequence[int]
    ) -> DeviceBatch:
        """backend.rs:98 with FilterProjectArgs (args.rs:10-15)."""
        lv, nl = _leaf_array(predicate)
        proj = _i32_array(projection)
        a = _abi.FilterProjectArgs(input.handle, lv, nl, proj, len(projection))
        h = C.c_void_p()
        _abi.check(_L().oxb_filter_project(self.handle, stream.handle, C.byref(a), C.byref(h)))
        for p in projection:
            if not 0 <= p < len(input.schema):
                raise Plan(f"projection index {p} out of range")
        return DeviceBatch(h.value, pa.schema([input.schema.field(p) for p in projection]))

    def filter_project_noalloc(
        self,
        stream: DeviceStream,
        input: DeviceBatch,
        predicate: Optional[Predicate],
        projection: Sequence[int],
        out_values: Sequence[int],
        out_validity: Sequence[Optional[int]],
        capacity: int,
    ) -> int:
        """filter_project into caller-owned device buffers (addresses in
        out_values / out_validity, one per projected column), allocating
        nothing; returns the selected row count.  No reference counterpart:
        the C header states the buffer sizes, the row limit and the
        sharing rule."""
        lv, nl = _leaf_array(predicate)
        proj = _i32_array(projection)
        a = _abi.FilterProjectArgs(input.handle, lv, nl, proj, len(projection))
        vals = (C.c_void_p * max(1, len(projection)))(*[C.c_void_p(v) for v in out_values])
        valid = (C.c_void_p * max(1, len(projection)))(*[C.c_void_p(v or 0) for v in out_validity])
        rows = C.c_int64(0)
        status = _L().oxb_filter_project_noalloc(
            self.handle, stream.handle, C.byref(a), vals, valid, capacity, C.byref(rows)
        )
        self.last_noalloc_rows = rows.value
        _abi.check(status)
        return rows.value

    def prepare_join_build(
        self, stream: DeviceStream, build: DeviceBatch, key: int, index=None
    ) -> DeviceJoinTable:
        """backend.rs:129 with JoinBuildArgs (args.rs:21-30).  `index` is the
        host's JoinTable as (keys, starts, counts, rows) numpy arrays, or None
        to index the build side on the device."""
        ix_ptr = None
        keep = None
        if index is not None:
            keys, starts, counts, rows = (
                np.ascontiguousarray(index[0], dtype=np.int64),
                np.ascontiguousarray(index[1], dtype=np.uint32),
                np.ascontiguousarray(index[2], dtype=np.uint32),
                np.ascontiguousarray(index[3], dtype=np.uint32),
            )
            keep = (keys, starts, counts, rows)
            ix = _abi.JoinIndex(
                keys.ctypes.data_as(C.POINTER(C.c_int64)),
                starts.ctypes.data_as(C.POINTER(C.c_uint32)),
                counts.ctypes.data_as(C.POINTER(C.c_uint32)),
                len(keys),
                rows.ctypes.data_as(C.POINTER(C.c_uint32)),
                len(rows),
            )
            ix_ptr = C.pointer(ix)
        a = _abi.JoinBuildArgs(build.handle, key, 0, ix_ptr)
        h = C.c_void_p()
        _abi.check(_L().oxb_prepare_join_build(self.handle, stream.handle, C.byref(a), C.byref(h)))
        del keep
        return DeviceJoinTable(h.value, build)

    def probe_join(self, stream: DeviceStream, probe: DeviceBatch, key: int, table: DeviceJoinTable) -> DeviceJoinMatches:
        """backend.rs:153 with JoinProbeArgs (args.rs:34-41)."""
        a = _abi.JoinProbeArgs(probe.handle, key, 0, table.handle)
        h = C.c_void_p()
        _abi.check(_L().oxb_probe_join(self.handle, stream.handle, C.byref(a), C.byref(h)))
        return DeviceJoinMatches(h.value, table)

    def hash_join(
        self,
        stream: DeviceStream,
        left: DeviceBatch,
        right: DeviceBatch,
        table: DeviceJoinTable,
        matches: DeviceJoinMatches,
        first: int,
        rows: int,
        projection: Optional[Sequence[int]] = None,
    ) -> DeviceBatch:
        """backend.rs:114 with HashJoinArgs (args.rs:45-60)."""
        proj = _i32_array(projection) if projection is not None else None
        a = _abi.HashJoinArgs(
            left.handle,
            right.handle,
            table.handle,
            matches.handle,
            first,
            rows,
            proj,
            len(projection) if projection is not None else 0,
            0,
        )
        h = C.c_void_p()
        _abi.check(_L().oxb_hash_join(self.handle, stream.handle, C.byref(a), C.byref(h)))
        fields = list(left.schema) + list(right.schema)
        sel = list(projection) if projection is not None else list(range(len(fields)))
        return DeviceBatch(h.value, pa.schema([fields[i] for i in sel]))

    def aggregate(
        self, stream: DeviceStream, input: DeviceBatch, spec: AggregateSpec, predicate: Optional[Predicate] = None
    ) -> DeviceBatch:
        """backend.rs:166 with AggregateArgs (args.rs:64-69); an optional WHERE
        is fused in (filter_project then aggregate, in one pass)."""
        if len(spec.aggregates) > _abi.OXB_MAX_AGGREGATES:
            raise Unsupported("too many aggregates")
        cs = _abi.AggregateSpecC()
        cs.group_by = spec.group_by
        cs.naggregates = len(spec.aggregates)
        for j, (f, c) in enumerate(spec.aggregates):
            cs.funcs[j] = int(f)
            cs.columns[j] = int(c)
        lv, nl = _leaf_array(predicate)
        a = _abi.AggregateArgs(input.handle, C.pointer(cs), lv, nl, 0)
        h = C.c_void_p()
        _abi.check(_L().oxb_aggregate(self.handle, stream.handle, C.byref(a), C.byref(h)))
        return DeviceBatch(h.value, aggregate_output_schema(input.schema, spec))

    def aggregate_batches(
        self,
        stream: DeviceStream,
        inputs: Sequence[DeviceBatch],
        spec: AggregateSpec,
        predicate: Optional[Predicate] = None,
    ) -> DeviceBatch:
        """Every batch of one input partition folded into one result in one
        persistent launch (GpuAggregateExec, compute/src/exec/aggregate.rs)."""
        if not inputs:
            raise Plan("no input batches")
        if len(spec.aggregates) > _abi.OXB_MAX_AGGREGATES:
            raise Unsupported("too many aggregates")
        cs = _abi.AggregateSpecC()
        cs.group_by = spec.group_by
        cs.naggregates = len(spec.aggregates)
        for j, (f, c) in enumerate(spec.aggregates):
            cs.funcs[j] = int(f)
            cs.columns[j] = int(c)
        lv, nl = _leaf_array(predicate)
        handles = (C.c_void_p * len(inputs))(*[b.handle for b in inputs])
        a = _abi.AggregateBatchesArgs(
            C.cast(handles, C.c_void_p), len(inputs), 0, C.cast(C.pointer(cs), C.c_void_p),
            C.cast(lv, C.c_void_p) if lv is not None else None, nl, 0,
        )
        h = C.c_void_p()
        _abi.check(_L().oxb_aggregate_batches(self.handle, stream.handle, C.byref(a), C.byref(h)))
        return DeviceBatch(h.value, aggregate_output_schema(inputs[0].schema, spec))

    def join_aggregate(
        self,
        stream: DeviceStream,
        probe: DeviceBatch,
        probe_key: int,
        table: DeviceJoinTable,
        predicate: Optional[Predicate],
        group: Tuple[int, int],
        aggregates: Sequence[Tuple[AggregateFunction, int, int]],
    ) -> DeviceBatch:
        """The fused probe -> WHERE -> GROUP BY pass (no reference counterpart;
        equals GpuHashJoinExec followed by the aggregate).  `group` and each
        aggregate name a side (0 probe, 1 build) and a column."""
        a, schema, keep = _join_aggregate_args(probe, probe_key, table, predicate, group, aggregates)
        h = C.c_void_p()
        _abi.check(_L().oxb_join_aggregate(self.handle, stream.handle, C.byref(a), C.byref(h)))
        return DeviceBatch(h.value, schema)

    def join_aggregate_many(self, stream: DeviceStream, requests) -> List[DeviceBatch]:
        """Several join_aggregate requests, each (probe, probe_key, table,
        predicate, group, aggregates), in one launch where they share a shape
        (oxb_join_aggregate_many); results in request order."""
        built = [_join_aggregate_args(*r) for r in requests]
        arr = (_abi.JoinAggregateArgs * max(1, len(built)))(*[x[0] for x in built])
        outs = (C.c_void_p * max(1, len(built)))()
        _abi.check(_L().oxb_join_aggregate_many(self.handle, stream.handle, arr, len(built), outs))
        return [DeviceBatch(outs[i], built[i][1]) for i in range(len(built))]

    def server(self, memory_budget: int = 0, workers: int = 0, max_batch: int = 0) -> "Server":
        """A serving loop over resident tables (oxb_server_create)."""
        return Server(self, memory_budget, workers, max_batch)

    def vector_distance(
        self,
        stream: DeviceStream,
        input: DeviceBatch,
        column: int,
        query: Sequence[float],
        metric: DistanceMetric,
        output_name: str,
    ) -> DeviceBatch:
        """backend.rs:173 with VectorDistanceArgs (args.rs:72-84)."""
        q = np.ascontiguousarray(np.asarray(query, dtype=np.float32))
        a = _abi.VectorDistanceArgs(input.handle, column, int(metric), q.ctypes.data_as(C.POINTER(C.c_float)), len(q), 0)
        h = C.c_void_p()
        _abi.check(_L().oxb_vector_distance(self.handle, stream.handle, C.byref(a), C.byref(h)))
        schema = input.schema.append(pa.field(output_name, pa.float32(), True))
        return DeviceBatch(h.value, schema)

    # --- instrumentation ----------------------------------------------------------
    def vector_index(self, stream: DeviceStream, input: DeviceBatch, column: int) -> "VectorIndex":
        """A resident BF16 copy of a vector column for vector_topk (the batch
        must outlive it)."""
        h = C.c_void_p()
        _abi.check(_L().oxb_vector_index_build(self.handle, stream.handle, input.handle, column, C.byref(h)))
        return VectorIndex(h.value, input)

    def vector_topk(
        self,
        stream: DeviceStream,
        index: "VectorIndex",
        input: DeviceBatch,
        predicate: Optional[Predicate],
        queries,
        k: int,
        metric: DistanceMetric,
        overfetch: int = 0,
        exact: bool = False,
        query_leaf=None,
    ):
        """ORDER BY distance, row LIMIT k per query over the rows `predicate`
        keeps: (ids int64 [Q, k], dist float32 [Q, k], stats dict).
        `query_leaf` = (column, Comparison, literals): query q also needs
        `column op literals[q]` (Literal objects of one type)."""
        q = np.ascontiguousarray(np.asarray(queries, dtype=np.float32))
        if q.ndim != 2:
            raise Plan("queries must be a 2-D array")
        lv, nl = _leaf_array(predicate)
        nq, dim = q.shape
        qcol, qop, qtype, qlits = -1, 0, 0, None
        if query_leaf is not None:
            qcol, cmp, lits = query_leaf
            if len(lits) != nq:
                raise Plan("one literal per query")
            qop, qtype = int(cmp), int(lits[0].type)
            raw = [
                int(np.float64(l.value).view(np.int64)) if int(l.type) == 2 else int(l.value) for l in lits
            ]
            qlits = np.ascontiguousarray(raw, dtype=np.int64)
        a = _abi.VectorTopkArgs(
            index.handle, input.handle, C.cast(lv, C.c_void_p) if lv is not None else None, nl, nq,
            q.ctypes.data, dim, k, int(metric), overfetch, 1 if exact else 0, qcol, qop, qtype, 0,
            qlits.ctypes.data if qlits is not None else None,
        )
        ids = np.empty((max(nq, 1), k), np.int64)
        dist = np.empty((max(nq, 1), k), np.float32)
        st = _abi.VectorTopkStats()
        _abi.check(
            _L().oxb_vector_topk(self.handle, stream.handle, C.byref(a), ids.ctypes.data, dist.ctypes.data, C.byref(st))
        )
        stats = {
            "reranked": st.reranked,
            "exact_queries": st.exact_queries,
            "max_score_error": st.max_score_error,
            "mean_score_error": st.mean_score_error,
        }
        return ids[:nq], dist[:nq], stats

    def set_kernel_timing(self, enabled: bool) -> None:
        _abi.check(_L().oxb_set_kernel_timing(self.handle, 1 if enabled else 0))

    def last_kernel_time(self) -> Tuple[str, float]:
        """(name, milliseconds) of the last operator's main kernel on this
        thread, timed with CUDA events on its stream."""
        buf = C.create_string_buffer(64)
        ms = C.c_float(0.0)
        _abi.check(_L().oxb_last_kernel_time(self.handle, buf, 64, C.byref(ms)))
        return buf.value.decode(), ms.value

    @staticmethod
    def last_call_stats() -> dict:
        """The counters of the last operator or transfer call on this thread
        (oxb_last_call_stats): what OperatorStats::record_batch and
        record_transfer take (core/src/telemetry.rs:140-152)."""
        st = _abi.CallStats()
        _abi.check(_L().oxb_last_call_stats(C.byref(st)))
        return {f: getattr(st, f) for f, _ in _abi.CallStats._fields_}

    def operator_stats(self, op: int, reset: bool = False) -> dict:
        """This backend's totals for one operator (oxb_operator_stats_get);
        fallback_batches is always 0: the library has no CPU path."""
        st = _abi.OperatorStats()
        _abi.check(_L().oxb_operator_stats_get(self.handle, int(op), C.byref(st), 1 if reset else 0))
        return {f: getattr(st, f) for f, _ in _abi.OperatorStats._fields_}

    def set_autotune(self, enabled: bool) -> None:
        """First call per query shape times every kernel variant and keeps the fastest."""
        _abi.check(_L().oxb_set_autotune(self.handle, 1 if enabled else 0))

    def set_upload_staging(self, threads: int) -> None:
        """Host threads that stage large pageable columns through page-locked
        chunks in upload (0: one driver copy per buffer)."""
        _abi.check(_L().oxb_set_upload_staging(self.handle, threads))

    def set_agg_variant(self, combine: int = -1, rows_per_thread: int = 0) -> None:
        """Pins the aggregation kernel variant (-1 / 0: automatic)."""
        _abi.check(_L().oxb_set_agg_variant(self.handle, combine, rows_per_thread))

    @staticmethod
    def kernel_launches() -> int:
        return int(_L().oxb_kernel_launches())

    # --- capability probes (backend.rs:182-197) -------------------------------
    def supports_predicate(self, predicate: Optional[Predicate]) -> bool:
        lv, nl = _leaf_array(predicate)
        return bool(_L().oxb_supports_predicate(self.handle, lv, nl))

    def supports_hash_join(self) -> bool:
        return bool(_L().oxb_supports_hash_join(self.handle))

    def supports_aggregate(self) -> bool:
        return bool(_L().oxb_supports_aggregate(self.handle))

def _join_aggregate_args(probe, probe_key, table, predicate, group, aggregates):
    """The C arguments of a join-aggregate, its output schema, and what must
    stay alive while the call reads them."""
    build = table.build
    a = _abi.JoinAggregateArgs()
    a.probe = probe.handle
    a.probe_key = probe_key
    a.table = table.handle
    a.build = build.handle
    lv, nl = _leaf_array(predicate)
    a.leaves = lv
    a.nleaves = nl
    a.group_side, a.group_column = group
    a.naggregates = len(aggregates)
    for j, (f, side, col) in enumerate(aggregates):
        a.funcs[j] = int(f)
        a.sides[j] = int(side)
        a.columns[j] = int(col)
    schemas = (probe.schema, build.schema)
    key = schemas[group[0]].field(group[1])
    fields = [pa.field(key.name, key.type, True)]
    for f, side, col in aggregates:
        f = AggregateFunction(f)
        if f == AggregateFunction.CountStar:
            fields.append(pa.field("COUNT(*)", pa.int64(), True))
            continue
        fld = schemas[side].field(col)
        if f == AggregateFunction.Count:
            t = pa.int64()
        elif f == AggregateFunction.Sum:
            t = pa.float64() if pa.types.is_float64(fld.type) else pa.int64()
        elif f == AggregateFunction.Avg:
            t = pa.float64()
        else:
            t = fld.type
        fields.append(pa.field(f"{f.sql_name()}({fld.name})", t, True))
    return a, pa.schema(fields), lv


class Server:
    """The serving loop (oxb_server_*): submit returns a ticket at once,
    worker threads run admitted work on their own streams, and top-k requests
    that differ only in query, k and per-query literal share a scan."""

    def __init__(self, backend: "CudaBackend", memory_budget: int = 0, workers: int = 0, max_batch: int = 0):
        self._backend = backend
        cfg = _abi.ServerConfig(memory_budget, workers, max_batch)
        h = C.c_void_p()
        _abi.check(_L().oxb_server_create(backend.handle, C.byref(cfg), C.byref(h)))
        self.handle = h.value
        self._schemas = {}

    def submit_topk(self, index, input, predicate, query, k: int, metric, query_leaf=None) -> int:
        """`query_leaf` = (column, Comparison, Literal): this query's own leaf,
        appended to `predicate`'s leaves."""
        lfs = list(leaves(predicate))
        if query_leaf is not None:
            from .params import Compare

            col, cmp, lit = query_leaf
            lfs.append(Compare(col, cmp, lit))
        arr = (_abi.Leaf * max(1, len(lfs)))()
        for i, lf in enumerate(lfs):
            arr[i].column = lf.column
            arr[i].op = int(lf.op)
            arr[i].lit_type = int(lf.literal.type)
            if int(lf.literal.type) == 2:
                arr[i].lit.f = float(lf.literal.value)
            else:
                arr[i].lit.i = int(lf.literal.value)
        q = np.ascontiguousarray(np.asarray(query, dtype=np.float32))
        r = _abi.TopkRequest(index.handle, input.handle, C.cast(arr, C.c_void_p), len(lfs),
                             1 if query_leaf is not None else 0, q.ctypes.data, q.size, k, int(metric), 0)
        t = C.c_uint64()
        _abi.check(_L().oxb_server_submit_topk(self.handle, C.byref(r), C.byref(t)))
        return t.value

    def submit_join_aggregate(self, probe, probe_key, table, predicate, group, aggregates) -> int:
        a, schema, keep = _join_aggregate_args(probe, probe_key, table, predicate, group, aggregates)
        t = C.c_uint64()
        _abi.check(_L().oxb_server_submit_join_aggregate(self.handle, C.byref(a), C.byref(t)))
        self._schemas[t.value] = schema
        return t.value

    def wait_topk(self, ticket: int, k: int):
        ids = np.empty(k, np.int64)
        dist = np.empty(k, np.float32)
        lat = C.c_double()
        _abi.check(_L().oxb_server_wait_topk(self.handle, ticket, ids.ctypes.data, dist.ctypes.data, C.byref(lat)))
        return ids, dist, lat.value

    def wait_batch(self, ticket: int):
        h = C.c_void_p()
        lat = C.c_double()
        schema = self._schemas.pop(ticket, None)
        _abi.check(_L().oxb_server_wait_batch(self.handle, ticket, C.byref(h), C.byref(lat)))
        return DeviceBatch(h.value, schema), lat.value

    def stats(self, reset: bool = False) -> dict:
        st = _abi.ServerStats()
        _abi.check(_L().oxb_server_stats_get(self.handle, C.byref(st), 1 if reset else 0))
        return {f: getattr(st, f) for f, _ in _abi.ServerStats._fields_}

    def close(self) -> None:
        h, self.handle = getattr(self, "handle", None), None
        if h:
            _release("oxb_server_destroy", h)

    def __del__(self):
        self.close()
