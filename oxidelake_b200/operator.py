"""GpuOperator: per-batch orchestration above the backend.

Mirrors crates/oxidelake-compute/src/operator.rs: only device-eligible
columns travel (``device_eligible`` / ``travels``, operator.rs:48-61); when a
projected column cannot (Utf8, ...), a row-id column travels instead and the
host gathers that column by row id after the download (``SidePlan``,
operator.rs:90-160).  The join is built once per operator (``JoinBuild``,
operator.rs:171-239) and its output is emitted in chunks of at most
``batch_size`` rows (``next_join_chunk``, operator.rs:752-814).  Telemetry
follows ``OperatorStats`` (crates/oxidelake-core/src/telemetry.rs:99-190).

Unlike the reference, there is no per-batch CPU fallback: a device error
fails the call (``fallback_batches`` stays 0).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Iterator, List, Optional, Sequence

import numpy as np
import pyarrow as pa

from .backend import CudaBackend, DeviceBatch, DeviceStream
from .columns import extract, is_device_eligible
from .errors import Plan
from .params import AggregateSpec, DistanceMetric, Predicate, columns as pred_columns

ROW_ID = "__oxb_row_id"


@dataclass
class OperatorStats:
    """telemetry.rs:99-190: what one operator did."""

    batches: int = 0
    rows_in: int = 0
    rows_out: int = 0
    bytes_h2d: int = 0
    bytes_d2h: int = 0
    fallback_batches: int = 0
    device_ns: int = 0
    latencies_ns: List[int] = field(default_factory=list)

    def record_batch(self, rows_in: int, rows_out: int, ns: int) -> None:
        self.batches += 1
        self.rows_in += rows_in
        self.rows_out += rows_out
        self.device_ns += ns
        self.latencies_ns.append(ns)

    def record_transfer(self, h2d: int, d2h: int) -> None:
        self.bytes_h2d += h2d
        self.bytes_d2h += d2h


def _batch_bytes(b: pa.RecordBatch) -> int:
    return sum(extract(b.column(i)).total_bytes() for i in range(b.num_columns))


class SidePlan:
    """Which columns of one side travel (operator.rs:90-160): the device
    sub-batch, and for each wanted column either its index in that sub-batch
    or 'host' (gathered by row id)."""

    def __init__(self, schema: pa.Schema, needed: Sequence[int], wanted: Sequence[int]):
        self.schema = schema
        travel = []
        for i in list(needed) + list(wanted):
            if is_device_eligible(schema.field(i).type) and i not in travel:
                travel.append(i)
        self.host_cols = [i for i in wanted if not is_device_eligible(schema.field(i).type)]
        self.needs_row_id = bool(self.host_cols)
        self.travel = travel
        self.position = {c: p for p, c in enumerate(travel)}
        if self.needs_row_id:
            self.row_id_pos = len(travel)

    def sub_batch(self, batch: pa.RecordBatch) -> pa.RecordBatch:
        arrays = [batch.column(i) for i in self.travel]
        names = [batch.schema.field(i).name for i in self.travel]
        if self.needs_row_id:
            arrays.append(pa.array(np.arange(batch.num_rows, dtype=np.int64)))
            names.append(ROW_ID)
        fields = [batch.schema.field(i) for i in self.travel]
        if self.needs_row_id:
            fields.append(pa.field(ROW_ID, pa.int64(), False))
        return pa.RecordBatch.from_arrays(arrays, schema=pa.schema(fields))


class GpuOperator:
    """operator.rs:439-449 over a CudaBackend."""

    def __init__(self, backend: CudaBackend, stats: Optional[OperatorStats] = None, batch_size: int = 65_536):
        self.backend = backend
        self.stream: DeviceStream = backend.create_stream()
        self.stats = stats or OperatorStats()
        self.batch_size = batch_size

    def _upload(self, b: pa.RecordBatch) -> DeviceBatch:
        self.stats.record_transfer(_batch_bytes(b), 0)
        return self.backend.upload(self.stream, b)

    def _download(self, d: DeviceBatch) -> pa.RecordBatch:
        out = self.backend.download(self.stream, d)
        self.stats.record_transfer(0, _batch_bytes(out) if out.num_rows else 0)
        return out

    # ---- filter + projection (operator.rs:603-705) -----------------------
    def filter_project(self, batch: pa.RecordBatch, predicate: Optional[Predicate], projection: Sequence[int]) -> pa.RecordBatch:
        t0 = time.perf_counter_ns()
        for p in projection:
            if not 0 <= p < batch.num_columns:
                raise Plan(f"projection index {p} out of range for a batch with {batch.num_columns} columns")
        plan = SidePlan(batch.schema, pred_columns(predicate) if predicate is not None else [], projection)
        sub = plan.sub_batch(batch)
        dev = self._upload(sub)
        remap = _remap(predicate, plan.position)
        dev_proj = [plan.position[p] for p in projection if p in plan.position]
        if plan.needs_row_id:
            dev_proj.append(plan.row_id_pos)
        out_dev = self.backend.filter_project(self.stream, dev, remap, dev_proj)
        got = self._download(out_dev)
        rows = got.column(len(dev_proj) - 1) if plan.needs_row_id else None
        arrays, fields = [], []
        k = 0
        for p in projection:
            if p in plan.position:
                arrays.append(got.column(k))
                k += 1
            else:
                arrays.append(batch.column(p).take(rows))
            fields.append(batch.schema.field(p))
        out = pa.RecordBatch.from_arrays(arrays, schema=pa.schema(fields))
        self.stats.record_batch(batch.num_rows, out.num_rows, time.perf_counter_ns() - t0)
        return out

    # ---- hash join (operator.rs:717-992) ------------------------------------
    def hash_join(
        self,
        probe: pa.RecordBatch,
        probe_key: int,
        build: pa.RecordBatch,
        build_key: int,
        projection: Optional[Sequence[int]] = None,
    ) -> Iterator[pa.RecordBatch]:
        """Inner join, probe columns ++ build columns (or `projection` of
        that), in chunks of at most `batch_size` rows."""
        width = probe.num_columns
        allcols = list(range(width + build.num_columns))
        sel = list(projection) if projection is not None else allcols
        lwant = [c for c in sel if c < width]
        rwant = [c - width for c in sel if c >= width]
        lplan = SidePlan(probe.schema, [probe_key], lwant)
        rplan = SidePlan(build.schema, [build_key], rwant)
        ldev = self._upload(lplan.sub_batch(probe))
        rdev = self._upload(rplan.sub_batch(build))
        table = self.backend.prepare_join_build(self.stream, rdev, rplan.position[build_key])
        matches = self.backend.probe_join(self.stream, ldev, lplan.position[probe_key], table)
        lw = len(lplan.travel) + (1 if lplan.needs_row_id else 0)
        dev_sel = [lplan.position[c] for c in lwant if c in lplan.position]
        dev_sel += [lplan.row_id_pos] if lplan.needs_row_id else []
        rsel = [lw + rplan.position[c] for c in rwant if c in rplan.position]
        rsel += [lw + rplan.row_id_pos] if rplan.needs_row_id else []
        total = len(matches)
        first = 0
        while first < total:
            t0 = time.perf_counter_ns()
            rows = min(self.batch_size, total - first)
            got = self._download(self.backend.hash_join(self.stream, ldev, rdev, table, matches, first, rows, dev_sel + rsel))
            lrows = got.column(len(dev_sel) - 1) if lplan.needs_row_id else None
            rrows = got.column(len(dev_sel) + len(rsel) - 1) if rplan.needs_row_id else None
            arrays, fields = [], []
            li = ri = 0
            for c in sel:
                if c < width:
                    if c in lplan.position:
                        arrays.append(got.column(dev_sel.index(lplan.position[c])))
                    else:
                        arrays.append(probe.column(c).take(lrows))
                    fields.append(probe.schema.field(c))
                else:
                    b = c - width
                    if b in rplan.position:
                        arrays.append(got.column(len(dev_sel) + rsel.index(lw + rplan.position[b])))
                    else:
                        arrays.append(build.column(b).take(rrows))
                    fields.append(build.schema.field(b))
            first += rows
            out = pa.RecordBatch.from_arrays(arrays, schema=pa.schema(fields))
            self.stats.record_batch(probe.num_rows if first == rows else 0, out.num_rows, time.perf_counter_ns() - t0)
            yield out

    # ---- aggregate (operator.rs:994-1075) -----------------------------------
    def aggregate(self, batch: pa.RecordBatch, spec: AggregateSpec, predicate: Optional[Predicate] = None) -> pa.RecordBatch:
        t0 = time.perf_counter_ns()
        needed = [spec.group_by] + [c for f, c in spec.aggregates if int(f) != 5]
        needed += pred_columns(predicate) if predicate is not None else []
        plan = SidePlan(batch.schema, needed, [])
        for c in needed:
            if c not in plan.position:
                from .errors import Unsupported

                raise Unsupported(f"column {c} of type {batch.schema.field(c).type} cannot be aggregated on the device")
        dev = self._upload(plan.sub_batch(batch))
        dspec = AggregateSpec(plan.position[spec.group_by], [(f, plan.position.get(c, 0)) for f, c in spec.aggregates])
        out = self._download(self.backend.aggregate(self.stream, dev, dspec, _remap(predicate, plan.position)))
        # Names follow the caller's schema, not the sub-batch's.
        from .backend import aggregate_output_schema

        out = pa.RecordBatch.from_arrays(out.columns, schema=aggregate_output_schema(batch.schema, spec))
        self.stats.record_batch(batch.num_rows, out.num_rows, time.perf_counter_ns() - t0)
        return out

    # ---- vector distance (operator.rs:1077-1144) -----------------------------
    def vector_distance(self, batch: pa.RecordBatch, column: int, query, metric: DistanceMetric, output_name: str) -> pa.RecordBatch:
        t0 = time.perf_counter_ns()
        sub = pa.RecordBatch.from_arrays([batch.column(column)], schema=pa.schema([batch.schema.field(column)]))
        dev = self._upload(sub)
        got = self._download(self.backend.vector_distance(self.stream, dev, 0, query, metric, output_name))
        out = pa.RecordBatch.from_arrays(list(batch.columns) + [got.column(1)], schema=batch.schema.append(got.schema.field(1)))
        self.stats.record_batch(batch.num_rows, out.num_rows, time.perf_counter_ns() - t0)
        return out


def _remap(predicate: Optional[Predicate], position) -> Optional[Predicate]:
    """The predicate over the sub-batch's column numbering."""
    from .params import And, Compare

    if predicate is None:
        return None
    if isinstance(predicate, Compare):
        return Compare(position[predicate.column], predicate.op, predicate.literal)
    return And(_remap(predicate.left, position), _remap(predicate.right, position))
