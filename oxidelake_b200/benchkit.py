"""Shared pieces of the measurement scripts: seeded synthetic inputs made on
the device, page-locked host copies of batches for end-to-end timing, and
the host copies of device batches that a checker reads.

Inputs made on the device keep a measurement run short at the configured
sizes (200M rows, 10M x 768 vectors); the generators are torch's seeded
device generators, so a run is repeatable.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np
import pyarrow as pa

from . import _abi, columns


def pinned_batch(backend, batch: pa.RecordBatch) -> Tuple[pa.RecordBatch, list]:
    """The batch with every column's values and validity copied into
    page-locked host memory; the second item keeps those buffers alive."""
    arrays, keep = [], []
    for i in range(batch.num_columns):
        cb = columns.extract(batch.column(i))
        bufs = []
        for part in (cb.validity, cb.values):
            if part is None:
                bufs.append(None)
                continue
            raw = np.ascontiguousarray(part).view(np.uint8).reshape(-1)
            hb = backend.alloc_pinned_host(max(1, raw.nbytes))
            hb.view()[: raw.nbytes] = raw
            keep.append(hb)
            bufs.append(pa.foreign_buffer(hb.view().ctypes.data, raw.nbytes, base=hb))
        dt = batch.schema.field(i).type
        n = cb.length
        if pa.types.is_fixed_size_list(dt):
            child = pa.Array.from_buffers(pa.float32(), n * dt.list_size, [None, bufs[1]])
            arrays.append(pa.Array.from_buffers(dt, n, [bufs[0]], children=[child]))
        else:
            arrays.append(pa.Array.from_buffers(dt, n, [bufs[0], bufs[1]]))
    return pa.RecordBatch.from_arrays(arrays, schema=batch.schema), keep


def batch_bytes(batch: pa.RecordBatch) -> int:
    """Bytes a batch's columns take in the transfer layout (values and
    validity bitmaps)."""
    return sum(columns.extract(batch.column(i)).total_bytes() for i in range(batch.num_columns))


def _pack_bits(valid):
    """A bool tensor (length a multiple of 8) as an LSB-first bitmap."""
    import torch

    w = torch.tensor([1, 2, 4, 8, 16, 32, 64, 128], dtype=torch.int32, device=valid.device)
    return (valid.view(-1, 8).to(torch.int32) * w).sum(dim=1).to(torch.uint8)


CONFIG3_SCHEMA = pa.schema([pa.field("g", pa.int64()), pa.field("x", pa.int32(), True), pa.field("f", pa.int32())])


def config3_sizes(total_rows: int, seed: int, min_rows: int = 8192, max_rows: int = 1 << 20) -> List[int]:
    """Seeded uneven batch sizes in [min_rows, max_rows] summing to total_rows."""
    rng = np.random.default_rng(seed)
    sizes, left = [], total_rows
    while left > 0:
        n = int(min(left, rng.integers(min_rows, max_rows + 1)))
        sizes.append(n)
        left -= n
    return sizes


def config3_device(backend, total_rows: int, distinct: int, seed: int = 0x0A11CE + 3, min_rows: int = 8192,
                   max_rows: int = 1 << 20):
    """The high-cardinality input made on the device, as uneven batches of
    8K-1M rows: g Int64 uniform over `distinct` values, x Int32
    U[-1e6, 1e6] with 2 % NULLs (a validity bitmap per batch), f Int32
    U[0, 100) (the WHERE column: `f < s` keeps s %).  Each column of each
    batch is its own allocation, so every column starts aligned."""
    import torch

    gen = torch.Generator(device="cuda").manual_seed(seed)
    out = []
    for n in config3_sizes(total_rows, seed, min_rows, max_rows):
        g = torch.randint(0, distinct, (n,), dtype=torch.int64, device="cuda", generator=gen)
        x = torch.randint(-1_000_000, 1_000_001, (n,), dtype=torch.int32, device="cuda", generator=gen)
        f = torch.randint(0, 100, (n,), dtype=torch.int32, device="cuda", generator=gen)
        padded = (n + 7) // 8 * 8
        valid = torch.rand(padded, device="cuda", generator=gen) >= 0.02
        valid[n:] = False
        bits = _pack_bits(valid)
        descs = [
            _abi.Column(_abi.TYPE_INT64, 1, n, g.data_ptr(), None),
            _abi.Column(_abi.TYPE_INT32, 1, n, x.data_ptr(), bits.data_ptr()),
            _abi.Column(_abi.TYPE_INT32, 1, n, f.data_ptr(), None),
        ]
        out.append(backend.batch_from_device(CONFIG3_SCHEMA, descs, n, keep=(g, x, f, bits)))
    return out


def host_copy(batch) -> pa.RecordBatch:
    """A device batch made by config3_device or vector_table, copied to host
    Arrow arrays through torch (the tensors the batch keeps)."""
    tensors = batch._keep
    n = batch.num_rows()
    arrays = []
    if batch.schema == CONFIG3_SCHEMA:
        g, x, f, bits = (t.cpu().numpy() for t in tensors)
        arrays = [
            pa.array(g),
            pa.Array.from_buffers(pa.int32(), n, [pa.py_buffer(bits), pa.py_buffer(x)]),
            pa.array(f),
        ]
        return pa.RecordBatch.from_arrays(arrays, schema=CONFIG3_SCHEMA)
    raise ValueError("not a batch this module made")


def vector_table(backend, rows: int, dim: int, seed: int, filter_hi: int):
    """N rows x dim FP32 ~ N(0,1), each row L2-normalised, and an Int64
    filter column uniform in [0, filter_hi), made on the device.  Returns the
    device batch (columns f, emb) and the two tensors."""
    import torch

    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.randn(rows, dim, device="cuda", generator=g)
    x /= x.norm(dim=1, keepdim=True)
    f = torch.randint(0, filter_hi, (rows,), device="cuda", generator=g, dtype=torch.int64)
    torch.cuda.synchronize()
    schema = pa.schema([pa.field("f", pa.int64()), pa.field("emb", pa.list_(pa.float32(), dim))])
    batch = backend.batch_from_device(
        schema,
        [_abi.Column(_abi.TYPE_INT64, 1, rows, f.data_ptr(), None),
         _abi.Column(_abi.TYPE_VECTOR_F32, dim, rows, x.data_ptr(), None)],
        rows, keep=(x, f),
    )
    return batch, x, f


def unit_queries(count: int, dim: int, seed: int) -> np.ndarray:
    """Queries from the table's distribution: N(0,1), L2-normalised."""
    q = np.random.default_rng(seed).standard_normal((count, dim)).astype(np.float32)
    q /= np.linalg.norm(q, axis=1, keepdims=True).astype(np.float32)
    return q


def percentile_ms(lat_s: Sequence[float], p: float) -> float:
    return float(np.percentile(np.asarray(lat_s) * 1e3, p)) if len(lat_s) else float("nan")
