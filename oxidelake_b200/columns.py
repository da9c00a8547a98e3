"""Arrow column <-> device transfer format.

Mirrors crates/oxidelake-device/src/columns.rs: a column travels as its
values, tightly packed from row 0, plus an optional LSB-first validity bitmap
re-based to bit 0 (``extract``, columns.rs:192-251); ``rebuild``
(columns.rs:253-289) turns downloaded bytes back into an Arrow array.
Int64 / Float64 / Int32 / Float32 and FixedSizeList<Float32, n> travel;
anything else is ``Unsupported`` (columns.rs:51-80).  A NULL element inside a
valid vector row is refused (columns.rs:115-135, 226-235): the distance
kernels have no element validity.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np
import pyarrow as pa

from . import _abi
from .errors import Unsupported

_NP = {
    _abi.TYPE_INT64: np.int64,
    _abi.TYPE_FLOAT64: np.float64,
    _abi.TYPE_INT32: np.int32,
    _abi.TYPE_FLOAT32: np.float32,
    _abi.TYPE_VECTOR_F32: np.float32,
}


def type_code(dt: pa.DataType) -> tuple[int, int]:
    """(oxb_type, dim) of an Arrow type, or Unsupported."""
    if pa.types.is_int64(dt):
        return _abi.TYPE_INT64, 1
    if pa.types.is_float64(dt):
        return _abi.TYPE_FLOAT64, 1
    if pa.types.is_int32(dt):
        return _abi.TYPE_INT32, 1
    if pa.types.is_float32(dt):
        return _abi.TYPE_FLOAT32, 1
    if pa.types.is_fixed_size_list(dt) and pa.types.is_float32(dt.value_type) and dt.list_size > 0:
        return _abi.TYPE_VECTOR_F32, dt.list_size
    raise Unsupported(f"column type {dt} does not travel to the device")


def is_device_eligible(dt: pa.DataType) -> bool:
    """columns.rs:61 (plus Int32 and Float32)."""
    try:
        type_code(dt)
        return True
    except Unsupported:
        return False


def _rebase_bits(buf: pa.Buffer, offset: int, length: int) -> np.ndarray:
    raw = np.frombuffer(buf, dtype=np.uint8)
    if offset % 8 == 0:
        return raw[offset // 8 : offset // 8 + (length + 7) // 8].copy()
    bits = np.unpackbits(raw, bitorder="little")[offset : offset + length]
    return np.packbits(bits, bitorder="little")


@dataclass
class ColumnBytes:
    """columns.rs:28-40: values from row 0, validity re-based to bit 0."""

    type: int
    dim: int
    length: int
    values: np.ndarray
    validity: Optional[np.ndarray]

    def descriptor(self) -> _abi.Column:
        return _abi.Column(
            self.type,
            self.dim,
            self.length,
            self.values.ctypes.data if self.length else None,
            self.validity.ctypes.data if self.validity is not None else None,
        )

    def total_bytes(self) -> int:
        return self.values.nbytes + (self.validity.nbytes if self.validity is not None else 0)


def extract(array: pa.Array) -> ColumnBytes:
    """columns.rs:192-251."""
    if isinstance(array, pa.ChunkedArray):
        array = array.combine_chunks()
    code, dim = type_code(array.type)
    n = len(array)
    validity = None
    if array.null_count > 0:
        validity = _rebase_bits(array.buffers()[0], array.offset, n)
    if code == _abi.TYPE_VECTOR_F32:
        child = array.values  # the whole child, not offset-adjusted
        start = array.offset * dim
        if n and child.null_count > 0:
            cbits = _rebase_bits(child.buffers()[0], child.offset + start, n * dim) if child.buffers()[0] else None
            if cbits is not None:
                elem_ok = np.unpackbits(cbits, bitorder="little")[: n * dim].reshape(n, dim).all(axis=1)
                row_ok = (
                    np.unpackbits(validity, bitorder="little")[:n].astype(bool)
                    if validity is not None
                    else np.ones(n, dtype=bool)
                )
                bad = np.nonzero(row_ok & ~elem_ok)[0]
                if bad.size:
                    raise Unsupported(f"row {int(bad[0])} holds a NULL element inside a valid vector")
        buf = child.buffers()[1]
        values = np.frombuffer(buf, dtype=np.float32, count=n * dim, offset=(child.offset + start) * 4) if n else np.zeros(0, np.float32)
    else:
        dtype = _NP[code]
        buf = array.buffers()[1]
        width = np.dtype(dtype).itemsize
        values = np.frombuffer(buf, dtype=dtype, count=n, offset=array.offset * width) if n else np.zeros(0, dtype)
    return ColumnBytes(code, dim, n, np.ascontiguousarray(values), validity)


def rebuild(dt: pa.DataType, values: np.ndarray, validity: Optional[np.ndarray], length: int) -> pa.Array:
    """columns.rs:253-289."""
    vbuf = pa.py_buffer(validity) if validity is not None else None
    if pa.types.is_fixed_size_list(dt):
        child = pa.Array.from_buffers(pa.float32(), length * dt.list_size, [None, pa.py_buffer(values)])
        return pa.Array.from_buffers(dt, length, [vbuf], children=[child])
    return pa.Array.from_buffers(dt, length, [vbuf, pa.py_buffer(values)])


def numpy_dtype(code: int):
    return _NP[code]
