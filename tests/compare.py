"""Result comparison for the parity tests: bit-exact for integers, indices,
and any float the reference computes exactly; within a stated tolerance for
Float64 SUM/AVG: 1e-12 of max(|result|, sum of |inputs|) per group.  For
inputs of one sign that is 1e-12 relative to the result; where a group's
inputs cancel, the reference's own sequential sum is only that accurate, so
the bound is taken against the inputs' magnitude (the scale comes from the
oracle run on |x|).  The device sums themselves are held to 1e-12 relative
to the exact sum in test_gpu_aggregate.py.
"""
from __future__ import annotations

import numpy as np
import pyarrow as pa

FLOAT_SUM_RTOL = 1e-12


def _bits(arr: pa.Array) -> list:
    if isinstance(arr, pa.ChunkedArray):
        arr = arr.combine_chunks()
    valid = arr.is_valid().to_numpy(zero_copy_only=False)
    t = arr.type
    if pa.types.is_float64(t):
        v = arr.fill_null(0.0).to_numpy(zero_copy_only=False).view(np.uint64)
    elif pa.types.is_float32(t):
        v = arr.fill_null(0.0).to_numpy(zero_copy_only=False).view(np.uint32)
    elif pa.types.is_fixed_size_list(t):
        vals = arr.values.to_numpy(zero_copy_only=False).view(np.uint32)
        off = arr.offset * t.list_size
        v = [tuple(vals[off + i * t.list_size : off + (i + 1) * t.list_size]) for i in range(len(arr))]
        return [x if ok else None for x, ok in zip(v, valid)]
    else:
        return [x if ok else None for x, ok in zip(arr.to_pylist(), valid)]
    return [int(x) if ok else None for x, ok in zip(v, valid)]


def _primitive_equal(got: pa.Array, want: pa.Array, what: str) -> None:
    """Bit-exact comparison of two integer or float columns in numpy: the
    same validity, and the same value bits wherever a row is valid."""
    if isinstance(got, pa.ChunkedArray):
        got = got.combine_chunks()
    if isinstance(want, pa.ChunkedArray):
        want = want.combine_chunks()
    gv = got.is_valid().to_numpy(zero_copy_only=False)
    wv = want.is_valid().to_numpy(zero_copy_only=False)
    bad = gv != wv
    width = got.type.bit_width // 8
    view = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[width]
    zero = 0.0 if pa.types.is_floating(got.type) else 0
    g = got.fill_null(zero).to_numpy(zero_copy_only=False).view(view)
    w = want.fill_null(zero).to_numpy(zero_copy_only=False).view(view)
    bad |= gv & wv & (g != w)
    if bad.any():
        i = np.nonzero(bad)[0][:5]
        raise AssertionError(f"{what}: differs at rows {i.tolist()}: got {[got[j].as_py() for j in i]} "
                             f"want {[want[j].as_py() for j in i]}")


def assert_columns_equal(got: pa.Array, want: pa.Array, what: str = "") -> None:
    assert len(got) == len(want), f"{what}: {len(got)} rows, want {len(want)}"
    assert got.type == want.type, f"{what}: type {got.type}, want {want.type}"
    if pa.types.is_integer(got.type) or pa.types.is_floating(got.type):
        _primitive_equal(got, want, what)
        return
    g, w = _bits(got), _bits(want)
    if g != w:
        bad = [i for i, (a, b) in enumerate(zip(g, w)) if a != b][:5]
        raise AssertionError(f"{what}: differs at rows {bad}: got {[g[i] for i in bad]} want {[w[i] for i in bad]}")


def abs_columns(batch: pa.RecordBatch, cols) -> pa.RecordBatch:
    """The batch with the Float64 columns `cols` replaced by their |x|."""
    import pyarrow.compute as pc

    arrays = [pc.abs(batch.column(i)) if i in cols and pa.types.is_float64(batch.schema.field(i).type) else batch.column(i) for i in range(batch.num_columns)]
    return pa.RecordBatch.from_arrays(arrays, schema=batch.schema)


def assert_close_f64(got: pa.Array, want: pa.Array, what: str = "", rtol: float = FLOAT_SUM_RTOL, scale=None) -> None:
    assert len(got) == len(want), what
    gv = got.is_valid().to_numpy(zero_copy_only=False)
    wv = want.is_valid().to_numpy(zero_copy_only=False)
    assert (gv == wv).all(), f"{what}: validity differs"
    g = got.fill_null(0.0).to_numpy(zero_copy_only=False)
    w = want.fill_null(0.0).to_numpy(zero_copy_only=False)
    same_nan = np.isnan(g) & np.isnan(w)
    inf_eq = np.isinf(w) & (g == w)
    err = np.abs(g - w)
    mag = np.abs(w) if scale is None else np.maximum(np.abs(w), np.abs(scale))
    ok = same_nan | inf_eq | (err <= rtol * mag) | (g == w)
    if not ok.all():
        i = np.nonzero(~ok)[0][:5]
        raise AssertionError(f"{what}: rel err > {rtol} at {i.tolist()}: got {g[i]} want {w[i]}")


def assert_batches_equal(got: pa.RecordBatch, want: pa.RecordBatch, float_sum_cols=(), scale=None) -> None:
    """Bit-exact except the named Float64 SUM/AVG columns (1e-12 of the
    larger of |result| and, when `scale` is given, that column of `scale`:
    the same query over |x|)."""
    assert got.num_columns == want.num_columns, (got.schema, want.schema)
    assert got.num_rows == want.num_rows, (got.num_rows, want.num_rows)
    for i in range(want.num_columns):
        name = want.schema.field(i).name
        if i in float_sum_cols or name in float_sum_cols:
            sc = None
            if scale is not None:
                sc = scale.column(i).fill_null(0.0).to_numpy(zero_copy_only=False)
            assert_close_f64(got.column(i), want.column(i), name, scale=sc)
        else:
            assert_columns_equal(got.column(i), want.column(i), name)
