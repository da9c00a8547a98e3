"""oxb_filter_project_noalloc: filter + projection into caller buffers with
its scratch in a static device array.  Each case runs the existing entry
point (oxb_filter_project) and the allocation-free one on the same batch,
twice in a row, and requires the same rows bit for bit; two cases also hold
them against the oracle, one at exactly the row limit.  The file is named
to be collected last, so it also runs after every other GPU test has used
the device."""
import ctypes as C

import numpy as np
import pyarrow as pa
import pytest

from compare import assert_batches_equal
from oxidelake_b200 import _abi
from oxidelake_b200.errors import Execution, Unsupported
from oxidelake_b200.params import Comparison as Cmp
from oxidelake_b200.params import Literal, and_, compare

pytestmark = pytest.mark.gpu


def _batch(n, seed, vector=False):
    rng = np.random.default_rng(seed)
    k = pa.array(rng.integers(-50, 50, n), pa.int64(), mask=rng.random(n) < 0.1)
    v = pa.array(rng.normal(0, 10, n), pa.float64(), mask=rng.random(n) < 0.05)
    q = pa.array(rng.integers(0, 100, n, dtype=np.int32))
    cols, names = [k, v, q], ["k", "v", "q"]
    if vector:
        flat = pa.array(rng.normal(0, 1, n * 3).astype(np.float32))
        cols.append(pa.FixedSizeListArray.from_arrays(flat, 3))
        names.append("e")
    return pa.RecordBatch.from_arrays(cols, names=names)


def _run_noalloc(backend, stream, dev, batch, pred, projection, capacity):
    """Allocates the output buffers (the caller's, not the call's), runs the
    allocation-free entry point and returns the rows as a record batch."""
    bufs, vals, valid, descs = [], [], [], []
    for p in projection:
        d = dev.column(p)
        width = 4 * d.dim if d.type == _abi.TYPE_VECTOR_F32 else (8 if d.type in (_abi.TYPE_INT64, _abi.TYPE_FLOAT64) else 4)
        vb = backend.alloc_device(max(8, capacity * width))
        bufs.append(vb)
        vals.append(vb.device_ptr())
        if d.validity:
            bb = backend.alloc_device(max(4, (capacity + 31) // 32 * 4))
            bufs.append(bb)
            valid.append(bb.device_ptr())
        else:
            valid.append(None)
    rows = backend.filter_project_noalloc(stream, dev, pred, projection, vals, valid, capacity)
    for i, p in enumerate(projection):
        d = dev.column(p)
        descs.append(_abi.Column(d.type, d.dim, rows, vals[i], valid[i] or 0))
    schema = pa.schema([batch.schema.field(p) for p in projection])
    view = backend.batch_from_device(schema, descs, rows, keep=bufs)
    return backend.download(stream, view)


def _existing(backend, stream, dev, pred, projection):
    return backend.download(stream, backend.filter_project(stream, dev, pred, projection))


CASES = [
    (3_000_000, and_(compare(0, Cmp.GtEq, Literal.int64(-10)), compare(1, Cmp.Lt, Literal.float64(4.0))), [2, 0, 1]),
    (1_000, compare(2, Cmp.Gt, Literal.int32(60)), [1, 3, 0]),
    (70_000, compare(1, Cmp.GtEq, Literal.float64(-0.0)), [0, 2]),
]


@pytest.mark.parametrize("n,pred,projection", CASES, ids=["3M", "1K-vector", "70K"])
def test_same_rows_as_filter_project_two_calls_in_a_row(backend, stream, n, pred, projection):
    vector = 3 in projection
    for call in range(2):
        batch = _batch(n, seed=100 * n + call, vector=vector)
        dev = backend.upload(stream, batch)
        want = _existing(backend, stream, dev, pred, projection)
        got = _run_noalloc(backend, stream, dev, batch, pred, projection, capacity=n)
        assert got.num_rows == want.num_rows
        assert_batches_equal(got, want)


def test_large_then_small_reuses_the_scratch(backend, stream):
    """A small call after a large one reads none of the large call's words."""
    pred = compare(0, Cmp.Lt, Literal.int64(0))
    for n, seed in ((2_500_000, 1), (333, 2), (2_500_000, 3)):
        batch = _batch(n, seed)
        dev = backend.upload(stream, batch)
        want = _existing(backend, stream, dev, pred, [0, 1, 2])
        got = _run_noalloc(backend, stream, dev, batch, pred, [0, 1, 2], capacity=n)
        assert_batches_equal(got, want)


def test_empty_input_and_empty_selection(backend, stream):
    for n, pred in ((0, None), (5_000, compare(2, Cmp.Gt, Literal.int32(1000)))):
        batch = _batch(n, 9)
        dev = backend.upload(stream, batch)
        got = _run_noalloc(backend, stream, dev, batch, pred, [0, 1], capacity=max(n, 1))
        assert got.num_rows == 0


def test_capacity_too_small_reports_the_count(backend, stream):
    batch = _batch(10_000, 4)
    dev = backend.upload(stream, batch)
    want = _existing(backend, stream, dev, None, [0])
    with pytest.raises(Execution):
        _run_noalloc(backend, stream, dev, batch, None, [0], capacity=100)
    assert backend.last_noalloc_rows == want.num_rows == 10_000


def test_rejects_more_rows_than_the_scratch_holds(backend, stream):
    n = _abi.OXB_NOALLOC_MAX_ROWS + 1
    batch = pa.RecordBatch.from_arrays([pa.array(np.zeros(n, dtype=np.int32))], names=["q"])
    dev = backend.upload(stream, batch)
    buf = backend.alloc_device(4)
    with pytest.raises(Unsupported):
        backend.filter_project_noalloc(stream, dev, None, [0], [buf.device_ptr()], [None], 1)


def test_exactly_the_maximum_rows_against_the_oracle(backend, stream):
    """An input of exactly OXB_NOALLOC_MAX_ROWS rows fills the static mask,
    tile counts and scan partials to the last word: the rows equal the
    oracle's filter_project (cpu/kernels.rs:144-152) and the existing entry
    point's, on two calls in a row."""
    import oracle
    from oxidelake_b200.params import leaves

    n = _abi.OXB_NOALLOC_MAX_ROWS
    pred = and_(compare(0, Cmp.GtEq, Literal.int64(-30)), compare(2, Cmp.Lt, Literal.int32(71)))
    projection = [1, 2, 0]
    for call in range(2):
        batch = _batch(n, seed=500 + call)
        dev = backend.upload(stream, batch)
        got = _run_noalloc(backend, stream, dev, batch, pred, projection, capacity=n)
        want = oracle.filter_project(batch, leaves(pred), projection)
        assert got.num_rows == want.num_rows > n // 3
        assert_batches_equal(got, want)
        assert_batches_equal(got, _existing(backend, stream, dev, pred, projection))
        del dev


def test_vector_projection_against_the_oracle(backend, stream):
    import oracle
    from oxidelake_b200.params import leaves

    pred = compare(1, Cmp.Lt, Literal.float64(2.5))
    for call in range(2):
        batch = _batch(123_457, seed=900 + call, vector=True)
        dev = backend.upload(stream, batch)
        got = _run_noalloc(backend, stream, dev, batch, pred, [3, 1], capacity=batch.num_rows)
        assert_batches_equal(got, oracle.filter_project(batch, leaves(pred), [3, 1]))
