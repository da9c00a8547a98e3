"""Fused filter + projection on the B200 against the oracle
(cpu/kernels.rs:99-152 semantics): bit-exact rows, in row order."""
import json
import struct
from pathlib import Path

import numpy as np
import pyarrow as pa
import pytest

import oracle
from compare import assert_batches_equal
from datagen import conformance_left, demo_table, special_floats
from oxidelake_b200.errors import Plan, Unsupported
from oxidelake_b200.operator import GpuOperator
from oxidelake_b200.params import Comparison as Cmp
from oxidelake_b200.params import Literal, and_, compare, leaves

pytestmark = pytest.mark.gpu
G = json.loads((Path(__file__).parent / "golden" / "reference_vectors.json").read_text())


def fb(h):
    return struct.unpack("<d", struct.pack("<Q", int(h, 16)))[0]


def f64_array(hexes):
    vals = np.array([0 if h is None else int(h, 16) for h in hexes], dtype=np.uint64).view(np.float64)
    return pa.array(vals, pa.float64(), mask=np.array([h is None for h in hexes]))


def pred_from(spec):
    names = {"k": 0, "v": 1}
    p = None
    for c, op, v in spec:
        lit = Literal.int64(v) if c == "k" else Literal.float64(fb(v))
        leaf = compare(names[c], Cmp[op], lit)
        p = leaf if p is None else and_(p, leaf)
    return p


def test_golden_filter_drops_null_predicates_and_projects(backend):
    g = G["filter_drops_null_predicates_and_projects"]
    batch = pa.RecordBatch.from_arrays(
        [pa.array(g["k"], pa.int64()), f64_array(g["v"]), pa.array(g["s"], pa.utf8())], names=["k", "v", "s"]
    )
    p = and_(compare(0, Cmp.GtEq, Literal.int64(2)), compare(1, Cmp.Lt, Literal.float64(4.0)))
    op = GpuOperator(backend)
    out = op.filter_project(batch, p, g["projection"])
    assert out.schema.names == g["expect_names"]
    assert out.column(1).to_pylist() == g["expect_k"]
    assert out.column(0).to_pylist() == [None, "e"]
    assert op.stats.fallback_batches == 0 and op.stats.bytes_h2d > 0


def test_golden_float_comparisons(backend, stream):
    g = G["float_comparisons_order_as_datafusion_does"]
    batch = pa.RecordBatch.from_arrays([f64_array(g["values"]), pa.array(np.arange(7, dtype=np.int64))], names=["v", "i"])
    dev = backend.upload(stream, batch)
    for op, lit, want in g["cases"]:
        out = backend.download(stream, backend.filter_project(stream, dev, compare(0, Cmp[op], Literal.float64(fb(lit))), [1]))
        assert out.column(0).to_pylist() == want, (op, lit)


def test_golden_type_mismatch_is_unsupported(backend, stream):
    batch = pa.RecordBatch.from_arrays([pa.array([1, 2], pa.int64()), pa.array([1.0, 2.0])], names=["k", "v"])
    dev = backend.upload(stream, batch)
    with pytest.raises(Unsupported):
        backend.filter_project(stream, dev, compare(1, Cmp.Eq, Literal.int64(1)), [0])
    with pytest.raises(Plan):
        backend.filter_project(stream, dev, compare(5, Cmp.Eq, Literal.int64(1)), [0])
    with pytest.raises(Plan):
        backend.filter_project(stream, dev, None, [7])


@pytest.mark.parametrize("seed", G["special_float_filter_predicates"]["shapes"]["seeds"])
@pytest.mark.parametrize("rows", G["special_float_filter_predicates"]["shapes"]["sizes"])
def test_special_floats_filter_like_the_reference(backend, seed, rows):
    """conformance.rs:1492-1520 on the device."""
    batch = special_floats(seed, rows)
    op = GpuOperator(backend)
    for spec in G["special_float_filter_predicates"]["predicates"]:
        p = pred_from(spec)
        got = op.filter_project(batch, p, [2, 0, 1])
        want = oracle.filter_project(batch, leaves(p), [2, 0, 1])
        assert_batches_equal(got, want)
    assert op.stats.fallback_batches == 0


@pytest.mark.parametrize("seed", [1, 7, 42])
@pytest.mark.parametrize("rows", [0, 1, 7, 64, 1000, 70_001])
def test_conformance_shapes_with_vectors(backend, seed, rows):
    batch = conformance_left(seed, rows)
    op = GpuOperator(backend)
    for p in [
        compare(0, Cmp.GtEq, Literal.int64(2)),
        and_(compare(0, Cmp.GtEq, Literal.int64(2)), compare(1, Cmp.Lt, Literal.float64(4.0))),
        compare(1, Cmp.Eq, Literal.float64(2.25)),
        None,
    ]:
        got = op.filter_project(batch, p, [3, 0, 2, 1])
        want = oracle.filter_project(batch, leaves(p), [3, 0, 2, 1])
        assert_batches_equal(got, want)


def test_large_multi_leaf_int32_and_sliced_input(backend, stream):
    rng = np.random.default_rng(11)
    n = 3_000_017
    a = rng.integers(-1000, 1000, n).astype(np.int32)
    b = rng.standard_normal(n)
    c = rng.integers(0, 1 << 40, n)
    batch = pa.RecordBatch.from_arrays(
        [
            pa.array(a, pa.int32(), mask=rng.random(n) < 0.03),
            pa.array(b, pa.float64(), mask=rng.random(n) < 0.02),
            pa.array(c, pa.int64()),
            pa.FixedSizeListArray.from_arrays(pa.array(rng.standard_normal(n * 3).astype(np.float32)), 3),
        ],
        names=["a", "b", "c", "e"],
    )
    p = and_(
        and_(compare(0, Cmp.Gt, Literal.int32(-500)), compare(1, Cmp.LtEq, Literal.float64(0.7))),
        compare(2, Cmp.Lt, Literal.int64(1 << 39)),
    )
    for sl in (batch, batch.slice(13, n - 100)):
        dev = backend.upload(stream, sl)
        got = backend.download(stream, backend.filter_project(stream, dev, p, [3, 2, 1, 0]))
        want = oracle.filter_project(sl, leaves(p), [3, 2, 1, 0])
        assert_batches_equal(got, want)


def test_demo_table_filters(backend):
    batch = demo_table(65_536 + 1000, 42)
    op = GpuOperator(backend)
    p = and_(compare(1, Cmp.GtEq, Literal.int64(20)), compare(2, Cmp.Lt, Literal.float64(12.5)))
    got = op.filter_project(batch, p, [0, 3, 4, 2])
    want = oracle.filter_project(batch, leaves(p), [0, 3, 4, 2])
    assert_batches_equal(got, want)


def test_empty_and_all_rows(backend, stream):
    batch = pa.RecordBatch.from_arrays([pa.array([], pa.int64())], names=["k"])
    dev = backend.upload(stream, batch)
    out = backend.download(stream, backend.filter_project(stream, dev, compare(0, Cmp.Eq, Literal.int64(1)), [0]))
    assert out.num_rows == 0
    batch = pa.RecordBatch.from_arrays([pa.array(np.arange(5000, dtype=np.int64))], names=["k"])
    dev = backend.upload(stream, batch)
    out = backend.download(stream, backend.filter_project(stream, dev, None, [0, 0]))
    assert out.column(0).to_pylist() == list(range(5000)) == out.column(1).to_pylist()
