"""Vector distance on the B200: bit-exact with the reference's sequential
Float32 l2 / cosine (cpu/kernels.rs:909-927)."""
import json
import math
from pathlib import Path

import numpy as np
import pyarrow as pa
import pytest

import oracle
from compare import assert_columns_equal
from oxidelake_b200.errors import Plan, Unsupported
from oxidelake_b200.operator import GpuOperator
from oxidelake_b200.params import DistanceMetric

pytestmark = pytest.mark.gpu
G = json.loads((Path(__file__).parent / "golden" / "reference_vectors.json").read_text())


def test_golden_vector_distances(backend, stream):
    g = G["vector_distances"]
    vec = pa.FixedSizeListArray.from_arrays(pa.array(g["values"], pa.float32()), g["dim"], mask=pa.array([not v for v in g["valid"]]))
    batch = pa.RecordBatch.from_arrays([vec], names=["vec"])
    dev = backend.upload(stream, batch)
    out = backend.download(stream, backend.vector_distance(stream, dev, 0, g["query"], DistanceMetric.L2, "d"))
    d = out.column(1).to_pylist()
    assert d[0] == 0.0 and d[1] is None and np.float32(d[2]) == np.sqrt(np.float32(20.0))
    out = backend.download(stream, backend.vector_distance(stream, dev, 0, g["query"], DistanceMetric.Cosine, "d"))
    c = out.column(1).to_pylist()
    assert abs(c[0]) < 1e-6 and c[1] is None and abs(c[2] - (1 - 3 / 5)) < 1e-6
    with pytest.raises(Plan):
        backend.vector_distance(stream, dev, 0, [1.0], DistanceMetric.L2, "d")
    zero = pa.RecordBatch.from_arrays([pa.FixedSizeListArray.from_arrays(pa.array([0.0, 0.0], pa.float32()), 2)], names=["v"])
    out = backend.download(stream, backend.vector_distance(stream, backend.upload(stream, zero), 0, [1.0, 0.0], DistanceMetric.Cosine, "d"))
    assert math.isnan(out.column(1).to_pylist()[0])


@pytest.mark.parametrize("dim", [1, 4, 8, 33, 64, 65, 100, 768])
@pytest.mark.parametrize("metric", [DistanceMetric.L2, DistanceMetric.Cosine])
def test_bit_exact_against_the_sequential_reference(backend, stream, dim, metric):
    rng = np.random.default_rng(dim * 7 + int(metric))
    n = 20_011 if dim < 100 else 5_003
    vals = rng.standard_normal(n * dim).astype(np.float32)
    vals[:dim] = 0.0  # a zero-norm row: cosine NaN
    vec = pa.FixedSizeListArray.from_arrays(pa.array(vals), dim, mask=pa.array(rng.random(n) < 0.05))
    batch = pa.RecordBatch.from_arrays([vec, pa.array(np.arange(n, dtype=np.int64))], names=["e", "id"])
    q = rng.standard_normal(dim).astype(np.float32)
    op = GpuOperator(backend)
    got = op.vector_distance(batch, 0, q, metric, "d")
    want = oracle.vector_distance(batch, 0, q, int(metric))
    assert_columns_equal(got.column(2), want, f"dim={dim} {metric.name}")
    assert got.schema.field(2).name == "d" and got.column(1).to_pylist() == batch.column(1).to_pylist()


def test_null_element_in_a_valid_row_is_refused(backend, stream):
    child = pa.array([1.0, None, 3.0, 4.0], pa.float32())
    vec = pa.FixedSizeListArray.from_arrays(child, 2)
    with pytest.raises(Unsupported):
        backend.upload(stream, pa.RecordBatch.from_arrays([vec], names=["v"]))


@pytest.mark.parametrize("dim", [32, 132, 768])
@pytest.mark.parametrize("metric", [DistanceMetric.L2, DistanceMetric.Cosine])
def test_many_row_blocks_per_cta(backend, stream, dim, metric):
    """Enough rows that each CTA of the pipelined kernel (dim a multiple of
    4, at least 32) folds several 128-row blocks through its copy ring, and
    a ragged last block; bit-exact against the sequential reference."""
    rng = np.random.default_rng(dim + 3 * int(metric))
    n = 150_001 if dim < 768 else 60_013
    vals = rng.standard_normal(n * dim).astype(np.float32)
    vec = pa.FixedSizeListArray.from_arrays(pa.array(vals), dim, mask=pa.array(rng.random(n) < 0.01))
    batch = pa.RecordBatch.from_arrays([pa.array(np.arange(n)), vec], names=["id", "emb"])
    q = rng.standard_normal(dim).astype(np.float32)
    got = backend.download(stream, backend.vector_distance(stream, backend.upload(stream, batch), 1, q, metric, "d"))
    want = oracle.vector_distance(batch, 1, q, int(metric))
    assert_columns_equal(got.column(2), want, f"dim={dim} {metric.name}")
