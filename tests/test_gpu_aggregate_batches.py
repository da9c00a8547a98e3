"""Many uneven RecordBatches folded by one persistent launch
(oxb_aggregate_batches) equal the oracle's aggregate of their concatenation:
bit-exact group keys, COUNT, integer SUM, MIN and MAX; Float64 SUM/AVG to
the stated tolerance."""
import numpy as np
import pyarrow as pa
import pytest

import oracle
from compare import abs_columns, assert_batches_equal
from datagen import config3_batches
from oxidelake_b200.params import AggregateFunction as F
from oxidelake_b200.params import AggregateSpec, Literal, compare, leaves
from oxidelake_b200.params import Comparison as Cmp

pytestmark = pytest.mark.gpu

SPEC = AggregateSpec(0, [(F.Sum, 1), (F.Min, 1), (F.Max, 1), (F.Count, 1)])


def fold(backend, stream, batches, spec, pred):
    devs = [backend.upload(stream, b) for b in batches]
    return backend.download(stream, backend.aggregate_batches(stream, devs, spec, pred))


def want(batches, spec, pred):
    whole = pa.Table.from_batches(batches).combine_chunks().to_batches()[0]
    return whole, oracle.aggregate(whole, spec.group_by, [(int(f), c) for f, c in spec.aggregates], leaves(pred))


@pytest.mark.parametrize("selectivity", [1, 50, 99])
def test_high_cardinality_uneven_batches(backend, stream, selectivity):
    batches = config3_batches(3_000_000, 200_000, seed=selectivity, min_rows=800, max_rows=400_000)
    assert len({b.num_rows for b in batches}) > 3
    pred = compare(2, Cmp.Lt, Literal.int32(selectivity))
    got = fold(backend, stream, batches, SPEC, pred)
    _, w = want(batches, SPEC, pred)
    assert got.num_rows == w.num_rows
    assert_batches_equal(got, w)


def test_empty_batches_null_keys_and_float_sums(backend, stream):
    rng = np.random.default_rng(8)
    batches = []
    for n in (0, 5000, 1, 0, 70_000, 1023, 1025):
        g = rng.integers(-500, 500, n).astype(np.int64)
        if n > 2:
            g[0] = np.iinfo(np.int64).min
        v = rng.uniform(-50, 50, n)
        batches.append(
            pa.RecordBatch.from_arrays(
                [pa.array(g, mask=rng.random(n) < 0.05), pa.array(v, mask=rng.random(n) < 0.1),
                 pa.array(rng.integers(0, 10, n).astype(np.int32))],
                names=["g", "v", "f"],
            )
        )
    spec = AggregateSpec(0, [(F.Sum, 1), (F.Avg, 1), (F.CountStar, 0), (F.Min, 1), (F.Max, 2)])
    pred = compare(2, Cmp.GtEq, Literal.int32(2))
    got = fold(backend, stream, batches, spec, pred)
    whole, w = want(batches, spec, pred)
    scale = oracle.aggregate(abs_columns(whole, {1}), 0, [(int(f), c) for f, c in spec.aggregates], leaves(pred))
    assert_batches_equal(got, w, float_sum_cols=(1, 2), scale=scale)


def test_one_batch_equals_aggregate(backend, stream):
    batches = config3_batches(300_000, 50_000, seed=3, min_rows=300_000, max_rows=300_000)
    dev = backend.upload(stream, batches[0])
    single = backend.download(stream, backend.aggregate(stream, dev, SPEC))
    got = fold(backend, stream, batches, SPEC, None)
    assert_batches_equal(got, single)
