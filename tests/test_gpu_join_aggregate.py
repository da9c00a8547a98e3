"""The fused probe -> WHERE -> GROUP BY pass on the B200 equals the plain
plan (join, then aggregate) as the oracle computes it."""
import numpy as np
import pyarrow as pa
import pytest

import oracle
from compare import assert_batches_equal
from datagen import config2
from oxidelake_b200.params import AggregateFunction as F
from oxidelake_b200.params import Comparison as Cmp
from oxidelake_b200.params import Literal, compare, leaves

pytestmark = pytest.mark.gpu

AGGS = [(F.Sum, 0, 1), (F.Sum, 0, 2), (F.CountStar, 0, 0), (F.Avg, 0, 1)]


def run(backend, stream, build, probe, pred, group, aggs, device_index=True):
    bdev, pdev = backend.upload(stream, build), backend.upload(stream, probe)
    index = None if device_index else oracle.JoinTable(build, 0).runs()
    table = backend.prepare_join_build(stream, bdev, 0, index)
    return backend.download(stream, backend.join_aggregate(stream, pdev, 0, table, pred, group, aggs))


@pytest.mark.parametrize("probe_rows", [0, 1, 1000, 2_000_000])
def test_config2_shape(backend, stream, probe_rows):
    build, probe = config2(20_000, probe_rows, seed=probe_rows + 1)
    pred = compare(2, Cmp.Gt, Literal.int32(10))
    got = run(backend, stream, build, probe, pred, (1, 1), AGGS)
    want = oracle.join_aggregate(probe, build, 0, 0, leaves(pred), (1, 1), [(int(f), s, c) for f, s, c in AGGS])
    assert_batches_equal(got, want, float_sum_cols=(1, 4))


def test_duplicates_nulls_and_probe_side_groups(backend, stream):
    rng = np.random.default_rng(2)
    nb, npr = 5_000, 300_000
    build = pa.RecordBatch.from_arrays(
        [pa.array(rng.integers(0, 2_000, nb), pa.int64(), mask=rng.random(nb) < 0.02), pa.array(rng.integers(0, 50, nb).astype(np.int32), mask=rng.random(nb) < 0.05)],
        names=["key", "attr"],
    )
    probe = pa.RecordBatch.from_arrays(
        [
            pa.array(rng.integers(0, 2_500, npr), pa.int64(), mask=rng.random(npr) < 0.02),
            pa.array(rng.uniform(0, 100, npr), mask=rng.random(npr) < 0.03),
            pa.array(rng.integers(1, 51, npr).astype(np.int32)),
            pa.array(rng.integers(-5, 5, npr), pa.int64(), mask=rng.random(npr) < 0.1),
        ],
        names=["fk", "payload", "qty", "g"],
    )
    pred = compare(2, Cmp.LtEq, Literal.int32(30))
    aggs = [(F.Sum, 0, 1), (F.Min, 1, 1), (F.Max, 0, 1), (F.Count, 1, 1), (F.CountStar, 0, 0), (F.Sum, 0, 2)]
    for group in [(1, 1), (0, 3)]:
        for device_index in (True, False):
            got = run(backend, stream, build, probe, pred, group, aggs, device_index)
            want = oracle.join_aggregate(probe, build, 0, 0, leaves(pred), group, [(int(f), s, c) for f, s, c in aggs])
            assert_batches_equal(got, want, float_sum_cols=(1,))
