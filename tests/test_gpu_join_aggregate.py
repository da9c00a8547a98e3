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
from oxidelake_b200.params import AggregateSpec, Literal, compare, leaves

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


@pytest.mark.parametrize("combine", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("rpt", [1, 2])
def test_every_kernel_variant(backend, stream, combine, rpt):
    """Each compiled variant of the row-loop kernels (the autotuner's
    choices) gives the plain plan's result."""
    build, probe = config2(3_000, 400_000 + 777, seed=rpt * 2 + combine)
    pred = compare(2, Cmp.Gt, Literal.int32(10))
    backend.set_agg_variant(combine, rpt)
    try:
        got = run(backend, stream, build, probe, pred, (1, 1), AGGS)
        want = oracle.join_aggregate(probe, build, 0, 0, leaves(pred), (1, 1), [(int(f), s, c) for f, s, c in AGGS])
        assert_batches_equal(got, want, float_sum_cols=(1, 4))
        # the plain aggregate's row loop, many accumulators (no combining) and few
        aggs5 = [(F.Sum, 1), (F.Min, 1), (F.Max, 2), (F.Count, 2), (F.Avg, 1), (F.CountStar, 0)]
        spec = AggregateSpec(0, aggs5)
        rng = np.random.default_rng(combine + 7 * rpt)
        n = 300_001
        batch = pa.RecordBatch.from_arrays(
            [
                pa.array(rng.integers(0, 700, n), pa.int64(), mask=rng.random(n) < 0.01),
                pa.array(rng.uniform(-5, 5, n), mask=rng.random(n) < 0.02),
                pa.array(rng.integers(-9, 9, n).astype(np.int32), mask=rng.random(n) < 0.03),
            ],
            names=["g", "v", "x"],
        )
        dev = backend.upload(stream, batch)
        for sp in (spec, AggregateSpec(0, [(F.Sum, 1), (F.CountStar, 0)])):
            got = backend.download(stream, backend.aggregate(stream, dev, sp))
            want = oracle.aggregate(batch, 0, [(int(f), c) for f, c in sp.aggregates])
            sums = [1 + j for j, (f, c) in enumerate(sp.aggregates) if f in (F.Sum, F.Avg) and c == 1]
            assert_batches_equal(got, want, float_sum_cols=sums)
    finally:
        backend.set_agg_variant(-1, 0)
