"""The fused probe -> WHERE -> GROUP BY pass on the B200 equals the plain
plan (join, then aggregate) as the oracle computes it."""
import numpy as np
import pyarrow as pa
import pytest

import oracle
from compare import abs_columns, assert_batches_equal
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


@pytest.mark.parametrize("combine", [0, 1, 2, 3, 4, 5, 6, 7, 8, 11, 12, 13, 14, 15, 16])
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
            scale = oracle.aggregate(abs_columns(batch, {1}), 0, [(int(f), c) for f, c in sp.aggregates])
            sums = [1 + j for j, (f, c) in enumerate(sp.aggregates) if f in (F.Sum, F.Avg) and c == 1]
            assert_batches_equal(got, want, float_sum_cols=sums, scale=scale)
    finally:
        backend.set_agg_variant(-1, 0)


@pytest.mark.parametrize("rpt", [2, 4, 8])
@pytest.mark.parametrize("form", [5, 6, 7, 8, 11, 12, 13, 14, 15, 16],
                         ids=["dense", "hashed", "dense-vec", "hashed-vec", "dense-stream", "hashed-stream",
                              "dense-lean", "hashed-lean", "dense-lean4", "hashed-lean4"])
def test_fused_probe_table_edges(backend, stream, rpt, form):
    """The fused probe-table kernel (a build-side group key, probe-side
    inputs) on the cases its fast path hands to the slow one: build keys
    that repeat, NULL group keys, the INT64_MIN key on both sides, and group
    keys outside the sampled span (the group-key sample reads build rows
    0, 4, 8, ... of these 32768, so rows 1 mod 4 stay unsampled)."""
    rng = np.random.default_rng(40 + rpt)
    nb, npr = 32_768, 500_000
    key = rng.permutation(nb).astype(np.int64)
    key[:300] = key[300:600]  # 300 keys appear twice
    key[600] = np.iinfo(np.int64).min
    attr = rng.integers(0, 40, nb).astype(np.int32)
    outliers = np.array([701, 705, 709, 713, 717])
    attr[outliers] = [2_000_000_000, -2_000_000_000, 1_000_000, 77_777, -5]
    attr_null = rng.random(nb) < 0.03
    attr_null[outliers] = False
    build = pa.RecordBatch.from_arrays(
        [pa.array(key, pa.int64(), mask=rng.random(nb) < 0.01), pa.array(attr, mask=attr_null)],
        names=["key", "attr"],
    )
    fk = rng.integers(0, nb + nb // 10, npr).astype(np.int64)
    fk[rng.random(npr) < 0.01] = np.iinfo(np.int64).min
    hot = rng.random(npr) < 0.2
    fk[hot] = key[outliers[rng.integers(0, 5, hot.sum())]]
    probe = pa.RecordBatch.from_arrays(
        [
            pa.array(fk, pa.int64(), mask=rng.random(npr) < 0.02),
            pa.array(rng.uniform(-100, 100, npr), mask=rng.random(npr) < 0.03),
            pa.array(rng.integers(1, 51, npr).astype(np.int32), mask=rng.random(npr) < 0.01),
        ],
        names=["fk", "payload", "qty"],
    )
    pred = compare(2, Cmp.Gt, Literal.int32(10))
    aggs = [(F.Sum, 0, 1), (F.Sum, 0, 2), (F.CountStar, 0, 0), (F.Avg, 0, 1), (F.Min, 0, 2), (F.Max, 0, 1)]
    backend.set_agg_variant(form, rpt)
    backend.set_kernel_timing(True)
    try:
        for agg_set, fused in ((aggs[:4], True), (aggs, False)):
            got = run(backend, stream, build, probe, pred, (1, 1), agg_set)
            name = backend.last_kernel_time()[0]
            # the lean kernels take no validity bitmaps: these columns have
            # them, so forms 13 to 16 run the interpreted fused kernel
            assert ("fused" in name) == fused and ("fused-dense" in name) == (fused and form in (5, 7, 11, 13, 15)), name
            assert "lean" not in name, name
            assert ("vec" in name) == (fused and form in (7, 8)), name
            assert ("stream" in name) == (fused and form in (11, 12)), name
            spec = [(int(f), s, c) for f, s, c in agg_set]
            want = oracle.join_aggregate(probe, build, 0, 0, leaves(pred), (1, 1), spec)
            scale = oracle.join_aggregate(abs_columns(probe, {1}), build, 0, 0, leaves(pred), (1, 1), spec)
            assert_batches_equal(got, want, float_sum_cols=(1, 4), scale=scale)
    finally:
        backend.set_agg_variant(-1, 0)
        backend.set_kernel_timing(False)


@pytest.mark.parametrize("form", [5, 6, 7, 8, 11, 12, 13, 14, 15, 16],
                         ids=["dense", "hashed", "dense-vec", "hashed-vec", "dense-stream", "hashed-stream",
                              "dense-lean", "hashed-lean", "dense-lean4", "hashed-lean4"])
def test_fused_float_sums_in_and_out_of_the_fixed_point_window(backend, stream, form):
    """The fused kernels fold a Float64 SUM as an exact integer in a window
    placed from a sample of the column, and every other value through the
    compensated Float64 path: values far above the sampled range (on rows
    the sample does not read), values below the window's unit, NaN, both
    infinities, -0.0 alone, negatives that cancel.  Each group's sum equals
    the oracle's (NaN and infinities bit for bit in kind) and, where finite,
    the exactly rounded sum to 1e-12 of its magnitude."""
    import math

    rng = np.random.default_rng(77 + form)
    nb, npr = 1000, 400_000
    build = pa.RecordBatch.from_arrays([pa.array(np.arange(nb, dtype=np.int64)),
                                        pa.array((np.arange(nb) % 50).astype(np.int32))], names=["key", "attr"])
    fk = rng.integers(0, nb, npr).astype(np.int64)
    x = rng.uniform(-1000.0, 1000.0, npr)
    sampled = np.zeros(npr, bool)
    sampled[np.minimum((np.arange(8192) * npr / 8192).astype(np.int64), npr - 1)] = True
    free = np.nonzero(~sampled)[0]
    big = rng.choice(free, 300, replace=False)
    x[big] = rng.choice([-1.0, 1.0], 300) * rng.uniform(1e9, 1e12, 300)  # above the window
    tiny = rng.choice(free, 300, replace=False)
    x[tiny] = rng.uniform(-1e-20, 1e-20, 300)  # below its unit
    g = fk % 50
    x[np.nonzero(g == 7)[0][:1]] = np.nan
    x[np.nonzero(g == 8)[0][:2]] = np.inf
    i9 = np.nonzero(g == 9)[0]
    x[i9[:1]], x[i9[1:2]] = np.inf, -np.inf
    x[g == 10] = -0.0
    # the lean kernels (forms 13 to 16) take columns without validity bitmaps
    null = rng.random(npr) < (0.0 if form in (13, 14, 15, 16) else 0.02)
    null[~np.isfinite(x)] = False  # the NaN and infinities stay in their groups
    probe = pa.RecordBatch.from_arrays([pa.array(fk), pa.array(x, mask=null),
                                        pa.array(rng.integers(1, 51, npr).astype(np.int32))],
                                       names=["fk", "payload", "qty"])
    aggs = [(F.Sum, 0, 1), (F.CountStar, 0, 0), (F.Avg, 0, 1)]
    spec = [(int(f), s, c) for f, s, c in aggs]
    backend.set_agg_variant(form, 2 if form in (5, 6) else 4)
    backend.set_kernel_timing(True)
    try:
        got = run(backend, stream, build, probe, None, (1, 1), aggs)
        name = backend.last_kernel_time()[0]
        assert ("lean" in name) == (form in (13, 14, 15, 16)) and ("lean4" in name) == (form in (15, 16)), name
    finally:
        backend.set_agg_variant(-1, 0)
        backend.set_kernel_timing(False)
    want = oracle.join_aggregate(probe, build, 0, 0, [], (1, 1), spec)
    scale = oracle.join_aggregate(abs_columns(probe, {1}), build, 0, 0, [], (1, 1), spec)
    assert_batches_equal(got, want, float_sum_cols=(1, 3), scale=scale)
    sums = got.column(1).to_numpy(zero_copy_only=False)
    assert np.isnan(sums[7]) and sums[8] == np.inf and np.isnan(sums[9])
    assert sums[10] == 0.0 and not np.signbit(sums[10])
    valid = probe.column(1).is_valid().to_numpy(zero_copy_only=False)
    for grp in range(50):
        if grp in (7, 8, 9):
            continue
        vals = x[(g == grp) & valid]
        exact = math.fsum(vals.tolist())
        assert abs(sums[grp] - exact) <= 1e-12 * abs(exact) + 1e-300, (grp, sums[grp], exact)


@pytest.mark.parametrize("form", [13, 15])
def test_sum_of_the_where_column(backend, stream, form):
    """The compiled kernels reuse a WHERE column's loaded values for a sum
    over the same column: SUM(qty) under WHERE qty > 10, and SUM(payload)
    under WHERE payload >= -40.5 AND qty < 45 (a Float64 leaf, compared by
    its order key, summed as its raw value), each equal to the oracle's."""
    from oxidelake_b200.params import and_

    build, probe = config2(5_000, 300_001, seed=17 + form)
    x = probe.column(1).to_numpy(zero_copy_only=False).copy()
    x[::7] = -x[::7]  # negative payloads too
    probe = pa.RecordBatch.from_arrays([probe.column(0), pa.array(x), probe.column(2)], names=probe.schema.names)
    cases = [
        (compare(2, Cmp.Gt, Literal.int32(10)), [(F.Sum, 0, 2), (F.CountStar, 0, 0)], ()),
        (and_(compare(1, Cmp.GtEq, Literal.float64(-40.5)), compare(2, Cmp.Lt, Literal.int32(45))),
         [(F.Sum, 0, 1), (F.Sum, 0, 2), (F.CountStar, 0, 0)], (1,)),
    ]
    backend.set_agg_variant(form, 1)
    backend.set_kernel_timing(True)
    try:
        for pred, aggs, fcols in cases:
            got = run(backend, stream, build, probe, pred, (1, 1), aggs)
            assert "lean" in backend.last_kernel_time()[0]
            spec = [(int(f), s, c) for f, s, c in aggs]
            want = oracle.join_aggregate(probe, build, 0, 0, leaves(pred), (1, 1), spec)
            # the scale: |x| on the rows the WHERE keeps (they still pass it)
            xs = np.where(x >= -40.5, np.abs(x), x)
            sprobe = pa.RecordBatch.from_arrays([probe.column(0), pa.array(xs), probe.column(2)], names=probe.schema.names)
            scale = oracle.join_aggregate(sprobe, build, 0, 0, leaves(pred), (1, 1), spec)
            assert_batches_equal(got, want, float_sum_cols=fcols, scale=scale)
    finally:
        backend.set_agg_variant(-1, 0)
        backend.set_kernel_timing(False)


def test_many_requests_in_one_launch(backend, stream):
    """Join-aggregates that differ in their probe batch and WHERE literal run
    as one launch (oxb_join_aggregate_many), each into its own table: every
    result equals its own call's and the oracle's.  Request sizes from 0 rows
    to several tiles; one request with NULL payloads (which the compiled
    kernel does not take) runs alone, inside the same call."""
    build, probe = config2(20_000, 700_000, seed=91)
    rng = np.random.default_rng(92)
    bdev = backend.upload(stream, build)
    table = backend.prepare_join_build(stream, bdev, 0)
    sizes = [0, 1, 1000, 8191, 8193, 60_000, 250_000, 380_815]
    reqs, hosts = [], []
    off = 0
    for i, n in enumerate(sizes):
        part = probe.slice(off, n)
        off += n
        if i == 3:  # NULL payloads
            pay = part.column(1).to_numpy(zero_copy_only=False)
            part = pa.RecordBatch.from_arrays([part.column(0), pa.array(pay, mask=rng.random(n) < 0.1), part.column(2)],
                                              names=part.schema.names)
        lit = int(rng.integers(1, 50))
        hosts.append((part, lit))
        reqs.append((backend.upload(stream, part), 0, table, compare(2, Cmp.Gt, Literal.int32(lit)), (1, 1), AGGS))
    backend.set_kernel_timing(True)
    try:
        outs = backend.join_aggregate_many(stream, reqs)
        assert "many" in backend.last_kernel_time()[0]
    finally:
        backend.set_kernel_timing(False)
    spec = [(int(f), s, c) for f, s, c in AGGS]
    for (part, lit), r, o in zip(hosts, reqs, outs):
        got = backend.download(stream, o)
        alone = backend.download(stream, backend.join_aggregate(stream, *r))
        want = oracle.join_aggregate(part, build, 0, 0, [(2, 3, 3, lit)], (1, 1), spec)
        assert_batches_equal(got, want, float_sum_cols=(1, 4))
        assert_batches_equal(got, alone, float_sum_cols=(1, 4))


def test_many_requests_of_different_shapes_run_alone(backend, stream):
    build, probe = config2(5_000, 90_000, seed=93)
    bdev = backend.upload(stream, build)
    table = backend.prepare_join_build(stream, bdev, 0)
    pdev = backend.upload(stream, probe)
    aggs2 = [(F.Sum, 0, 2), (F.CountStar, 0, 0)]
    reqs = [(pdev, 0, table, compare(2, Cmp.Gt, Literal.int32(20)), (1, 1), AGGS),
            (pdev, 0, table, compare(2, Cmp.Lt, Literal.int32(20)), (1, 1), aggs2)]
    outs = backend.join_aggregate_many(stream, reqs)
    for r, o in zip(reqs, outs):
        got = backend.download(stream, o)
        spec = [(int(f), s, c) for f, s, c in r[5]]
        lf = r[3]
        want = oracle.join_aggregate(probe, build, 0, 0, leaves(lf), (1, 1), spec)
        assert_batches_equal(got, want, float_sum_cols=(1, 4) if len(spec) == 4 else ())
