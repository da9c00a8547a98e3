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
from oxidelake_b200.params import AggregateSpec, Literal, and_, compare, leaves
from oxidelake_b200.params import Comparison as Cmp

pytestmark = pytest.mark.gpu

SPEC = AggregateSpec(0, [(F.Sum, 1), (F.Min, 1), (F.Max, 1), (F.Count, 1)])


def fold(backend, stream, batches, spec, pred):
    devs = [backend.upload(stream, b) for b in batches]
    return backend.download(stream, backend.aggregate_batches(stream, devs, spec, pred))


def want(batches, spec, pred):
    whole = pa.Table.from_batches(batches).combine_chunks().to_batches()[0]
    return whole, oracle.aggregate(whole, spec.group_by, [(int(f), c) for f, c in spec.aggregates], leaves(pred))


@pytest.mark.parametrize("variant", [-1, 9], ids=["auto", "partitioned"])
@pytest.mark.parametrize("selectivity", [1, 50, 99])
def test_high_cardinality_uneven_batches(backend, stream, selectivity, variant):
    batches = config3_batches(3_000_000, 200_000, seed=selectivity, min_rows=800, max_rows=400_000)
    assert len({b.num_rows for b in batches}) > 3
    pred = compare(2, Cmp.Lt, Literal.int32(selectivity))
    backend.set_agg_variant(variant, 0)
    try:
        got = fold(backend, stream, batches, SPEC, pred)
    finally:
        backend.set_agg_variant(-1, 0)
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


def _wide_batches(seed, distinct, sizes):
    """Many groups with Float64 values that cancel (5 % NULL), an Int32
    column without NULLs, NULL keys and the key INT64_MIN."""
    rng = np.random.default_rng(seed)
    out = []
    for n in sizes:
        g = rng.integers(-distinct // 2, distinct // 2, n).astype(np.int64)
        if n > 4:
            g[:2] = np.iinfo(np.int64).min
        v = rng.uniform(-1e6, 1e6, n) * rng.choice([1.0, 1e-9], n)
        out.append(
            pa.RecordBatch.from_arrays(
                [pa.array(g, mask=rng.random(n) < 0.03), pa.array(v, mask=rng.random(n) < 0.05),
                 pa.array(rng.integers(-1000, 1000, n).astype(np.int32)),
                 pa.array(rng.integers(0, 100, n).astype(np.int32))],
                names=["g", "v", "x", "f"],
            )
        )
    return out


@pytest.mark.parametrize("variant", [-1, 9, 10, 0], ids=["auto", "partitioned", "partitioned-64", "direct"])
def test_many_groups_every_variant(backend, stream, variant):
    """The hash-partitioned passes (two levels of partitions here; pinned
    with 64 partitions their shared tables overflow into the HBM table) and
    the single persistent kernel give the oracle's groups: Float64 SUM and
    AVG to the stated tolerance, everything else bit-exact."""
    batches = _wide_batches(40 + variant, 400_000, (0, 70_001, 1, 300_000, 8192, 0, 621_807))
    # four accumulators (SUM, COUNT and MIN of v, MAX of x): two stored columns
    spec = AggregateSpec(0, [(F.Sum, 1), (F.Avg, 1), (F.Min, 1), (F.Max, 2), (F.CountStar, 0), (F.Count, 1)])
    pred = compare(3, Cmp.Lt, Literal.int32(70))
    backend.set_agg_variant(variant, 0)
    backend.set_kernel_timing(True)
    try:
        got = fold(backend, stream, batches, spec, pred)
        name = backend.last_kernel_time()[0]
    finally:
        backend.set_agg_variant(-1, 0)
        backend.set_kernel_timing(False)
    if variant >= 0:
        assert ("partitioned" in name) == (variant in (9, 10)), name
    whole, w = want(batches, spec, pred)
    scale = oracle.aggregate(abs_columns(whole, {1}), 0, [(int(f), c) for f, c in spec.aggregates], leaves(pred))
    assert got.num_rows == w.num_rows
    assert_batches_equal(got, w, float_sum_cols=(1, 2), scale=scale)


def test_partitioned_int32_key_and_sums(backend, stream):
    """An Int32 group key, integer SUM that wraps, and two accumulators on
    one column: one stored column in the partition buffers."""
    rng = np.random.default_rng(77)
    batches = []
    for n in (123_457, 500_000, 3):
        g = rng.integers(-300_000, 300_000, n).astype(np.int32)
        x = rng.integers(np.iinfo(np.int64).min // 2, np.iinfo(np.int64).max // 2, n, dtype=np.int64)
        batches.append(pa.RecordBatch.from_arrays([pa.array(g, mask=rng.random(n) < 0.01), pa.array(x)], names=["g", "x"]))
    spec = AggregateSpec(0, [(F.Sum, 1), (F.Min, 1), (F.Count, 1)])
    backend.set_agg_variant(9, 0)  # about 600K groups: 4096 partitions in two levels
    try:
        got = fold(backend, stream, batches, spec, None)
    finally:
        backend.set_agg_variant(-1, 0)
    _, w = want(batches, spec, None)
    assert_batches_equal(got, w)


@pytest.mark.parametrize("ncols", [2, 3], ids=["32-byte-records", "48-byte-records"])
def test_partitioned_wide_records(backend, stream, ncols):
    """Two or three stored columns (32- or 48-byte partition records):
    AVG of a nullable Int32 (a Float64 sum of integers), MAX of a Float64
    with NaN and signed zeros (totalOrder), MAX and MIN of an Int64, through
    the partitioned passes; Float64 results to the stated tolerance, the
    rest bit-exact."""
    rng = np.random.default_rng(90 + ncols)
    batches = []
    for n in (150_000, 7, 333_333, 0, 90_000):
        g = rng.integers(0, 250_000, n).astype(np.int64)
        x = rng.integers(-2_000_000_000, 2_000_000_000, n).astype(np.int32)
        v = rng.standard_normal(n) * 1e3
        if n > 10:
            v[:4] = [np.nan, -0.0, 0.0, -np.inf]
        y = rng.integers(np.iinfo(np.int64).min // 4, np.iinfo(np.int64).max // 4, n, dtype=np.int64)
        batches.append(
            pa.RecordBatch.from_arrays(
                [pa.array(g, mask=rng.random(n) < 0.01), pa.array(x, mask=rng.random(n) < 0.04), pa.array(v),
                 pa.array(y)],
                names=["g", "x", "v", "y"],
            )
        )
    aggs = [(F.Avg, 1), (F.Max, 2), (F.Min, 1)] if ncols == 2 else [(F.Avg, 1), (F.Max, 2), (F.Max, 3)]
    spec = AggregateSpec(0, aggs)
    backend.set_agg_variant(9, 0)
    backend.set_kernel_timing(True)
    try:
        got = fold(backend, stream, batches, spec, None)
        name = backend.last_kernel_time()[0]
    finally:
        backend.set_agg_variant(-1, 0)
        backend.set_kernel_timing(False)
    assert "partitioned" in name, name
    whole, w = want(batches, spec, None)
    scale = oracle.aggregate(abs_columns(whole, {1}), 0, [(int(f), c) for f, c in spec.aggregates], [])
    assert got.num_rows == w.num_rows
    assert_batches_equal(got, w, float_sum_cols=(1,), scale=scale)


def _fold_named(backend, stream, batches, spec, pred, variant):
    """The fold with the variant pinned, and the name of the timed passes."""
    backend.set_agg_variant(variant, 0)
    backend.set_kernel_timing(True)
    try:
        got = fold(backend, stream, batches, spec, pred)
        name = backend.last_kernel_time()[0]
    finally:
        backend.set_agg_variant(-1, 0)
        backend.set_kernel_timing(False)
    return got, name


@pytest.mark.parametrize("selectivity", [1, 50, 99])
def test_dense_range_pinned(backend, stream, selectivity):
    """Keys that fill their range, through the dense passes (variant 17:
    partitions by key offset, 8-byte records, no hashing, groups emitted in
    key order without a sort): bit-exact against the oracle."""
    batches = config3_batches(3_000_000, 200_000, seed=100 + selectivity, min_rows=800, max_rows=400_000)
    pred = compare(2, Cmp.Lt, Literal.int32(selectivity))
    got, name = _fold_named(backend, stream, batches, SPEC, pred, 17)
    assert name == "agg_batches_dense", name
    _, w = want(batches, SPEC, pred)
    assert got.num_rows == w.num_rows
    assert_batches_equal(got, w)


def test_dense_range_chosen_automatically(backend, stream):
    """Enough kept rows over a filled range: the automatic choice is the
    dense passes, with the oracle's groups."""
    batches = config3_batches(6_000_000, 1_000_000, seed=5, min_rows=8192, max_rows=1 << 20)
    pred = compare(2, Cmp.Lt, Literal.int32(99))
    got, name = _fold_named(backend, stream, batches, SPEC, pred, -1)
    assert name == "agg_batches_dense", name
    _, w = want(batches, SPEC, pred)
    assert got.num_rows == w.num_rows
    assert_batches_equal(got, w)


def test_dense_range_null_and_min_keys_and_carries(backend, stream):
    """NULL keys (the NULL group last), the key INT64_MIN (first), groups
    whose values are all NULL, COUNT(*) beside COUNT(x), empty batches, and
    Int64 sums of Int32 extremes that carry across 32 bits both ways."""
    rng = np.random.default_rng(123)
    batches = []
    for n in (0, 40_000, 1, 250_000, 7, 123_456):
        g = rng.integers(-3000, 3000, n).astype(np.int64)
        x = rng.choice(np.array([2**31 - 1, -(2**31), 1, -1, 0, 123_456_789], dtype=np.int32), n)
        xm = (rng.random(n) < 0.05) | ((g >= 100) & (g < 110))
        if n > 10:
            g[:3] = np.iinfo(np.int64).min
        batches.append(
            pa.RecordBatch.from_arrays(
                [pa.array(g, mask=rng.random(n) < 0.01), pa.array(x, mask=xm),
                 pa.array(rng.integers(0, 100, n).astype(np.int32))],
                names=["g", "x", "f"],
            )
        )
    spec = AggregateSpec(0, [(F.Sum, 1), (F.Min, 1), (F.Max, 1), (F.Count, 1), (F.CountStar, 0)])
    pred = compare(2, Cmp.Lt, Literal.int32(90))
    got, name = _fold_named(backend, stream, batches, spec, pred, 17)
    assert name == "agg_batches_dense", name
    _, w = want(batches, spec, pred)
    assert got.num_rows == w.num_rows
    assert_batches_equal(got, w)


def test_dense_range_int32_key_without_bitmaps(backend, stream):
    """An Int32 group key over negative and positive values with gaps, and
    an Int32 input without a validity bitmap (COUNT(x) is then the row
    count), with no WHERE."""
    rng = np.random.default_rng(321)
    batches = []
    for n in (90_000, 3, 410_000):
        g = (rng.integers(-100_000, 100_000, n) * 3).astype(np.int32)
        x = rng.integers(np.iinfo(np.int32).min, np.iinfo(np.int32).max, n, dtype=np.int64).astype(np.int32)
        batches.append(pa.RecordBatch.from_arrays([pa.array(g), pa.array(x)], names=["g", "x"]))
    spec = AggregateSpec(0, [(F.Sum, 1), (F.Max, 1), (F.Count, 1)])
    got, name = _fold_named(backend, stream, batches, spec, None, 17)
    assert name == "agg_batches_dense", name
    _, w = want(batches, spec, None)
    assert got.num_rows == w.num_rows
    assert_batches_equal(got, w)


def test_dense_range_outlier_keys_fall_back(backend, stream):
    """A handful of keys far outside the sampled range: the count pass sees
    them, and the fold takes the other passes, with the oracle's groups."""
    rng = np.random.default_rng(11)
    batches = []
    for n in (300_000, 200_000):
        g = rng.integers(0, 100_000, n).astype(np.int64)
        g[n // 2 + 1] = 10**12
        g[n // 3 + 7] = -(10**12)
        x = rng.integers(-1000, 1000, n).astype(np.int32)
        batches.append(pa.RecordBatch.from_arrays([pa.array(g), pa.array(x, mask=rng.random(n) < 0.02)], names=["g", "x"]))
    got, name = _fold_named(backend, stream, batches, SPEC, None, 17)
    assert name != "agg_batches_dense", name
    _, w = want(batches, SPEC, None)
    assert got.num_rows == w.num_rows
    assert_batches_equal(got, w)


def test_dense_range_two_leaf_where(backend, stream):
    """A WHERE of a Float64 and an Int64 leaf (signed zeros, NaN and
    infinities in the Float64 column) through the compiled dense passes:
    four rows a load, the comparisons as masks; ragged batch ends."""
    rng = np.random.default_rng(77)
    batches = []
    for n in (131_071, 5, 262_147, 40_001):
        g = rng.integers(-500_000, 500_000, n).astype(np.int64)
        x = rng.integers(-(2**31), 2**31 - 1, n, dtype=np.int64).astype(np.int32)
        v = rng.uniform(-1, 1, n)
        if n > 10:
            v[:6] = [np.nan, -0.0, 0.0, np.inf, -np.inf, 0.25]
        w = rng.integers(0, 100, n).astype(np.int64)
        batches.append(
            pa.RecordBatch.from_arrays(
                [pa.array(g), pa.array(x, mask=rng.random(n) < 0.03), pa.array(v), pa.array(w)],
                names=["g", "x", "v", "w"],
            )
        )
    pred = and_(compare(2, Cmp.GtEq, Literal.float64(-0.0)), compare(3, Cmp.LtEq, Literal.int64(50)))
    spec = AggregateSpec(0, [(F.Sum, 1), (F.Min, 1), (F.Max, 1), (F.Count, 1), (F.CountStar, 0)])
    got, name = _fold_named(backend, stream, batches, spec, pred, 17)
    assert name == "agg_batches_dense", name
    _, w = want(batches, spec, pred)
    assert got.num_rows == w.num_rows
    assert_batches_equal(got, w)


@pytest.mark.parametrize("end", ["top", "bottom"])
def test_dense_range_at_the_ends_of_int64(backend, stream, end):
    """Keys within 100K of INT64_MAX, or of INT64_MIN with INT64_MIN itself
    among them (its own slot, emitted first): the widened range is clamped
    at the ends of the Int64 order, and the groups still equal the oracle's."""
    rng = np.random.default_rng(5 if end == "top" else 6)
    i64 = np.iinfo(np.int64)
    batches = []
    for n in (70_000, 3, 130_001):
        off = rng.integers(0, 100_000, n).astype(np.int64)
        g = i64.max - off if end == "top" else i64.min + 1 + off
        if end == "bottom" and n > 10:
            g[:4] = i64.min
        x = rng.integers(-1000, 1000, n).astype(np.int32)
        batches.append(pa.RecordBatch.from_arrays([pa.array(g), pa.array(x, mask=rng.random(n) < 0.05)], names=["g", "x"]))
    spec = AggregateSpec(0, [(F.Sum, 1), (F.Min, 1), (F.Max, 1), (F.Count, 1), (F.CountStar, 0)])
    got, name = _fold_named(backend, stream, batches, spec, None, 17)
    assert name == "agg_batches_dense", name
    _, w = want(batches, spec, None)
    assert got.num_rows == w.num_rows
    assert_batches_equal(got, w)


def test_dense_range_where_keeping_nothing_in_range(backend, stream):
    """A WHERE that keeps only rows whose key is NULL: no record reaches the
    dense passes, and the only group is the NULL one."""
    rng = np.random.default_rng(9)
    n = 300_000
    g = rng.integers(0, 50_000, n).astype(np.int64)
    nullkey = rng.random(n) < 0.1
    f = np.where(nullkey, 1, 0).astype(np.int32)
    x = rng.integers(-5, 5, n).astype(np.int32)
    batch = pa.RecordBatch.from_arrays([pa.array(g, mask=nullkey), pa.array(x), pa.array(f)], names=["g", "x", "f"])
    pred = compare(2, Cmp.Eq, Literal.int32(1))
    got, _ = _fold_named(backend, stream, [batch], SPEC, pred, 17)
    _, w = want([batch], SPEC, pred)
    assert got.num_rows == w.num_rows == 1
    assert_batches_equal(got, w)
