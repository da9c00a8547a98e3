"""Grouped aggregation on the B200 against the oracle
(cpu/kernels.rs:478-818): groups sorted by key with NULL last; COUNT,
integer SUM (wrapping), MIN/MAX (totalOrder for floats) bit-exact; Float64
SUM/AVG within 1e-12 relative."""
import json
import struct
from pathlib import Path

import numpy as np
import pyarrow as pa
import pytest

import oracle
from compare import abs_columns, assert_batches_equal, assert_columns_equal
from datagen import config1, splitmix64_stream
from oxidelake_b200.errors import Plan, Unsupported
from oxidelake_b200.params import AggregateFunction as F
from oxidelake_b200.params import AggregateSpec, Literal, and_, compare, leaves
from oxidelake_b200.params import Comparison as Cmp

pytestmark = pytest.mark.gpu
G = json.loads((Path(__file__).parent / "golden" / "reference_vectors.json").read_text())
NAMES = {"Sum": F.Sum, "Count": F.Count, "Min": F.Min, "Max": F.Max}


def f64_array(hexes):
    vals = np.array([0 if h is None else int(h, 16) for h in hexes], dtype=np.uint64).view(np.float64)
    return pa.array(vals, pa.float64(), mask=np.array([h is None for h in hexes]))


def run(backend, stream, batch, spec, pred=None):
    dev = backend.upload(stream, batch)
    return backend.download(stream, backend.aggregate(stream, dev, spec, pred))


def want(batch, spec, pred=None):
    return oracle.aggregate(batch, spec.group_by, [(int(f), c) for f, c in spec.aggregates], leaves(pred))


def float_sum_cols(batch, spec):
    return [1 + j for j, (f, c) in enumerate(spec.aggregates) if (f == F.Sum and pa.types.is_float64(batch.schema.field(c).type)) or f == F.Avg]


def magnitude(batch, spec, pred=None):
    """The query over |x| of the summed Float64 columns the predicate does
    not read: per group, the scale of its sums' tolerance."""
    pred_cols = {lf.column for lf in leaves(pred)}
    cols = {c for f, c in spec.aggregates if f in (F.Sum, F.Avg)} - pred_cols
    return want(abs_columns(batch, cols), spec, pred)


def check(backend, stream, batch, spec, pred=None, exact_floats=False):
    got = run(backend, stream, batch, spec, pred)
    w = want(batch, spec, pred)
    assert got.schema.names == w.schema.names
    if exact_floats:
        assert_batches_equal(got, w)
    else:
        assert_batches_equal(got, w, float_sum_cols(batch, spec), scale=magnitude(batch, spec, pred))
    return got


def test_golden_groups_nulls_last_and_skips_null_values(backend, stream):
    g = G["aggregate_groups_nulls_last_and_skips_null_values"]
    batch = pa.RecordBatch.from_arrays([pa.array([1, 2, None, 2, 5], pa.int64()), pa.array([0.5, None, 2.5, 3.5, -1.0])], names=["k", "v"])
    spec = AggregateSpec(0, [(NAMES[f], c) for f, c in g["aggregates"]])
    out = check(backend, stream, batch, spec, exact_floats=True)
    assert out.column(0).to_pylist() == g["expect_keys"]
    assert out.schema.field(1).name == g["expect_name_1"] and out.schema.field(4).name == g["expect_name_4"]
    assert out.column(4).to_pylist() == g["expect_maxk"]


def test_golden_edge_rows_bit_exact(backend, stream):
    g = G["batch_by_batch_and_merged_partials_equal_one_pass"]
    rows = g["rows"]
    batch = pa.RecordBatch.from_arrays(
        [pa.array([r[0] for r in rows], pa.int64()), pa.array([r[1] for r in rows], pa.int64()), f64_array([r[2] for r in rows])],
        names=["k", "i", "f"],
    )
    spec = AggregateSpec(0, [(NAMES[f], c) for f, c in g["aggregates"]])
    out = check(backend, stream, batch, spec, exact_floats=True)
    assert out.column(1).to_pylist() == g["expect_col1"]


def test_golden_sum_overflow_wraps(backend, stream):
    g = G["sum_overflow_wraps"]
    batch = pa.RecordBatch.from_arrays(
        [pa.array([r[0] for r in g["rows"]], pa.int64()), pa.array([r[1] for r in g["rows"]], pa.int64())], names=["k", "x"]
    )
    out = check(backend, stream, batch, AggregateSpec(0, [(F.Sum, 1), (F.Count, 1)]))
    rows = ["|".join("NULL" if v is None else str(v) for v in r) for r in zip(*[c.to_pylist() for c in out.columns])]
    assert sorted(rows) == g["expect_rows"]
    assert out.column(1).to_pylist() == g["device_expect_sums"]


def test_golden_float_min_max_total_order(backend, stream):
    g = G["float_min_max_total_order"]
    rows = g["device_rows"]
    batch = pa.RecordBatch.from_arrays([pa.array([r[0] for r in rows], pa.int64()), f64_array([r[1] for r in rows])], names=["k", "v"])
    out = check(backend, stream, batch, AggregateSpec(0, [(F.Min, 1), (F.Max, 1)]), exact_floats=True)
    assert_columns_equal(out.column(1), f64_array(g["device_expect_min"]))
    assert_columns_equal(out.column(2), f64_array(g["device_expect_max"]))


def test_golden_signed_zeros(backend, stream):
    g = G["signed_zeros"]
    rows = g["one_sign_rows"]
    batch = pa.RecordBatch.from_arrays([pa.array([r[0] for r in rows], pa.int64()), f64_array([r[1] for r in rows])], names=["k", "v"])
    out = check(backend, stream, batch, AggregateSpec(0, [(F.Min, 1), (F.Max, 1)]), exact_floats=True)
    assert_columns_equal(out.column(1), f64_array([e[1] for e in g["one_sign_expect"]]))
    assert_columns_equal(out.column(2), f64_array([e[2] for e in g["one_sign_expect"]]))
    for pair in (["0x0000000000000000", "0x8000000000000000"], ["0x8000000000000000", "0x0000000000000000"]):
        b = pa.RecordBatch.from_arrays([pa.array([1, 1], pa.int64()), f64_array(pair)], names=["k", "v"])
        out = check(backend, stream, b, AggregateSpec(0, [(F.Min, 1), (F.Max, 1)]), exact_floats=True)
        assert_columns_equal(out.column(1), f64_array([g["both_zeros_expect"][0]]))


def numbering_cases():
    """cuda/mod.rs:1161-1260: the keys, then x and v per row, all drawn by
    splitmix64 from state 29 in the reference's order."""
    state = 29
    r, state = splitmix64_stream(state, 65_536)
    hundred = [None if int(x) % 50 == 0 else (int(x) >> 8) % 100 for x in r]
    cases = [
        ("no rows", []),
        ("only NULL keys", [None] * 1000),
        ("a group per row", [i - 5000 for i in range(10_000)]),
        ("extreme keys", [[-(2**63), 2**63 - 1, None, 0, -1][i % 5] for i in range(4096)]),
        ("100 keys in one GPU batch", hundred),
    ]
    out = []
    for name, keys in cases:
        n = len(keys)
        rr, state = splitmix64_stream(state, 2 * n)
        rx, rv = rr[0::2], rr[1::2]
        x = [None if int(a) % 40 == 0 else int(np.uint64(a).view(np.int64)) for a in rx]
        v = [None if int(b) % 40 == 0 else float(((int(b) >> 8) & 0xFFFFFFFF) % 400) / 4.0 - 50.0 for b in rv]
        out.append((name, pa.RecordBatch.from_arrays([pa.array(keys, pa.int64()), pa.array(x, pa.int64()), pa.array(v, pa.float64())], names=["k", "x", "v"])))
    return out


@pytest.mark.parametrize("case", numbering_cases(), ids=lambda c: c[0])
def test_numbering_cases_like_the_reference(backend, stream, case):
    _, batch = case
    spec = AggregateSpec(0, [(F.Sum, 1), (F.Count, 1), (F.Min, 1), (F.Max, 1), (F.Sum, 2), (F.Count, 2), (F.Min, 2), (F.Max, 2)])
    check(backend, stream, batch, spec, exact_floats=True)  # quarters: every order sums exactly


def test_widened_functions_and_int32(backend, stream):
    rng = np.random.default_rng(5)
    n = 500_000
    batch = pa.RecordBatch.from_arrays(
        [
            pa.array(rng.integers(-300, 300, n).astype(np.int32), pa.int32(), mask=rng.random(n) < 0.01),
            pa.array(rng.integers(-(10**6), 10**6, n).astype(np.int32), pa.int32(), mask=rng.random(n) < 0.02),
            pa.array(rng.uniform(-1e3, 1e3, n), pa.float64(), mask=rng.random(n) < 0.02),
            pa.array(rng.integers(-(2**62), 2**62, n), pa.int64()),
        ],
        names=["g", "x", "v", "w"],
    )
    spec = AggregateSpec(
        0,
        [(F.Sum, 1), (F.Min, 1), (F.Max, 1), (F.Count, 1), (F.Avg, 2), (F.Sum, 2), (F.CountStar, 0), (F.Avg, 1), (F.Sum, 3), (F.Max, 3)],
    )
    out = check(backend, stream, batch, spec)
    assert out.schema.field(0).type == pa.int32() and out.schema.field(1).type == pa.int64()
    assert out.schema.field(2).type == pa.int32() and out.schema.field(5).type == pa.float64()


def test_config1_query(backend, stream):
    """SELECT k, SUM(v), COUNT(*) FROM t WHERE k >= 2 AND v < 4.0 GROUP BY k."""
    batch = config1(1_000_000)
    pred = and_(compare(1, Cmp.GtEq, Literal.int64(2)), compare(2, Cmp.Lt, Literal.float64(4.0)))
    out = check(backend, stream, batch, AggregateSpec(1, [(F.Sum, 2), (F.CountStar, 0)]), pred)
    assert out.column(0).to_pylist() == list(range(2, 10))


def test_high_cardinality(backend, stream):
    rng = np.random.default_rng(9)
    n = 4_000_000
    batch = pa.RecordBatch.from_arrays(
        [
            pa.array(rng.integers(0, 1_000_000, n), pa.int64(), mask=rng.random(n) < 0.001),
            pa.array(rng.integers(-(10**6), 10**6, n).astype(np.int32), pa.int32(), mask=rng.random(n) < 0.02),
            pa.array(rng.integers(0, 100, n).astype(np.int32)),
        ],
        names=["g", "x", "f"],
    )
    spec = AggregateSpec(0, [(F.Sum, 1), (F.Min, 1), (F.Max, 1), (F.Count, 1)])
    check(backend, stream, batch, spec, compare(2, Cmp.Lt, Literal.int32(50)))
    check(backend, stream, batch, spec)


def test_errors(backend, stream):
    batch = pa.RecordBatch.from_arrays([pa.array([1.0, 2.0]), pa.array([1, 2], pa.int64())], names=["f", "k"])
    dev = backend.upload(stream, batch)
    with pytest.raises(Unsupported):
        backend.aggregate(stream, dev, AggregateSpec(0, [(F.Count, 1)]))
    with pytest.raises(Plan):
        backend.aggregate(stream, dev, AggregateSpec(5, [(F.Count, 1)]))
    out = run(backend, stream, batch.slice(0, 0), AggregateSpec(1, [(F.Count, 0)]))
    assert out.num_rows == 0 and out.num_columns == 2


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4])
def test_float_sums_are_exact_to_1e12_under_cancellation(backend, stream, variant):
    """Where a group's values cancel, the compensated device sums still equal
    the exactly rounded sum (math.fsum) to 1e-12 relative, whichever kernel
    variant folds them (the sequential sum of the reference is only accurate
    to about 1e-16 of the inputs' magnitude there)."""
    import math

    rng = np.random.default_rng(100 + variant)
    n, groups = 400_000, 300
    g = rng.integers(0, groups, n)
    v = rng.uniform(-5, 5, n)
    batch = pa.RecordBatch.from_arrays([pa.array(g), pa.array(v)], names=["g", "v"])
    backend.set_agg_variant(variant, 0)
    try:
        out = run(backend, stream, batch, AggregateSpec(0, [(F.Sum, 1), (F.Avg, 1), (F.CountStar, 0)]))
    finally:
        backend.set_agg_variant(-1, 0)
    order = np.argsort(g, kind="stable")
    bounds = np.searchsorted(g[order], np.arange(groups + 1))
    exact = np.array([math.fsum(v[order[bounds[k] : bounds[k + 1]]]) for k in range(groups)])
    got = out.column(1).to_numpy()
    assert out.column(0).to_pylist() == list(range(groups))
    rel = np.abs(got - exact) / np.abs(exact)
    assert rel.max() <= 1e-12, (rel.max(), int(rel.argmax()))
    counts = out.column(3).to_numpy()
    assert np.allclose(out.column(2).to_numpy(), exact / counts, rtol=1e-12, atol=0)


@pytest.mark.parametrize(
    "lo,span,distinct",
    [(-5, 32_767, 32_768), (1_000, 32_768, 20_000), (0, 200_000, 120_000), (-(1 << 40), 1 << 41, 5_000)],
    ids=["bitmap-edge", "dense-edge", "dense", "sparse-sort"],
)
def test_group_order_paths(backend, stream, lo, span, distinct):
    """The emitted groups in key order whichever way they are ordered: a key
    span below 32768 by a shared-memory bitmap, a span the keys fill to a
    quarter by presence flags in HBM, a wider one by the radix sort; the
    smallest and largest keys of the span always present, NULL keys last."""
    rng = np.random.default_rng(span % 997)
    keys = np.unique(np.concatenate([[lo, lo + span], rng.integers(lo, lo + span + 1, distinct)]))
    n = 300_000
    g = np.concatenate([keys, rng.choice(keys, n - len(keys))]).astype(np.int64)
    rng.shuffle(g)
    batch = pa.RecordBatch.from_arrays(
        [pa.array(g, mask=rng.random(n) < 0.01), pa.array(rng.integers(-9, 10, n).astype(np.int64))], names=["g", "x"]
    )
    spec = AggregateSpec(0, [(F.Sum, 1), (F.CountStar, 0), (F.Min, 1)])
    assert_batches_equal(run(backend, stream, batch, spec), want(batch, spec))
