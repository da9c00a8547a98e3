"""The oracle against every golden vector of the reference's own tests
(tests/golden/reference_vectors.json).  CPU only."""
import json
import math
import struct
from pathlib import Path

import numpy as np
import pyarrow as pa
import pytest

import oracle
from datagen import demo_digest, demo_table

G = json.loads((Path(__file__).parent / "golden" / "reference_vectors.json").read_text())
OPS = {"Eq": 0, "Lt": 1, "LtEq": 2, "Gt": 3, "GtEq": 4}
TYPES = {"Int64": 1, "Float64": 2, "Int32": 3}
FUNCS = {"Sum": 0, "Count": 1, "Min": 2, "Max": 3, "Avg": 4}


def fb(h):
    """float from a hex bit pattern (None stays None)."""
    return None if h is None else struct.unpack("<d", struct.pack("<Q", int(h, 16)))[0]


def bits(x):
    return None if x is None else "0x%016x" % struct.unpack("<Q", struct.pack("<d", x))[0]


def f64_array(hexes):
    vals = np.array([0 if h is None else int(h, 16) for h in hexes], dtype=np.uint64).view(np.float64)
    return pa.array(vals, pa.float64(), mask=np.array([h is None for h in hexes]))


def col_bits(arr):
    out = []
    vals = arr.fill_null(0.0).to_numpy(zero_copy_only=False).view(np.uint64)
    for i, ok in enumerate(arr.is_valid().to_pylist()):
        out.append("0x%016x" % int(vals[i]) if ok else None)
    return out


def kernels_batch():
    g = G["filter_drops_null_predicates_and_projects"]
    return pa.RecordBatch.from_arrays(
        [pa.array(g["k"], pa.int64()), f64_array(g["v"]), pa.array(g["s"], pa.utf8())], names=["k", "v", "s"]
    )


def leaf(c, op, t, v):
    return (c, OPS[op], TYPES[t], fb(v) if t == "Float64" else v)


def test_filter_drops_null_predicates_and_projects():
    g = G["filter_drops_null_predicates_and_projects"]
    out = oracle.filter_project(kernels_batch(), [leaf(*l) for l in g["leaves"]], g["projection"])
    assert out.schema.names == g["expect_names"]
    assert out.column(1).to_pylist() == g["expect_k"]


def test_float_comparisons_order_as_datafusion_does():
    g = G["float_comparisons_order_as_datafusion_does"]
    batch = pa.RecordBatch.from_arrays([f64_array(g["values"])], names=["v"])
    for op, lit, want in g["cases"]:
        rows = oracle.filter_rows(batch, [(0, OPS[op], 2, fb(lit))])
        assert rows.tolist() == want, (op, lit)


def test_filter_type_mismatch_is_unsupported():
    g = G["filter_type_mismatch_is_unsupported"]
    with pytest.raises(oracle.OracleError) as e:
        oracle.filter_project(kernels_batch(), [leaf(*g["leaf"])], g["projection"])
    assert e.value.is_unsupported()


def right_batch(g):
    return pa.RecordBatch.from_arrays([pa.array(g["rk"], pa.int64()), pa.array(g["name"], pa.utf8())], names=["rk", "name"])


def test_join_skips_null_keys_and_multiplies_matches():
    g = G["join_skips_null_keys_and_multiplies_matches"]
    out = oracle.hash_join(kernels_batch(), right_batch(g), 0, 0)
    assert out.num_columns == g["expect_columns"]
    assert out.num_rows == g["expect_rows"]
    assert sorted(out.column(4).to_pylist()) == g["expect_sorted_names"]


def test_join_matches_gather_in_ranges_equal_one_gather():
    g = G["join_matches_gather_in_ranges_equal_one_gather"]
    left, right = kernels_batch(), right_batch(g)
    table = oracle.JoinTable(right, 0)
    m = oracle.JoinMatches(left, 0, table)
    assert len(m) == g["expect_matches"]
    li, ri = m.pairs(0, len(m))
    assert [[int(a), int(b)] for a, b in zip(li, ri)] == g["expect_pairs"]
    whole = oracle.hash_join_gather(left, right, table, m, 0, len(m), None).select(g["projection"])
    for chunk in g["chunks"]:
        parts, first = [], 0
        while first < len(m):
            rows = min(chunk, len(m) - first)
            parts.append(oracle.hash_join_gather(left, right, table, m, first, rows, g["projection"]))
            first += rows
        assert pa.Table.from_batches(parts).to_pydict() == whole.to_pydict(), chunk
    for first, rows in g["out_of_range"]:
        with pytest.raises(oracle.OracleError):
            m.pairs(first, rows if rows < 2**63 else 2**64 - 1)


def test_aggregate_groups_nulls_last_and_skips_null_values():
    g = G["aggregate_groups_nulls_last_and_skips_null_values"]
    out = oracle.aggregate(kernels_batch(), 0, [(FUNCS[f], c) for f, c in g["aggregates"]])
    assert out.column(0).to_pylist() == g["expect_keys"]
    assert col_bits(out.column(1)) == g["expect_sums"]
    assert out.column(2).to_pylist() == g["expect_counts"]
    assert out.schema.field(1).name == g["expect_name_1"]
    assert out.schema.field(4).name == g["expect_name_4"]
    assert out.column(4).to_pylist() == g["expect_maxk"]


def edge_batch(rows):
    return pa.RecordBatch.from_arrays(
        [pa.array([r[0] for r in rows], pa.int64()), pa.array([r[1] for r in rows], pa.int64()), f64_array([r[2] for r in rows])],
        names=["k", "i", "f"],
    )


def all_bits(batch):
    out = []
    for c in batch.columns:
        if pa.types.is_float64(c.type):
            out.append(col_bits(c))
        else:
            out.append(c.to_pylist())
    return out


def test_batch_by_batch_and_merged_partials_equal_one_pass():
    g = G["batch_by_batch_and_merged_partials_equal_one_pass"]
    rows = g["rows"]
    aggs = [(FUNCS[f], c) for f, c in g["aggregates"]]
    whole = oracle.aggregate(edge_batch(rows), 0, aggs)
    for split in range(1, len(rows)):
        a, b = edge_batch(rows[:split]), edge_batch(rows[split:])
        streamed = oracle.GroupedAggregator(a.schema, 0, aggs)
        streamed.update(a)
        streamed.update(b)
        merged = oracle.GroupedAggregator(a.schema, 0, aggs)
        merged.merge(oracle.aggregate(b, 0, aggs))
        merged.merge(oracle.aggregate(a, 0, aggs))
        assert all_bits(streamed.finish()) == all_bits(whole), split
        assert all_bits(merged.finish()) == all_bits(whole), split
    assert whole.column(1).to_pylist() == g["expect_col1"]
    assert col_bits(whole.column(7)) == g["expect_col7_bits"]
    assert col_bits(whole.column(8)) == g["expect_col8_bits"]


def test_aggregate_over_empty_batch_has_no_groups():
    g = G["aggregate_over_empty_batch_has_no_groups"]
    out = oracle.aggregate(kernels_batch().slice(0, 0), 0, [(1, 1)])
    assert out.num_rows == g["expect_rows"]
    assert out.num_columns == g["expect_columns"]


def test_total_order_keys_order_like_total_cmp_and_round_trip():
    g = G["total_order_keys"]
    vals = [fb(h) for h in g["values_in_order"]]
    keys = [oracle.total_order_key(v) for v in vals]
    for v, k in zip(vals, keys):
        assert bits(oracle.from_total_order_key(k)) == bits(v)
    assert keys == sorted(keys) and len(set(keys)) == len(keys)
    assert bits(oracle.from_total_order_key(2**63 - 1)) == g["from_key_max_bits"]
    assert bits(oracle.from_total_order_key(-(2**63))) == g["from_key_min_bits"]


def test_vector_distances():
    g = G["vector_distances"]
    vec = pa.FixedSizeListArray.from_arrays(pa.array(g["values"], pa.float32()), g["dim"], mask=pa.array([not v for v in g["valid"]]))
    batch = pa.RecordBatch.from_arrays([vec], names=["vec"])
    d = oracle.vector_distance(batch, 0, g["query"], oracle.L2).to_pylist()
    assert d[0] == 0.0 and d[1] is None and d[2] == np.float32(math.sqrt(np.float32(20.0)))
    assert np.float32(d[2]) == np.sqrt(np.float32(20.0))
    c = oracle.vector_distance(batch, 0, g["query"], oracle.COSINE).to_pylist()
    assert abs(c[0]) < g["cosine_tolerance"] and c[1] is None
    assert abs(c[2] - g["expect_cosine_approx"][2]) < g["cosine_tolerance"]
    a, b = g["zero_norm_cosine_is_nan"]
    assert math.isnan(oracle.cosine(a, b))


def test_sum_overflow_wraps():
    g = G["sum_overflow_wraps"]
    batch = pa.RecordBatch.from_arrays(
        [pa.array([r[0] for r in g["rows"]], pa.int64()), pa.array([r[1] for r in g["rows"]], pa.int64())], names=["k", "x"]
    )
    out = oracle.aggregate(batch, 0, [(0, 1), (1, 1)])
    rows = ["|".join("NULL" if v is None else str(v) for v in r) for r in zip(*[c.to_pylist() for c in out.columns])]
    assert sorted(rows) == g["expect_rows"]
    assert out.column(1).to_pylist() == g["device_expect_sums"]


def test_float_min_max_total_order():
    g = G["float_min_max_total_order"]
    first, rest = [], []
    for k, values, _ in g["groups"]:
        for i, v in enumerate(values):
            (first if i == 0 else rest).append((k, v))
    want = {k: (mn, mx) for k, _, (mn, mx) in g["groups"]}
    for order in ([first, rest], [rest, first]):
        agg = None
        for part in order:
            b = pa.RecordBatch.from_arrays([pa.array([r[0] for r in part], pa.int64()), f64_array([r[1] for r in part])], names=["k", "v"])
            if agg is None:
                agg = oracle.GroupedAggregator(b.schema, 0, [(2, 1), (3, 1)])
            agg.update(b)
        out = agg.finish()
        got = {k: (a, b) for k, a, b in zip(out.column(0).to_pylist(), col_bits(out.column(1)), col_bits(out.column(2)))}
        assert got == want
    rows = g["device_rows"]
    b = pa.RecordBatch.from_arrays([pa.array([r[0] for r in rows], pa.int64()), f64_array([r[1] for r in rows])], names=["k", "v"])
    out = oracle.aggregate(b, 0, [(2, 1), (3, 1)])
    assert col_bits(out.column(1)) == g["device_expect_min"]
    assert col_bits(out.column(2)) == g["device_expect_max"]


def test_signed_zeros():
    g = G["signed_zeros"]
    rows = g["one_sign_rows"]
    b = pa.RecordBatch.from_arrays([pa.array([r[0] for r in rows], pa.int64()), f64_array([r[1] for r in rows])], names=["k", "v"])
    out = oracle.aggregate(b, 0, [(2, 1), (3, 1)])
    got = [[k, a, c] for k, a, c in zip(out.column(0).to_pylist(), col_bits(out.column(1)), col_bits(out.column(2)))]
    assert got == g["one_sign_expect"]
    for pair in (["0x0000000000000000", "0x8000000000000000"], ["0x8000000000000000", "0x0000000000000000"]):
        b = pa.RecordBatch.from_arrays([pa.array([1, 1], pa.int64()), f64_array(pair)], names=["k", "v"])
        out = oracle.aggregate(b, 0, [(2, 1), (3, 1)])
        assert [col_bits(out.column(1))[0], col_bits(out.column(2))[0]] == g["both_zeros_expect"]


def test_special_float_filters_select_by_total_order():
    """conformance.rs:1459-1490 `selects`, by hand, against the oracle."""
    from datagen import special_floats

    g = G["special_float_filter_predicates"]
    for seed in g["shapes"]["seeds"]:
        for n in g["shapes"]["sizes"]:
            batch = special_floats(seed, n)
            for pred in g["predicates"]:
                leaves = [(0 if c == "k" else 1, OPS[op], 1 if c == "k" else 2, v if c == "k" else fb(v)) for c, op, v in pred]
                got = oracle.filter_rows(batch, leaves).tolist()
                want = []
                kk, vv = batch.column(0).to_pylist(), batch.column(1)
                vbits = vv.fill_null(0.0).to_numpy(zero_copy_only=False)
                vval = vv.is_valid().to_pylist()
                for r in range(n):
                    ok = True
                    for c, op, lit in pred:
                        if c == "k":
                            if kk[r] is None:
                                ok = False
                                break
                            o = (kk[r] > lit) - (kk[r] < lit)
                        else:
                            if not vval[r]:
                                ok = False
                                break
                            x = 0.0 if vbits[r] == 0.0 else vbits[r]
                            y = fb(lit)
                            y = 0.0 if y == 0.0 else y
                            kx, ky = oracle.total_order_key(x), oracle.total_order_key(y)
                            o = (kx > ky) - (kx < ky)
                        ok = ok and {"Eq": o == 0, "Lt": o < 0, "LtEq": o <= 0, "Gt": o > 0, "GtEq": o >= 0}[op]
                    if ok:
                        want.append(r)
                assert got == want, (seed, n, pred)


def test_slot_hash_kats():
    for key, cap, want in G["slot_hash"]["cases"]:
        assert oracle.slot_hash(key, cap) == want


def test_demo_table_digest():
    g = G["demo_table_digest"]
    assert demo_digest(demo_table(g["rows"], g["seed"])) == g["digest"]


def test_parallel_join_aggregate_equals_one_pass():
    """The partitioned CPU baseline (threads > 1) equals the one-pass oracle:
    integers exactly, float sums within 1e-12 relative."""
    from datagen import config2

    build, probe = config2(2000, 50_000, seed=5)
    leaves = [(2, 3, 3, 10)]
    aggs = [(0, 0, 1), (0, 0, 2), (5, 0, 0), (4, 0, 1)]
    one = oracle.join_aggregate(probe, build, 0, 0, leaves, (1, 1), aggs, threads=1)
    par = oracle.join_aggregate(probe, build, 0, 0, leaves, (1, 1), aggs, threads=4)
    assert one.column(0).to_pylist() == par.column(0).to_pylist()
    assert one.column(2).to_pylist() == par.column(2).to_pylist()
    assert one.column(3).to_pylist() == par.column(3).to_pylist()
    a, b = np.array(one.column(1).to_pylist()), np.array(par.column(1).to_pylist())
    assert np.all(np.abs(a - b) <= 1e-12 * np.abs(a))


@pytest.mark.parametrize("threads", [2, 7])
def test_parallel_aggregate_equals_one_pass(threads):
    """The oracle's key-partitioned aggregate (the checker for the large
    configurations) gives the same bits as one sequential update: NULL
    keys, special floats, wrapping Int64 sums, Int32 widening, AVG."""
    rng = np.random.default_rng(31)
    n = 60_000
    specials = np.array([np.nan, -np.inf, np.inf, 0.0, -0.0, 1e300, -1e300, 3.5], np.float64)
    v = np.where(rng.random(n) < 0.2, specials[rng.integers(0, len(specials), n)], rng.uniform(-1e6, 1e6, n))
    big = np.where(rng.random(n) < 0.1, np.iinfo(np.int64).max - rng.integers(0, 5, n), rng.integers(-100, 100, n))
    batch = pa.RecordBatch.from_arrays(
        [pa.array(rng.integers(-3000, 3000, n), pa.int64(), mask=rng.random(n) < 0.02),
         pa.array(v, mask=rng.random(n) < 0.05),
         pa.array(big.astype(np.int64)),
         pa.array(rng.integers(-2**31, 2**31, n).astype(np.int32), mask=rng.random(n) < 0.05),
         pa.array(rng.integers(0, 100, n).astype(np.int32))],
        names=["g", "v", "big", "x", "f"])
    aggs = [(0, 1), (2, 1), (3, 1), (4, 1), (0, 2), (0, 3), (2, 3), (3, 3), (4, 3), (1, 3), (5, 0)]
    leaves = [(4, 1, 3, 70)]
    one = oracle.aggregate(batch, 0, aggs, leaves)
    par = oracle.aggregate(batch, 0, aggs, leaves, threads=threads)
    assert par.schema == one.schema and par.num_rows == one.num_rows
    for i in range(one.num_columns):
        a, b = one.column(i), par.column(i)
        assert a.is_valid().to_pylist() == b.is_valid().to_pylist()
        av = a.fill_null(0).to_numpy(zero_copy_only=False)
        bv = b.fill_null(0).to_numpy(zero_copy_only=False)
        assert (av.view(np.uint8) == bv.view(np.uint8)).all(), one.schema.field(i).name
