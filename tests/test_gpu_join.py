"""Hash join build / probe / ranged gather on the B200 against the oracle
(cpu/kernels.rs:185-472): matches in probe-row order then build order,
gathered bit-exactly in any range."""
import json
from pathlib import Path

import numpy as np
import pyarrow as pa
import pytest

import oracle
from compare import assert_batches_equal
from datagen import conformance_left, conformance_right
from oxidelake_b200.errors import Execution
from oxidelake_b200.operator import GpuOperator

pytestmark = pytest.mark.gpu
G = json.loads((Path(__file__).parent / "golden" / "reference_vectors.json").read_text())


def kernels_left():
    return pa.RecordBatch.from_arrays(
        [pa.array([1, 2, None, 2, 5], pa.int64()), pa.array([0.5, None, 2.5, 3.5, -1.0], pa.float64()), pa.array(np.arange(5, dtype=np.int32))],
        names=["k", "v", "i"],
    )


def test_golden_join_skips_null_keys_and_multiplies_matches(backend):
    g = G["join_skips_null_keys_and_multiplies_matches"]
    left = pa.RecordBatch.from_arrays(
        [pa.array([1, 2, None, 2, 5], pa.int64()), pa.array([0.5, None, 2.5, 3.5, -1.0]), pa.array(list("abcde"))],
        names=["k", "v", "s"],
    )
    right = pa.RecordBatch.from_arrays([pa.array(g["rk"], pa.int64()), pa.array(g["name"])], names=["rk", "name"])
    op = GpuOperator(backend)
    out = pa.Table.from_batches(list(op.hash_join(left, 0, right, 0)))
    assert out.num_columns == g["expect_columns"]
    assert out.num_rows == g["expect_rows"]
    assert sorted(out.column(4).to_pylist()) == g["expect_sorted_names"]
    assert op.stats.fallback_batches == 0


@pytest.mark.parametrize("device_index", [True, False])
def test_golden_matches_gather_in_ranges_equal_one_gather(backend, stream, device_index):
    g = G["join_matches_gather_in_ranges_equal_one_gather"]
    left = kernels_left()
    right = pa.RecordBatch.from_arrays(
        [pa.array(g["rk"], pa.int64()), pa.array(np.arange(len(g["rk"]), dtype=np.int64) * 10)], names=["rk", "tag"]
    )
    otable = oracle.JoinTable(right, 0)
    om = oracle.JoinMatches(left, 0, otable)
    ldev, rdev = backend.upload(stream, left), backend.upload(stream, right)
    table = backend.prepare_join_build(stream, rdev, 0, None if device_index else otable.runs())
    assert table.distinct_keys() == otable.distinct_keys() and table.rows() == otable.rows()
    m = backend.probe_join(stream, ldev, 0, table)
    assert len(m) == g["expect_matches"] == len(om)
    proj = [0, 1, 3, 4]
    whole = oracle.hash_join_gather(left, right, otable, om, 0, len(om), proj)
    for chunk in g["chunks"]:
        parts, first = [], 0
        while first < len(m):
            rows = min(chunk, len(m) - first)
            parts.append(backend.download(stream, backend.hash_join(stream, ldev, rdev, table, m, first, rows, proj)))
            first += rows
        got = pa.Table.from_batches(parts).combine_chunks().to_batches()[0]
        assert_batches_equal(got, whole)
    for first, rows in [(7, 1), (0, 8), (3, 5)]:
        with pytest.raises(Execution):
            backend.hash_join(stream, ldev, rdev, table, m, first, rows, proj)
    with pytest.raises(Execution):  # matches of another probe batch
        backend.hash_join(stream, backend.upload(stream, left.slice(0, 2)), rdev, table, m, 0, 1, proj)


@pytest.mark.parametrize("seed", [1, 7, 42])
@pytest.mark.parametrize("rows", [0, 1, 7, 64, 1000])
def test_conformance_shapes(backend, stream, seed, rows):
    left = conformance_left(seed, rows)
    right = conformance_right(seed, 501 if rows else 0)
    lsub = left.select([0, 1, 3])
    rsub = pa.RecordBatch.from_arrays([right.column(0), pa.array(np.arange(right.num_rows, dtype=np.int32))], names=["rk", "r"])
    otable = oracle.JoinTable(rsub, 0)
    om = oracle.JoinMatches(lsub, 0, otable)
    want = oracle.hash_join_gather(lsub, rsub, otable, om, 0, len(om))
    ldev, rdev = backend.upload(stream, lsub), backend.upload(stream, rsub)
    for index in (None, otable.runs()):
        table = backend.prepare_join_build(stream, rdev, 0, index)
        m = backend.probe_join(stream, ldev, 0, table)
        assert len(m) == len(om)
        got = backend.download(stream, backend.hash_join(stream, ldev, rdev, table, m, 0, len(m)))
        assert_batches_equal(got, want)


@pytest.mark.parametrize("key_type", [pa.int64(), pa.int32()])
def test_large_duplicates_extremes_and_nulls(backend, stream, key_type):
    rng = np.random.default_rng(3)
    nb, npr = 300_000, 1_000_000
    if key_type == pa.int64():
        universe = np.array([np.iinfo(np.int64).min, np.iinfo(np.int64).max, 0, -1], dtype=np.int64)
        bk = np.concatenate([universe, rng.integers(-50_000, 50_000, nb - 4)])
        pk = np.concatenate([universe, rng.integers(-60_000, 60_000, npr - 4)])
    else:
        bk = rng.integers(-50_000, 50_000, nb).astype(np.int32)
        pk = rng.integers(-60_000, 60_000, npr).astype(np.int32)
        bk[:2] = [np.iinfo(np.int32).min, np.iinfo(np.int32).max]
        pk[:2] = bk[:2]
    build = pa.RecordBatch.from_arrays(
        [pa.array(bk, key_type, mask=rng.random(nb) < 0.05), pa.array(rng.standard_normal(nb))], names=["bk", "bv"]
    )
    probe = pa.RecordBatch.from_arrays(
        [pa.array(pk, key_type, mask=rng.random(npr) < 0.05), pa.array(np.arange(npr, dtype=np.int64))], names=["pk", "pid"]
    )
    otable = oracle.JoinTable(build, 0)
    om = oracle.JoinMatches(probe, 0, otable)
    ldev, rdev = backend.upload(stream, probe), backend.upload(stream, build)
    table = backend.prepare_join_build(stream, rdev, 0)
    assert table.distinct_keys() == otable.distinct_keys()
    m = backend.probe_join(stream, ldev, 0, table)
    assert len(m) == len(om)
    # three uneven ranges, compared to the oracle's ranges
    cuts = [0, len(m) // 3, len(m) // 3 + 12_345, len(m)]
    for a, b in zip(cuts, cuts[1:]):
        got = backend.download(stream, backend.hash_join(stream, ldev, rdev, table, m, a, b - a, [1, 3, 0, 2]))
        want = oracle.hash_join_gather(probe, build, otable, om, a, b - a, [1, 3, 0, 2])
        assert_batches_equal(got, want)


def test_one_key_everywhere(backend, stream):
    """STATUS.md's skew cases: all build rows on one key."""
    build = pa.RecordBatch.from_arrays([pa.array(np.full(20_000, 7, np.int64)), pa.array(np.arange(20_000, dtype=np.int64))], names=["k", "b"])
    probe = pa.RecordBatch.from_arrays([pa.array(np.array([7, 8, 7] * 5, np.int64)), pa.array(np.arange(15, dtype=np.int64))], names=["k", "p"])
    otable = oracle.JoinTable(build, 0)
    om = oracle.JoinMatches(probe, 0, otable)
    ldev, rdev = backend.upload(stream, probe), backend.upload(stream, build)
    table = backend.prepare_join_build(stream, rdev, 0)
    m = backend.probe_join(stream, ldev, 0, table)
    assert len(m) == len(om) == 10 * 20_000
    got = backend.download(stream, backend.hash_join(stream, ldev, rdev, table, m, 65_536, 65_536))
    want = oracle.hash_join_gather(probe, build, otable, om, 65_536, 65_536)
    assert_batches_equal(got, want)


@pytest.mark.parametrize("key_type", [pa.int64(), pa.int32()])
@pytest.mark.parametrize("dup", [False, True], ids=["unique", "one-repeat"])
def test_dense_keys_placed_without_sort(backend, stream, key_type, dup):
    """Build keys that fill their range: unique ones are placed by key offset
    (no sort) and probed through the direct index, a single repeated key
    sends the build back to the sort; both give the oracle's table, matches
    and gathered rows, for probe keys missing inside the range and outside
    it on both sides."""
    rng = np.random.default_rng(11 + dup)
    nb, npr = 200_000, 600_000
    bk = (rng.permutation(nb) - 70_000).astype(key_type.to_pandas_dtype())
    if dup:
        bk[5] = bk[123_456]
    pk = rng.integers(-80_000, 140_000, npr).astype(key_type.to_pandas_dtype())
    if key_type == pa.int64():
        pk[7] = np.iinfo(np.int64).min  # no build row has it: no match through the direct index
    build = pa.RecordBatch.from_arrays(
        [pa.array(bk, key_type, mask=rng.random(nb) < 0.03), pa.array(np.arange(nb, dtype=np.int64))], names=["bk", "bv"]
    )
    probe = pa.RecordBatch.from_arrays(
        [pa.array(pk, key_type, mask=rng.random(npr) < 0.03), pa.array(np.arange(npr, dtype=np.int64))], names=["pk", "pid"]
    )
    otable = oracle.JoinTable(build, 0)
    om = oracle.JoinMatches(probe, 0, otable)
    ldev, rdev = backend.upload(stream, probe), backend.upload(stream, build)
    table = backend.prepare_join_build(stream, rdev, 0)
    assert table.distinct_keys() == otable.distinct_keys()
    m = backend.probe_join(stream, ldev, 0, table)
    assert len(m) == len(om)
    got = backend.download(stream, backend.hash_join(stream, ldev, rdev, table, m, 0, len(m), [1, 3, 0, 2]))
    want = oracle.hash_join_gather(probe, build, otable, om, 0, len(om), [1, 3, 0, 2])
    assert_batches_equal(got, want)


@pytest.mark.parametrize("shape", ["sparse", "dense-dups", "mixed"])
def test_gather_tiles_over_sparse_and_duplicate_matches(backend, stream, shape):
    """The gather cuts its output into 2048-row tiles and searches each
    tile's probe rows in shared memory when they fit (4096 rows), in HBM
    otherwise.  Sparse matches (one probe row in 20 matches: a tile spans
    about 40K probe rows), one build key repeated 5000 times (a tile inside
    one probe row) and a mix, each gathered whole and in windows that cut
    tiles at odd places, equal the oracle's rows."""
    rng = np.random.default_rng({"sparse": 1, "dense-dups": 2, "mixed": 3}[shape])
    nb, npr = 20_000, 400_000
    rk = np.arange(nb, dtype=np.int64)
    if shape != "sparse":
        rk[:5000] = 7  # key 7: 5000 build rows
    right = pa.RecordBatch.from_arrays([pa.array(rk), pa.array(rng.integers(0, 1 << 40, nb), pa.int64())],
                                       names=["rk", "tag"])
    if shape == "sparse":
        fk = np.where(rng.random(npr) < 0.05, rng.integers(0, nb, npr), -1 - rng.integers(0, 1000, npr))
    elif shape == "dense-dups":
        fk = np.where(rng.random(npr) < 0.001, 7, rng.integers(nb, 2 * nb, npr))
    else:
        fk = np.where(rng.random(npr) < 0.5, rng.integers(0, nb, npr), -5)
        fk[rng.random(npr) < 0.0005] = 7
    left = pa.RecordBatch.from_arrays(
        [pa.array(fk.astype(np.int64), mask=rng.random(npr) < 0.01),
         pa.array(rng.standard_normal(npr), mask=rng.random(npr) < 0.02),
         pa.array(rng.integers(-9, 9, npr).astype(np.int32))],
        names=["fk", "v", "q"],
    )
    otable = oracle.JoinTable(right, 0)
    om = oracle.JoinMatches(left, 0, otable)
    ldev, rdev = backend.upload(stream, left), backend.upload(stream, right)
    table = backend.prepare_join_build(stream, rdev, 0)
    m = backend.probe_join(stream, ldev, 0, table)
    total = len(m)
    assert total == len(om) and total > 10_000
    proj = [0, 1, 2, 4]
    whole = oracle.hash_join_gather(left, right, otable, om, 0, total, proj)
    got = backend.download(stream, backend.hash_join(stream, ldev, rdev, table, m, 0, total, proj))
    assert_batches_equal(got, whole)
    for first, rows in [(1, 2047), (2047, 2050), (total // 3, 4097), (total - 5001, 5001), (total - 1, 1)]:
        got = backend.download(stream, backend.hash_join(stream, ldev, rdev, table, m, first, rows, proj))
        assert_batches_equal(got, whole.slice(first, rows))
