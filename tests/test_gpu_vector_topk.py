"""ORDER BY l2|cosine(vec, q) LIMIT k on the B200 (BF16 tcgen05 scan, FP32
re-rank) against the oracle's FP32 top-k (cpu/kernels.rs:841-927 distances,
ties by row id): the same row ids and bit-identical FP32 distances."""
import numpy as np
import pyarrow as pa
import pytest

import oracle
from oxidelake_b200.params import Comparison as Cmp
from oxidelake_b200.params import DistanceMetric, Literal, compare, leaves

pytestmark = pytest.mark.gpu


def table(n, dim, seed, null_frac=0.0, normalize=False):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n, dim)).astype(np.float32)
    if normalize:
        v /= np.linalg.norm(v, axis=1, keepdims=True).astype(np.float32)
    vec = pa.FixedSizeListArray.from_arrays(pa.array(v.reshape(-1)), dim)
    if null_frac:
        mask = rng.random(n) < null_frac
        vec = pa.FixedSizeListArray.from_arrays(pa.array(v.reshape(-1)), dim, mask=pa.array(mask))
    f = pa.array(rng.integers(0, 100, n), pa.int64())
    return pa.RecordBatch.from_arrays([pa.array(np.arange(n, dtype=np.int64)), f, vec], names=["id", "f", "emb"]), v


def run(backend, stream, batch, queries, k, metric, pred=None, exact=False, overfetch=0):
    dev = backend.upload(stream, batch)
    ix = backend.vector_index(stream, dev, 2)
    return backend.vector_topk(stream, ix, dev, pred, queries, k, metric, overfetch=overfetch, exact=exact)


def check(got_ids, got_dist, want_ids, want_dist):
    assert got_ids.shape == want_ids.shape
    bad = np.nonzero((got_ids != want_ids).any(axis=1))[0]
    assert bad.size == 0, f"queries {bad[:5].tolist()} differ: got {got_ids[bad[0]].tolist()} want {want_ids[bad[0]].tolist()}"
    gd, wd = got_dist.view(np.uint32), want_dist.view(np.uint32)
    both_nan = np.isnan(got_dist) & np.isnan(want_dist)
    assert ((gd == wd) | both_nan).all(), "distances differ in their bits"


@pytest.mark.parametrize("metric", [DistanceMetric.L2, DistanceMetric.Cosine], ids=["l2", "cosine"])
@pytest.mark.parametrize("n,dim,nq,k", [(1000, 64, 3, 5), (20_000, 100, 130, 7), (50_000, 768, 64, 10)])
def test_matches_fp32_reference(backend, stream, metric, n, dim, nq, k):
    batch, v = table(n, dim, seed=n + dim, null_frac=0.02)
    rng = np.random.default_rng(7)
    queries = rng.standard_normal((nq, dim)).astype(np.float32)
    pred = compare(1, Cmp.Lt, Literal.int64(30))
    ids, dist, stats = run(backend, stream, batch, queries, k, metric, pred)
    want_ids, want_dist = oracle.vector_topk(batch, 2, queries, k, int(metric), leaves(pred), threads=oracle.cpu_threads())
    check(ids, dist, want_ids, want_dist)
    assert stats["reranked"] >= nq * k


@pytest.mark.parametrize("metric", [DistanceMetric.L2, DistanceMetric.Cosine], ids=["l2", "cosine"])
def test_normalized_rows_as_configured(backend, stream, metric):
    """L2-normalised rows, 256 queries from the same distribution, top-10 with
    a 30 %-selective filter: the configured shape at a smaller row count."""
    batch, v = table(200_000, 768, seed=11, normalize=True)
    rng = np.random.default_rng(12)
    q = rng.standard_normal((256, 768)).astype(np.float32)
    q /= np.linalg.norm(q, axis=1, keepdims=True).astype(np.float32)
    pred = compare(1, Cmp.Lt, Literal.int64(30))
    ids, dist, stats = run(backend, stream, batch, q, 10, metric, pred)
    want_ids, want_dist = oracle.vector_topk(batch, 2, q, 10, int(metric), leaves(pred), threads=oracle.cpu_threads())
    check(ids, dist, want_ids, want_dist)
    assert stats["exact_queries"] <= 256
    assert 0.0 <= stats["mean_score_error"] <= stats["max_score_error"] < 0.05


def test_ties_zero_norms_and_short_results(backend, stream):
    """Duplicated rows tie and are ordered by row id; zero vectors give a NaN
    cosine distance, which sorts last; fewer qualifying rows than k pad with
    id -1 and NaN."""
    rng = np.random.default_rng(3)
    n, dim = 3000, 16
    v = rng.integers(-2, 3, (n, dim)).astype(np.float32)
    v[100:200] = v[0]
    v[300:310] = 0.0
    batch = pa.RecordBatch.from_arrays(
        [pa.array(np.arange(n, dtype=np.int64)), pa.array(rng.integers(0, 100, n), pa.int64()),
         pa.FixedSizeListArray.from_arrays(pa.array(v.reshape(-1)), dim)],
        names=["id", "f", "emb"],
    )
    q = np.vstack([v[0], rng.integers(-2, 3, (4, dim)).astype(np.float32)])
    for metric in (DistanceMetric.L2, DistanceMetric.Cosine):
        for k, pred in ((50, None), (40, compare(1, Cmp.Lt, Literal.int64(1))), (400, compare(1, Cmp.Eq, Literal.int64(5)))):
            ids, dist, _ = run(backend, stream, batch, q, k, metric, pred)
            want_ids, want_dist = oracle.vector_topk(batch, 2, q, k, int(metric), leaves(pred))
            check(ids, dist, want_ids, want_dist)


@pytest.mark.parametrize("metric", [DistanceMetric.L2, DistanceMetric.Cosine], ids=["l2", "cosine"])
def test_exact_path(backend, stream, metric):
    batch, v = table(30_000, 96, seed=5, null_frac=0.05)
    q = np.random.default_rng(9).standard_normal((5, 96)).astype(np.float32)
    pred = compare(1, Cmp.GtEq, Literal.int64(50))
    ids, dist, stats = run(backend, stream, batch, q, 12, metric, pred, exact=True)
    assert stats["exact_queries"] == 5
    want_ids, want_dist = oracle.vector_topk(batch, 2, q, 12, int(metric), leaves(pred))
    check(ids, dist, want_ids, want_dist)


def test_overfetch_one_still_exact(backend, stream):
    """With no over-fetch the bound check widens the re-ranked set or takes
    the exact path, so the answer is still the reference's."""
    batch, v = table(40_000, 128, seed=21)
    q = np.random.default_rng(22).standard_normal((20, 128)).astype(np.float32)
    ids, dist, stats = run(backend, stream, batch, q, 25, DistanceMetric.L2, overfetch=1)
    want_ids, want_dist = oracle.vector_topk(batch, 2, q, 25, int(DistanceMetric.L2), threads=oracle.cpu_threads())
    check(ids, dist, want_ids, want_dist)


@pytest.mark.parametrize("metric", [DistanceMetric.L2, DistanceMetric.Cosine], ids=["l2", "cosine"])
def test_per_query_filter_literals(backend, stream, metric):
    """Queries whose WHERE differs only in a literal share one scan: each
    query's answer equals its own top-k under its own predicate."""
    batch, v = table(60_000, 128, seed=31, null_frac=0.01)
    rng = np.random.default_rng(32)
    nq = 150
    q = rng.standard_normal((nq, 128)).astype(np.float32)
    lits = [int(t) for t in rng.integers(1, 100, nq)]
    shared = compare(0, Cmp.GtEq, Literal.int64(100))
    dev = backend.upload(stream, batch)
    ix = backend.vector_index(stream, dev, 2)
    ids, dist, st = backend.vector_topk(
        stream, ix, dev, shared, q, 9, metric, query_leaf=(1, Cmp.Lt, [Literal.int64(t) for t in lits])
    )
    for i in range(nq):
        pred = compare(1, Cmp.Lt, Literal.int64(lits[i]))
        wi, wd = oracle.vector_topk(batch, 2, q[i : i + 1], 9, int(metric), leaves(shared) + leaves(pred))
        check(ids[i : i + 1], dist[i : i + 1], wi, wd)
    # and the exact path with the same per-query literals
    ide, de, _ = backend.vector_topk(
        stream, ix, dev, shared, q[:4], 9, metric, exact=True, query_leaf=(1, Cmp.Lt, [Literal.int64(t) for t in lits[:4]])
    )
    check(ide, de, ids[:4], dist[:4])


@pytest.mark.parametrize("metric", [DistanceMetric.L2, DistanceMetric.Cosine], ids=["l2", "cosine"])
def test_selective_where_with_per_query_literals(backend, stream, metric):
    """A shared WHERE that keeps a fifth of the rows (the scan runs over the
    kept rows only, copied in row order) together with a per-query leaf over
    a nullable column: each query's answer is its own top-k; a WHERE that
    keeps nothing pads every answer with id -1 and NaN."""
    rng = np.random.default_rng(41)
    n, dim, nq, k = 50_000, 96, 70, 8
    v = rng.standard_normal((n, dim)).astype(np.float32)
    vec = pa.FixedSizeListArray.from_arrays(pa.array(v.reshape(-1)), dim, mask=pa.array(rng.random(n) < 0.02))
    f = pa.array(rng.integers(0, 100, n), pa.int64())
    w = pa.array(rng.integers(0, 1000, n), pa.int64(), mask=rng.random(n) < 0.05)
    batch = pa.RecordBatch.from_arrays([pa.array(np.arange(n, dtype=np.int64)), f, vec, w], names=["id", "f", "emb", "w"])
    q = rng.standard_normal((nq, dim)).astype(np.float32)
    lits = [int(t) for t in rng.integers(50, 1000, nq)]
    shared = compare(1, Cmp.Lt, Literal.int64(20))
    dev = backend.upload(stream, batch)
    ix = backend.vector_index(stream, dev, 2)
    ids, dist, _ = backend.vector_topk(
        stream, ix, dev, shared, q, k, metric, query_leaf=(3, Cmp.Lt, [Literal.int64(t) for t in lits])
    )
    for i in range(nq):
        pred = compare(3, Cmp.Lt, Literal.int64(lits[i]))
        wi, wd = oracle.vector_topk(batch, 2, q[i : i + 1], k, int(metric), leaves(shared) + leaves(pred))
        check(ids[i : i + 1], dist[i : i + 1], wi, wd)
    none = compare(1, Cmp.Lt, Literal.int64(0))
    ids0, dist0, _ = backend.vector_topk(stream, ix, dev, none, q[:3], k, metric)
    assert (ids0 == -1).all() and np.isnan(dist0).all()


def test_concurrent_calls_with_different_shared_memory(backend):
    """Host threads on their own streams run top-k calls with different k at
    once, so the scan and re-rank launch with different shared-memory sizes
    concurrently: every call equals the same call made alone."""
    import threading

    batch, _ = table(60_000, 128, seed=31)
    s0 = backend.create_stream()
    dev = backend.upload(s0, batch)
    ix = backend.vector_index(s0, dev, 2)
    rng = np.random.default_rng(32)
    calls = [(rng.standard_normal((3, 128)).astype(np.float32), k, compare(1, Cmp.Lt, Literal.int64(20 + 7 * i)))
             for i, k in enumerate([1, 5, 10, 32, 64, 100] * 2)]
    want = [backend.vector_topk(s0, ix, dev, p, q, k, DistanceMetric.L2)[:2] for q, k, p in calls]
    got = [None] * len(calls)
    errors = []

    def worker(w):
        s = backend.create_stream()
        try:
            for rep in range(3):
                for i in range(w, len(calls), 4):
                    q, k, p = calls[i]
                    got[i] = backend.vector_topk(s, ix, dev, p, q, k, DistanceMetric.L2)[:2]
        except Exception as e:  # reported below, on the test's thread
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(w,)) for w in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for (gi, gd), (wi, wd) in zip(got, want):
        check(gi, gd, wi, wd)
