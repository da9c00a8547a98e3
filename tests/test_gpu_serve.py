"""The serving loop on the B200: a mixed stream of top-k and join-aggregate
requests submitted together gives, request by request, the same result as
the direct call made alone (top-k bit for bit; Float64 sums to the stated
tolerance), while top-k requests that queue together share scans."""
import numpy as np
import pyarrow as pa
import pytest

from compare import assert_batches_equal
from datagen import config2
from oxidelake_b200 import errors
from oxidelake_b200.params import AggregateFunction as F
from oxidelake_b200.params import Comparison as Cmp
from oxidelake_b200.params import DistanceMetric, Literal, compare

pytestmark = pytest.mark.gpu

AGGS = [(F.Sum, 0, 1), (F.Sum, 0, 2), (F.CountStar, 0, 0), (F.Avg, 0, 1)]


@pytest.fixture(scope="module")
def resident(backend, stream):
    rng = np.random.default_rng(77)
    n, dim = 30_000, 128
    v = rng.standard_normal((n, dim)).astype(np.float32)
    vec = pa.RecordBatch.from_arrays(
        [pa.array(rng.integers(0, 1000, n), pa.int64()), pa.FixedSizeListArray.from_arrays(pa.array(v.reshape(-1)), dim)],
        names=["f", "emb"],
    )
    vdev = backend.upload(stream, vec)
    ix = backend.vector_index(stream, vdev, 1)
    build, probe = config2(5_000, 400_000, seed=78)
    bdev, pdev = backend.upload(stream, build), backend.upload(stream, probe)
    table = backend.prepare_join_build(stream, bdev, 0)
    return dict(vdev=vdev, ix=ix, dim=dim, pdev=pdev, table=table, rng=rng)


def requests(R, count):
    rng = np.random.default_rng(5)
    out = []
    for i in range(count):
        if i % 10 < 7:
            out.append(("topk", rng.standard_normal(R["dim"]).astype(np.float32), int(rng.choice([5, 10, 100])),
                        DistanceMetric.L2 if i % 3 else DistanceMetric.Cosine, int(rng.integers(1, 1000))))
        else:
            out.append(("ja", int(rng.integers(1, 50))))
    return out


def direct(backend, stream, R, req):
    if req[0] == "topk":
        _, q, k, metric, lit = req
        ids, dist, _ = backend.vector_topk(stream, R["ix"], R["vdev"], None, q[None, :], k, metric,
                                           query_leaf=(0, Cmp.Lt, [Literal.int64(lit)]))
        return ids[0], dist[0]
    return backend.download(stream, backend.join_aggregate(stream, R["pdev"], 0, R["table"],
                                                           compare(2, Cmp.Gt, Literal.int32(req[1])), (1, 1), AGGS))


def served(backend, stream, R, reqs, **cfg):
    srv = backend.server(**cfg)
    tickets = []
    for req in reqs:
        if req[0] == "topk":
            _, q, k, metric, lit = req
            tickets.append(srv.submit_topk(R["ix"], R["vdev"], None, q, k, metric,
                                           query_leaf=(0, Cmp.Lt, Literal.int64(lit))))
        else:
            tickets.append(srv.submit_join_aggregate(R["pdev"], 0, R["table"], compare(2, Cmp.Gt, Literal.int32(req[1])),
                                                     (1, 1), AGGS))
    results = []
    for req, t in zip(reqs, tickets):
        if req[0] == "topk":
            ids, dist, lat = srv.wait_topk(t, req[2])
            results.append((ids, dist))
        else:
            b, lat = srv.wait_batch(t)
            results.append(backend.download(stream, b))
        assert lat > 0
    st = srv.stats()
    srv.close()
    return results, st


def check_same(reqs, got, want):
    for req, g, w in zip(reqs, got, want):
        if req[0] == "topk":
            assert (g[0] == w[0]).all()
            assert ((g[1].view(np.uint32) == w[1].view(np.uint32)) | (np.isnan(g[1]) & np.isnan(w[1]))).all()
        else:
            assert_batches_equal(g, w, float_sum_cols=(1, 4))


def test_mixed_stream_equals_alone(backend, stream, resident):
    reqs = requests(resident, 80)
    want = [direct(backend, stream, resident, r) for r in reqs]
    got, st = served(backend, stream, resident, reqs)
    check_same(reqs, got, want)
    assert st["completed"] == len(reqs)
    assert st["batched_queries"] > 0, st  # queued requests shared launches
    assert st["dispatches"] < len(reqs)
    assert 0 < st["p50_us"] <= st["p99_us"] and st["qps"] > 0


def test_one_at_a_time_mode(backend, stream, resident):
    reqs = requests(resident, 12)
    want = [direct(backend, stream, resident, r) for r in reqs]
    got, st = served(backend, stream, resident, reqs, workers=1, max_batch=1)
    check_same(reqs, got, want)
    assert st["batched_queries"] == 0 and st["dispatches"] == len(reqs)


def test_admission_refuses_what_never_fits(backend, stream, resident):
    srv = backend.server(memory_budget=1 << 20)
    q = np.zeros(resident["dim"], np.float32)
    with pytest.raises(errors.AdmissionRejected):
        srv.submit_topk(resident["ix"], resident["vdev"], None, q, 10, DistanceMetric.L2)
    assert srv.stats()["rejected"] == 1
    srv.close()


def test_admission_defers_until_memory_frees(backend, stream, resident):
    """A budget with room for two requests' device memory and ten requests
    submitted at once: the server runs at most two at a time (the others wait
    in the queue until memory frees, with workers idle), every request
    completes, and each result equals its direct call."""
    rng = np.random.default_rng(11)
    reqs = []
    for i in range(10):  # distinct WHERE literals: no two share a scan
        reqs.append((rng.standard_normal(resident["dim"]).astype(np.float32), int(rng.choice([5, 10])), 100 + 83 * i))
    # One request alone: the server's estimate of its device memory.
    srv = backend.server(workers=1)
    q, k, lit = reqs[0]
    srv.wait_topk(srv.submit_topk(resident["ix"], resident["vdev"], compare(0, Cmp.Lt, Literal.int64(lit)), q, k,
                                  DistanceMetric.L2), k)
    one = srv.stats()["peak_bytes"]
    srv.close()
    assert one > 0
    budget = int(2.5 * one)
    srv = backend.server(memory_budget=budget, workers=6, max_batch=256)
    tickets = [srv.submit_topk(resident["ix"], resident["vdev"], compare(0, Cmp.Lt, Literal.int64(lit)), q, k,
                               DistanceMetric.L2) for q, k, lit in reqs]
    got = [srv.wait_topk(t, k) for t, (_, k, _) in zip(tickets, reqs)]
    st = srv.stats()
    srv.close()
    assert st["completed"] == 10 and st["rejected"] == 0 and st["dispatches"] == 10
    assert st["peak_bytes"] <= budget and st["peak_bytes"] < 3 * one
    for (q, k, lit), (ids, dist, _) in zip(reqs, got):
        want_ids, want_dist, _ = backend.vector_topk(stream, resident["ix"], resident["vdev"],
                                                     compare(0, Cmp.Lt, Literal.int64(lit)), q[None, :], k,
                                                     DistanceMetric.L2)
        assert (ids == want_ids[0]).all()
        assert (dist.view(np.uint32) == want_dist[0].view(np.uint32)).all()


def test_join_aggregates_share_launches(backend, stream, resident):
    """Join-aggregate requests queued together (probe batches of one shape,
    different WHERE literals) run as shared launches; each result equals its
    direct call."""
    reqs = [("ja", 5 + 3 * i) for i in range(12)]
    want = [direct(backend, stream, resident, r) for r in reqs]
    got, st = served(backend, stream, resident, reqs, workers=1, max_batch=64)
    check_same(reqs, got, want)
    assert st["completed"] == 12 and st["dispatches"] < 12 and st["batched_queries"] > 1, st
