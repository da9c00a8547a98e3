"""The checks bench.py runs at the measured sizes, on the CPU: the oracle's
top-k read in chunks of kept rows and merged equals one pass over the table,
and the parity helper reports a planted difference.  CPU only."""
import numpy as np
import pyarrow as pa
import pytest
import torch

import bench
import oracle


@pytest.mark.parametrize("metric", [0, 1], ids=["l2", "cosine"])
def test_chunked_oracle_topk_equals_one_pass(metric):
    rng = np.random.default_rng(3)
    n, d = 5000, 32
    x = rng.standard_normal((n, d)).astype(np.float32)
    x[100:200] = x[0]  # ties, broken by row id across chunk boundaries
    x[300:305] = 0.0  # zero norms: NaN cosine distances sort last
    f = rng.integers(0, 100, n)
    q = rng.standard_normal((5, d)).astype(np.float32)
    ids, dist, _, kept = bench.oracle_topk_kept(torch.from_numpy(x), torch.from_numpy(f), 30, q, 10, metric, 2, chunk=700)
    table = pa.RecordBatch.from_arrays([pa.array(f), pa.FixedSizeListArray.from_arrays(pa.array(x.reshape(-1)), d)],
                                       names=["f", "emb"])
    want_ids, want_d = oracle.vector_topk(table, 1, q, 10, metric, [(0, 1, 1, 30)], threads=2)
    assert kept == int((f < 30).sum())
    assert (ids == want_ids).all()
    assert (dist.view(np.uint32) == want_d.view(np.uint32)).all()


def test_parity_reports_a_planted_difference():
    build, probe = bench.gen_data(0, 2000, 50_000)
    want, _ = bench.oracle_join_aggregate(build, probe, 2)
    assert bench.parity(want, want, float_cols=(1, 4))["result"] == "ok"
    counts = want.column(3).to_numpy().copy()
    counts[7] += 1  # one COUNT(*) off by one
    bad = pa.RecordBatch.from_arrays([want.column(i) if i != 3 else pa.array(counts) for i in range(want.num_columns)],
                                     schema=want.schema)
    p = bench.parity(bad, want, float_cols=(1, 4))
    assert p["result"] == "mismatch" and "COUNT(*)" in p["detail"]
