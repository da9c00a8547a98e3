"""Filter + grouped aggregate at the configured shape: 1M rows (id i64, k i64
uniform in [0, 10), v f64 uniform in [0, 10), emb f32[8]),
SELECT k, SUM(v), COUNT(*) WHERE k >= 2 AND v < 4.0 GROUP BY k.

Prints one JSON line per path:
- "fused": the WHERE folded into the aggregate (one pass over k and v),
  CUDA-event time of the aggregate kernel and the whole call;
- "two-step": filter_project of (k, v), then the aggregate of the result
  (the whole call's time only);
- "e2e": upload of the query's columns (k, v) from page-locked host memory,
  the fused query, the download of the groups; and the same from pageable
  memory.
The input is 16 MB (k and v), far below L2: these times are launch and
latency bound, not HBM bound.

    python -m oxidelake_b200.bench_filter_agg [--rows N] [--repeats R]
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

QUERY = "SELECT k, SUM(v), COUNT(*) FROM t WHERE k >= 2 AND v < 4.0 GROUP BY k"


def measure(backend, stream, batch, repeats: int = 20) -> dict:
    """Times the config-1 query on `batch` (columns id, k, v, emb) three
    ways; returns the figures and the fused path's downloaded result."""
    from .benchkit import batch_bytes, pinned_batch
    from .params import AggregateFunction as F
    from .params import AggregateSpec, Literal, and_, compare
    from .params import Comparison as Cmp

    b, s = backend, stream
    dev = b.upload(s, batch)
    pred = and_(compare(1, Cmp.GtEq, Literal.int64(2)), compare(2, Cmp.Lt, Literal.float64(4.0)))
    spec = AggregateSpec(1, [(F.Sum, 2), (F.CountStar, 0)])
    spec2 = AggregateSpec(0, [(F.Sum, 1), (F.CountStar, 0)])
    rows = batch.num_rows
    algo_bytes = rows * 16  # k and v

    def timed(fn):
        fn()  # warm-up (tuning, first-call set-up)
        fn()
        kms, call = [], []
        for _ in range(repeats):
            t0 = time.perf_counter()
            fn()
            call.append((time.perf_counter() - t0) * 1e3)
            kms.append(b.last_kernel_time()[1])
        return min(kms), min(call)

    def fused():
        return b.aggregate(s, dev, spec, pred).num_rows()

    def two_step():
        f = b.filter_project(s, dev, pred, [1, 2])
        return b.aggregate(s, f, spec2).num_rows()

    out = {"rows": rows, "algorithmic_bytes": algo_bytes}
    kms, call = timed(fused)
    out["kernel"] = b.last_kernel_time()[0]
    out["kernel_ms"] = kms
    out["call_ms"] = call
    out["two_step_call_ms"] = timed(two_step)[1]
    out["result"] = b.download(s, b.aggregate(s, dev, spec, pred))

    kv = batch.select([1, 2])  # the columns the query reads
    pred_kv = and_(compare(0, Cmp.GtEq, Literal.int64(2)), compare(1, Cmp.Lt, Literal.float64(4.0)))
    spec_kv = AggregateSpec(0, [(F.Sum, 1), (F.CountStar, 0)])
    pinned, keep = pinned_batch(b, kv)

    def e2e(src):
        d = b.upload(s, src)
        return b.download(s, b.aggregate(s, d, spec_kv, pred_kv))

    for name, src in (("e2e", pinned), ("e2e_pageable", kv)):
        res = e2e(src)
        call = []
        for _ in range(repeats):
            t0 = time.perf_counter()
            res = e2e(src)
            call.append((time.perf_counter() - t0) * 1e3)
        out[name + "_ms"] = min(call)
        out[name + "_d2h_bytes"] = sum(res.column(i).nbytes for i in range(res.num_columns))
    out["e2e_h2d_bytes"] = batch_bytes(kv)
    del keep
    return out


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=1_000_000)
    ap.add_argument("--repeats", type=int, default=20)
    args = ap.parse_args()

    from datagen import config1
    from oxidelake_b200.backend import CudaBackend

    b = CudaBackend(0)
    s = b.create_stream()
    b.set_kernel_timing(True)
    m = measure(b, s, config1(args.rows), args.repeats)
    gb = m["algorithmic_bytes"]
    for path, ms, kms in (("fused", m["call_ms"], m["kernel_ms"]), ("two-step", m["two_step_call_ms"], None),
                          ("e2e", m["e2e_ms"], None), ("e2e-pageable", m["e2e_pageable_ms"], None)):
        print(json.dumps({
            "workload": "filter + grouped aggregate", "query": QUERY, "path": path, "rows": args.rows,
            "kernel_ms": round(kms, 4) if kms is not None else None, "call_ms": round(ms, 4),
            "algorithmic_gbs_call": round(gb / (ms / 1e3) / 1e9, 1), "data": "synthetic",
        }), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
