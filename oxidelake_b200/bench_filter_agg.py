"""Filter + grouped aggregate at the configured shape: 1M rows (id i64, k i64
uniform in [0, 10), v f64 uniform in [0, 10), emb f32[8]),
SELECT k, SUM(v), COUNT(*) WHERE k >= 2 AND v < 4.0 GROUP BY k.

Prints one JSON line per path:
- "fused": the WHERE folded into the aggregate (one pass over k and v),
  CUDA-event time of the aggregate kernel and the whole call;
- "two-step": filter_project of (k, v), then the aggregate of the result
  (the whole call's time only);
- "e2e": upload of the query's columns (k, v) from pageable host memory,
  the fused query, the download of the groups.
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


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=1_000_000)
    ap.add_argument("--repeats", type=int, default=20)
    args = ap.parse_args()

    from datagen import config1
    from oxidelake_b200.backend import CudaBackend
    from oxidelake_b200.params import AggregateFunction as F
    from oxidelake_b200.params import AggregateSpec, Literal, and_, compare
    from oxidelake_b200.params import Comparison as Cmp

    batch = config1(args.rows)
    b = CudaBackend(0)
    s = b.create_stream()
    b.set_kernel_timing(True)
    dev = b.upload(s, batch)
    pred = and_(compare(1, Cmp.GtEq, Literal.int64(2)), compare(2, Cmp.Lt, Literal.float64(4.0)))
    spec = AggregateSpec(1, [(F.Sum, 2), (F.CountStar, 0)])
    spec2 = AggregateSpec(0, [(F.Sum, 1), (F.CountStar, 0)])
    algo_bytes = args.rows * 16  # k and v

    def timed(fn):
        fn()  # warm-up (tuning, first-call set-up)
        fn()
        kms, call = [], []
        for _ in range(args.repeats):
            t0 = time.perf_counter()
            fn()
            call.append((time.perf_counter() - t0) * 1e3)
            kms.append(b.last_kernel_time()[1])
        return min(kms), min(call)

    def fused():
        out = b.aggregate(s, dev, spec, pred)
        return out.num_rows()

    def two_step():
        f = b.filter_project(s, dev, pred, [1, 2])
        out = b.aggregate(s, f, spec2)
        return out.num_rows()

    for name, fn in (("fused", fused), ("two-step", two_step)):
        kms, call = timed(fn)
        print(json.dumps({
            "workload": "filter + grouped aggregate", "path": name, "rows": args.rows,
            "kernel_ms": round(kms, 4) if name == "fused" else None,
            "call_ms": round(call, 4), "algorithmic_gbs_call": round(algo_bytes / (call / 1e3) / 1e9, 1),
            "data": "synthetic",
        }), flush=True)

    kv = batch.select([1, 2])  # the columns the query reads
    pred_kv = and_(compare(0, Cmp.GtEq, Literal.int64(2)), compare(1, Cmp.Lt, Literal.float64(4.0)))
    spec_kv = AggregateSpec(0, [(F.Sum, 1), (F.CountStar, 0)])

    def e2e():
        d = b.upload(s, kv)
        return b.download(s, b.aggregate(s, d, spec_kv, pred_kv)).num_rows

    e2e()
    call = []
    for _ in range(args.repeats):
        t0 = time.perf_counter()
        e2e()
        call.append((time.perf_counter() - t0) * 1e3)
    ms = min(call)
    print(json.dumps({
        "workload": "filter + grouped aggregate", "path": "e2e", "rows": args.rows, "call_ms": round(ms, 4),
        "algorithmic_gbs_call": round(algo_bytes / (ms / 1e3) / 1e9, 1), "data": "synthetic",
    }), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
