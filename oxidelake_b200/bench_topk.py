"""Vector top-k at the configured shape: N rows x 768 FP32 (L2-normalised,
seeded on the device), an int64 filter column uniform in [0, 100), 256 queries
from the same distribution, top-10 under WHERE f < 30, l2 and cosine.
Prints one JSON line per metric:
- the scan's CUDA-event time: the copy of the kept rows to a compacted table
  (a WHERE that keeps at most 40 % of the rows) plus the tcgen05 scan;
- TFLOP/s: 2 x queries x kept rows x dim, the algorithmic flops (the rows
  the WHERE drops need no distance);
- the whole call's time (queries from host memory, ids and distances back
  to host memory: the end-to-end time), how many queries took the exact
  path, and the BF16 score error against FP64 over the re-ranked candidates.

    python -m oxidelake_b200.bench_topk [--rows N] [--repeats R]
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))

SEED = 0x0A11CE + 4


def measure(backend, stream, ix, batch, queries, k: int, metric, pred, repeats: int = 3) -> dict:
    """Best scan time (CUDA events) and call time of `repeats` top-k calls;
    the last call's ids, distances and statistics."""
    b, s = backend, stream
    scan, call = [], []
    ids = dist = st = None
    for _ in range(repeats):
        t0 = time.perf_counter()
        ids, dist, st = b.vector_topk(s, ix, batch, pred, queries, k, metric)
        call.append((time.perf_counter() - t0) * 1e3)
        scan.append(b.last_kernel_time()[1])
    return {"scan_ms": min(scan), "call_ms": min(call), "ids": ids, "dist": dist, "stats": st,
            "h2d_bytes": int(queries.nbytes), "d2h_bytes": int(ids.nbytes + dist.nbytes)}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=10_000_000)
    ap.add_argument("--dim", type=int, default=768)
    ap.add_argument("--queries", type=int, default=256)
    ap.add_argument("--k", type=int, default=10)
    ap.add_argument("--repeats", type=int, default=3)
    args = ap.parse_args()

    import torch

    from oxidelake_b200.backend import CudaBackend
    from oxidelake_b200.benchkit import unit_queries, vector_table
    from oxidelake_b200.params import Comparison as Cmp
    from oxidelake_b200.params import DistanceMetric, Literal, compare

    n, d = args.rows, args.dim
    b = CudaBackend(0)
    s = b.create_stream()
    b.set_kernel_timing(True)
    batch, x, f = vector_table(b, n, d, SEED, 100)
    kept = int((f < 30).sum().item())
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ix = b.vector_index(s, batch, 1)
    build_s = time.perf_counter() - t0
    q = unit_queries(args.queries, d, 5)
    pred = compare(0, Cmp.Lt, Literal.int64(30))
    for metric in (DistanceMetric.L2, DistanceMetric.Cosine):
        m = measure(b, s, ix, batch, q, args.k, metric, pred, args.repeats)
        st = m["stats"]
        flops = 2.0 * args.queries * kept * d
        print(json.dumps({
            "workload": "vector top-k", "metric": metric.name.lower(), "rows": n, "kept_rows": kept, "dim": d,
            "queries": args.queries, "k": args.k, "filter": "f < 30 (30%)", "scan_ms": round(m["scan_ms"], 3),
            "tflops": round(flops / m["scan_ms"] / 1e9, 1),
            "call_ms": round(m["call_ms"], 3), "index_build_s": round(build_s, 3), "exact_queries": st["exact_queries"],
            "reranked": st["reranked"], "bf16_score_error_max": st["max_score_error"],
            "bf16_score_error_mean": st["mean_score_error"], "data": "synthetic",
        }), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
