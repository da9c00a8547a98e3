"""High-cardinality grouped aggregation at the configured shape: N rows as
uneven RecordBatches of 8K-1M rows (made on the device), int64 group key
uniform over 10M values, int32 x with 2 % NULLs, SUM/MIN/MAX/COUNT(x) under
WHERE f < s for s = 1 %, 50 % and 99 %, folded by one persistent launch
(oxb_aggregate_batches).  Prints one JSON line per selectivity: kernel time
(CUDA events), algorithmic GB/s (f and x's bitmap for every row, key and x
for the kept rows), the whole call's time, the end-to-end time from page-locked
host batches, and the group count.

    python -m oxidelake_b200.bench_batches [--rows N] [--variant V]

--variant pins the kernels as oxb_set_agg_variant does (-1 automatic, 9 the
hash-partitioned passes, 0 the single persistent kernel).  The kernel time
covers the pass over the input that sizes the table and the fold itself.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

GROUP_OUT_BYTES = 8 + 8 + 4 + 4 + 8  # g, SUM(x) i64, MIN(x), MAX(x), COUNT(x)


def kernel_bytes(rows: int, selectivity_pct: float) -> float:
    """Input bytes the fold must read: f (4 B) and x's validity bit for every
    row, then g (8 B) and x (4 B) for the rows the WHERE keeps."""
    return rows * (4 + 1 / 8) + rows * selectivity_pct / 100 * (8 + 4)


def spec_and_pred(selectivity_pct: int):
    from .params import AggregateFunction as F
    from .params import AggregateSpec, Literal, compare
    from .params import Comparison as Cmp

    spec = AggregateSpec(0, [(F.Sum, 1), (F.Min, 1), (F.Max, 1), (F.Count, 1)])
    return spec, compare(2, Cmp.Lt, Literal.int32(selectivity_pct))


def measure(backend, stream, batches, selectivity_pct: int, repeats: int = 2, download: bool = False) -> dict:
    """The fold of `batches` under WHERE f < selectivity_pct: best kernel
    time and call time of `repeats`; the downloaded groups when asked."""
    b, s = backend, stream
    spec, pred = spec_and_pred(selectivity_pct)
    kms, call = [], []
    name, groups, out = None, 0, None
    for _ in range(repeats):
        out = None  # the last call's groups freed first, so the pool already holds this call's memory
        t0 = time.perf_counter()
        out = b.aggregate_batches(s, batches, spec, pred)
        groups = out.num_rows()
        call.append((time.perf_counter() - t0) * 1e3)
        name, kt = b.last_kernel_time()
        kms.append(kt)
    rows = sum(x.num_rows() for x in batches)
    res = {"rows": rows, "batches": len(batches), "selectivity_pct": selectivity_pct, "kernel": name,
           "kernel_ms": min(kms), "call_ms": min(call), "groups": groups,
           "kernel_bytes": kernel_bytes(rows, selectivity_pct)}
    if download:
        res["result"] = b.download(s, out)
    return res


def measure_e2e(backend, stream, host_batches, selectivity_pct: int, repeats: int = 2) -> dict:
    """End to end through the public API: upload of every host batch, the
    fold, the download of the groups; wall clock, best of `repeats`."""
    from .benchkit import batch_bytes

    b, s = backend, stream
    spec, pred = spec_and_pred(selectivity_pct)
    times, d2h = [], 0
    for _ in range(repeats):
        t0 = time.perf_counter()
        devs = [b.upload(s, x) for x in host_batches]
        res = b.download(s, b.aggregate_batches(s, devs, spec, pred))
        times.append((time.perf_counter() - t0) * 1e3)
        d2h = sum(res.column(i).nbytes for i in range(res.num_columns))
        del devs
    return {"e2e_ms": min(times), "h2d_bytes": sum(batch_bytes(x) for x in host_batches), "d2h_bytes": d2h}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=200_000_000)
    ap.add_argument("--distinct", type=int, default=10_000_000)
    ap.add_argument("--repeats", type=int, default=2)
    ap.add_argument("--variant", type=int, default=-1)
    args = ap.parse_args()

    from oxidelake_b200.backend import CudaBackend
    from oxidelake_b200.benchkit import config3_device

    b = CudaBackend(0)
    s = b.create_stream()
    b.set_kernel_timing(True)
    b.set_agg_variant(args.variant, 0)
    devs = config3_device(b, args.rows, args.distinct)
    for sel in (1, 50, 99):
        m = measure(b, s, devs, sel, args.repeats)
        print(json.dumps({
            "workload": "grouped aggregate, many batches", "rows": m["rows"], "batches": m["batches"],
            "distinct": args.distinct, "selectivity_pct": sel, "kernel": m["kernel"],
            "kernel_ms": round(m["kernel_ms"], 3),
            "algorithmic_gbs": round(m["kernel_bytes"] / m["kernel_ms"] / 1e6, 1),
            "call_ms": round(m["call_ms"], 1), "groups": m["groups"], "data": "synthetic",
        }), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
