"""High-cardinality grouped aggregation at the configured shape: N rows as
uneven RecordBatches of 8K-1M rows, int64 group key uniform over 10M values,
int32 x with 2 % NULLs, SUM/MIN/MAX/COUNT(x) under WHERE f < s for s = 1 %,
50 % and 99 %, folded by one persistent launch (oxb_aggregate_batches).
Prints one JSON line per selectivity: kernel time (CUDA events), algorithmic
GB/s (f and its bitmap for every row, key and x for the kept rows), the
whole call's time and the group count.

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
sys.path.insert(0, str(ROOT / "tests"))


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=200_000_000)
    ap.add_argument("--distinct", type=int, default=10_000_000)
    ap.add_argument("--repeats", type=int, default=2)
    ap.add_argument("--variant", type=int, default=-1)
    args = ap.parse_args()

    from datagen import config3_batches
    from oxidelake_b200.backend import CudaBackend
    from oxidelake_b200.params import AggregateFunction as F
    from oxidelake_b200.params import AggregateSpec, Literal, compare
    from oxidelake_b200.params import Comparison as Cmp

    batches = config3_batches(args.rows, args.distinct)
    b = CudaBackend(0)
    s = b.create_stream()
    b.set_kernel_timing(True)
    b.set_agg_variant(args.variant, 0)
    devs = [b.upload(s, x) for x in batches]
    spec = AggregateSpec(0, [(F.Sum, 1), (F.Min, 1), (F.Max, 1), (F.Count, 1)])
    for sel in (1, 50, 99):
        pred = compare(2, Cmp.Lt, Literal.int32(sel))
        kms, call = [], []
        for _ in range(args.repeats):
            t0 = time.perf_counter()
            out = b.aggregate_batches(s, devs, spec, pred)
            groups = out.num_rows()
            call.append((time.perf_counter() - t0) * 1e3)
            name, kt = b.last_kernel_time()
            kms.append(kt)
        gb = args.rows * (4 + 1 / 8) / 1e9 + args.rows * sel / 100 * (8 + 4 + 1 / 8) / 1e9
        ms = min(kms)
        print(json.dumps({
            "workload": "grouped aggregate, many batches", "rows": args.rows, "batches": len(batches),
            "distinct": args.distinct, "selectivity_pct": sel, "kernel": name, "kernel_ms": round(ms, 3),
            "algorithmic_gbs": round(gb / ms * 1e3, 1), "call_ms": round(min(call), 1), "groups": groups,
            "data": "synthetic",
        }), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
