"""Served mixed stream over HBM-resident tables, against the plain
one-query-at-a-time path at the same offered load.

Resident: a vector table (N rows x 768 FP32, L2-normalised, filter column f
uniform over [0, 1e6)) with its BF16 index, and the hash join + aggregate
tables (1M-row build, probe rows sliced into request batches of 1K-1M rows,
log-uniform).  Requests arrive as a Poisson process: 70 % top-k (k in
{5, 10, 100}, WHERE f < t with selectivity log-uniform in 0.1 %-100 %), 30 %
join + aggregate over one probe slice (WHERE qty > c).  Synthetic data from
fixed seeds.  Prints one JSON line per path: achieved queries/s, p50 and p99
latency (submit to result), and how many top-k requests shared scans.

    python -m oxidelake_b200.bench_serve [--rows N] [--rate QPS] [--seconds S]
"""
from __future__ import annotations

import argparse
import json
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=10_000_000)
    ap.add_argument("--dim", type=int, default=768)
    ap.add_argument("--probe-rows", type=int, default=100_000_000)
    ap.add_argument("--rate", type=float, default=2500.0)
    ap.add_argument("--seconds", type=float, default=3.0)
    ap.add_argument("--plain-seconds", type=float, default=1.0)
    args = ap.parse_args()

    import pyarrow as pa
    import torch

    from datagen import config2
    from oxidelake_b200 import _abi
    from oxidelake_b200.backend import CudaBackend
    from oxidelake_b200.params import AggregateFunction as F
    from oxidelake_b200.params import Comparison as Cmp
    from oxidelake_b200.params import DistanceMetric, Literal, compare

    be = CudaBackend(0)
    s = be.create_stream()
    g = torch.Generator(device="cuda").manual_seed(0x0A11CE + 5)
    x = torch.randn(args.rows, args.dim, device="cuda", generator=g)
    x /= x.norm(dim=1, keepdim=True)
    f = torch.randint(0, 1_000_000, (args.rows,), device="cuda", generator=g, dtype=torch.int64)
    torch.cuda.synchronize()
    vschema = pa.schema([pa.field("f", pa.int64()), pa.field("emb", pa.list_(pa.float32(), args.dim))])
    vdev = be.batch_from_device(
        vschema,
        [_abi.Column(_abi.TYPE_INT64, 1, args.rows, f.data_ptr(), None),
         _abi.Column(_abi.TYPE_VECTOR_F32, args.dim, args.rows, x.data_ptr(), None)],
        args.rows, keep=(x, f),
    )
    ix = be.vector_index(s, vdev, 1)
    build, probe = config2(1_000_000, args.probe_rows, seed=0x0A11CE + 2)
    bdev, pdev = be.upload(s, build), be.upload(s, probe)
    table = be.prepare_join_build(s, bdev, 0)
    rng = np.random.default_rng(0x0A11CE + 5)
    # Request batches: probe slices of 1K-1M rows (log-uniform), views into the resident probe.
    slices = []
    cols = [pdev.column(i) for i in range(3)]
    for _ in range(64):
        n = int(np.exp(rng.uniform(np.log(1_000), np.log(1_000_000))))
        off = int(rng.integers(0, args.probe_rows - n))
        descs = [_abi.Column(c.type, c.dim, n, c.values + off * (8 if c.type in (1, 2) else 4), None) for c in cols]
        slices.append(be.batch_from_device(pdev.schema, descs, n, keep=pdev))
    aggs = [(F.Sum, 0, 1), (F.Sum, 0, 2), (F.CountStar, 0, 0), (F.Avg, 0, 1)]

    def make_requests(count, seed):
        r = np.random.default_rng(seed)
        out = []
        for _ in range(count):
            if r.random() < 0.7:
                q = r.standard_normal(args.dim).astype(np.float32)
                q /= np.linalg.norm(q)
                sel = float(np.exp(r.uniform(np.log(0.001), 0.0)))
                out.append(("topk", q, int(r.choice([5, 10, 100])), max(1, int(sel * 1_000_000))))
            else:
                out.append(("ja", int(r.integers(0, len(slices))), int(r.integers(1, 50))))
        return out

    def run(name, seconds, **cfg):
        count = max(1, int(args.rate * seconds))
        reqs = make_requests(count, 7)
        gaps = np.random.default_rng(8).exponential(1.0 / args.rate, count)
        srv = be.server(**cfg)
        tickets = [None] * count
        ready = threading.Semaphore(0)

        def submit():
            t0 = time.perf_counter()
            due = 0.0
            for i, req in enumerate(reqs):
                due += gaps[i]
                wait = t0 + due - time.perf_counter()
                if wait > 0:
                    time.sleep(wait)
                if req[0] == "topk":
                    tickets[i] = srv.submit_topk(ix, vdev, None, req[1], req[2], DistanceMetric.L2,
                                                 query_leaf=(0, Cmp.Lt, Literal.int64(req[3])))
                else:
                    tickets[i] = srv.submit_join_aggregate(slices[req[1]], 0, table,
                                                           compare(2, Cmp.Gt, Literal.int32(req[2])), (1, 1), aggs)
                ready.release()

        th = threading.Thread(target=submit)
        th.start()
        for i, req in enumerate(reqs):
            ready.acquire()
            if req[0] == "topk":
                srv.wait_topk(tickets[i], req[2])
            else:
                b, _ = srv.wait_batch(tickets[i])
                b.free()
        th.join()
        st = srv.stats()
        srv.close()
        line = {
            "path": name, "offered_qps": args.rate, "requests": count, "qps": round(st["qps"], 1),
            "p50_ms": round(st["p50_us"] / 1e3, 3), "p99_ms": round(st["p99_us"] / 1e3, 3),
            "dispatches": st["dispatches"], "topk_requests_sharing_scans": st["batched_queries"],
            "peak_admitted_gb": round(st["peak_bytes"] / 1e9, 2),
            "config": {"rows": args.rows, "dim": args.dim, "probe_rows": args.probe_rows, "mix": "70% top-k / 30% join+aggregate",
                       "budget_gb": 150, "data": "synthetic"},
        }
        print(json.dumps(line), flush=True)
        return line

    run("served", args.seconds, workers=2, max_batch=256)
    run("plain", args.plain_seconds, workers=1, max_batch=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
