"""The plain GpuBackend operators at sizes where HBM binds, each timed by
CUDA events around its device passes (last_kernel_time), with its roofline
against the measured HBM copy bandwidth:

- filter_project over the hash-join workload's probe batch (100M rows: fk
  i64, payload f64, qty i32), WHERE qty < 25 (about 48 % kept), projecting
  (fk, payload).  Algorithmic bytes: every column the call reads, read once
  (qty, fk, payload: 20 B a row), and the kept rows written (16 B each).
- probe_join of that batch against the 1M-row build side: reads fk (8 B a
  row) and writes each row's match offset and first build row (12 B a row).
- hash_join gathering (fk, payload, qty, attr) for every match: reads the
  offsets and starts (12 B a probe row) and each match's gathered values,
  and writes them (24 B a match each way; the build side's attr column is
  L2-resident, so its reads count once).
- vector_distance of one L2 query over 4M x 768 Float32 rows (12.6 GB):
  reads 3 KB a row and writes 4 B.

    python -m oxidelake_b200.bench_ops [--probe-rows N] [--vector-rows N]

Each call's result is compared with the oracle's on the same rows (whole
results for filter and join; a 262,144-row slice for the distances).
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def _timed(backend, fn, repeats: int):
    fn()  # first call: allocations warm
    fn()
    kms, call = [], []
    for _ in range(repeats):
        t0 = time.perf_counter()
        r = fn()
        call.append((time.perf_counter() - t0) * 1e3)
        kms.append(backend.last_kernel_time()[1])
        del r
    return float(np.median(kms)), float(np.median(call)), backend.last_kernel_time()[0]


def _line(name: str, kernel: str, kms: float, call_ms: float, algo: float, peak: float, **extra) -> dict:
    achieved = algo / (kms / 1e3) / 1e9
    return {"op": name, "kernel": kernel, "kernel_ms": round(kms, 4), "call_ms": round(call_ms, 4),
            "algorithmic_bytes": int(algo), "achieved_gbs": round(achieved, 1), "peak_gbs": peak,
            "frac": round(achieved / peak, 4), **extra}


def measure_filter_join(backend, stream, build, probe, bdev, pdev, peak: float, repeats: int = 10, check: bool = True):
    """filter_project, probe_join and hash_join on the hash-join workload's
    batches (host copies for the oracle, device copies for the calls)."""
    import oracle
    from compare import assert_columns_equal

    from .params import Comparison as Cmp
    from .params import Literal, compare

    b, s = backend, stream
    n = probe.num_rows
    b.set_kernel_timing(True)
    out = []

    pred = compare(2, Cmp.Lt, Literal.int32(25))
    proj = [0, 1]
    kms, call, kern = _timed(b, lambda: b.filter_project(s, pdev, pred, proj), repeats)
    res = b.filter_project(s, pdev, pred, proj)
    kept = res.num_rows()
    line = _line("filter_project", kern, kms, call, n * 20 + kept * 16, peak, rows=n, kept=kept,
                 query="WHERE qty < 25, projecting (fk, payload)")
    if check:
        got = b.download(s, res)
        want = oracle.filter_project(probe, [(2, 1, oracle.INT32, 25)], proj)
        ok = got.num_rows == want.num_rows
        if ok:
            for i in range(want.num_columns):
                try:
                    assert_columns_equal(got.column(i), want.column(i), want.schema.field(i).name)
                except AssertionError:
                    ok = False
        line["parity"] = {"result": "ok" if ok else "mismatch", "checked": f"all {kept} kept rows, bit for bit"}
        del got, want
    del res
    out.append(line)

    table = b.prepare_join_build(s, bdev, 0)
    kms, call, kern = _timed(b, lambda: b.probe_join(s, pdev, 0, table), repeats)
    matches = b.probe_join(s, pdev, 0, table)
    nm = len(matches)
    out.append(_line("probe_join", kern, kms, call, n * 20, peak, rows=n, matches=nm))

    width = probe.num_columns
    gproj = [0, 1, 2, width + 1]
    kms, call, kern = _timed(b, lambda: b.hash_join(s, pdev, bdev, table, matches, 0, nm, gproj), repeats)
    line = _line("hash_join", kern, kms, call, n * 12 + nm * 24 * 2 + build.num_rows * 4, peak, matches=nm,
                 projection="(fk, payload, qty, attr)")
    if check:
        got = b.download(s, b.hash_join(s, pdev, bdev, table, matches, 0, nm, gproj))
        t = oracle.JoinTable(build, 0)
        m = oracle.JoinMatches(probe, 0, t)
        ok = len(m) == nm and got.num_rows == nm
        if ok:
            want = oracle.hash_join_gather(probe, build, t, m, 0, nm, gproj)
            for i in range(want.num_columns):
                try:
                    assert_columns_equal(got.column(i), want.column(i), want.schema.field(i).name)
                except AssertionError:
                    ok = False
            del want
        line["parity"] = {"result": "ok" if ok else "mismatch",
                          "checked": f"all {nm} joined rows (probe order, then build order), bit for bit"}
        del got, m, t
    out.append(line)
    del matches, table
    b.set_kernel_timing(False)
    return out


def measure_distance(backend, stream, peak: float, rows: int = 4_000_000, dim: int = 768, repeats: int = 10,
                     check_rows: int = 262_144) -> dict:
    """vector_distance of one L2 query over a device-made rows x dim table."""
    import oracle
    import pyarrow as pa
    import torch

    from .benchkit import unit_queries, vector_table
    from .params import DistanceMetric

    b, s = backend, stream
    batch, x, f = vector_table(b, rows, dim, 11, 100)
    q = unit_queries(1, dim, 12)[0]
    b.set_kernel_timing(True)
    kms, call, kern = _timed(b, lambda: b.vector_distance(s, batch, 1, q, DistanceMetric.L2, "d"), repeats)
    line = _line("vector_distance", kern, kms, call, rows * (dim * 4 + 4), peak, rows=rows, dim=dim, metric="l2")
    b.set_kernel_timing(False)
    if check_rows:
        res = b.vector_distance(s, batch, 1, q, DistanceMetric.L2, "d")
        got = b.download_column(s, res, res.num_columns() - 1)
        lo = rows // 2
        hi = min(rows, lo + check_rows)
        xs = x[lo:hi].cpu().numpy()
        part = pa.RecordBatch.from_arrays(
            [pa.FixedSizeListArray.from_arrays(pa.array(xs.reshape(-1)), dim)], names=["emb"])
        want = oracle.vector_distance(part, 0, q, 0)
        gv = got.slice(lo, hi - lo).to_numpy(zero_copy_only=False).view(np.uint32)
        ok = bool((gv == want.to_numpy(zero_copy_only=False).view(np.uint32)).all())
        line["parity"] = {"result": "ok" if ok else "mismatch",
                          "checked": f"rows {lo}..{hi - 1} ({hi - lo} rows), distance bits"}
        del res, got
    del batch, x, f
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return line


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--probe-rows", type=int, default=100_000_000)
    ap.add_argument("--build-rows", type=int, default=1_000_000)
    ap.add_argument("--vector-rows", type=int, default=4_000_000)
    ap.add_argument("--repeats", type=int, default=10)
    ap.add_argument("--no-check", action="store_true")
    args = ap.parse_args()

    from datagen import config2

    from .backend import CudaBackend

    peak = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()).get("hbm_gbs", 6650.0) \
        if (ROOT / "MEASURED_PEAKS.json").exists() else 6650.0
    b = CudaBackend(0)
    s = b.create_stream()
    build, probe = config2(args.build_rows, args.probe_rows)
    bdev, pdev = b.upload(s, build), b.upload(s, probe)
    for line in measure_filter_join(b, s, build, probe, bdev, pdev, peak, args.repeats, not args.no_check):
        print(json.dumps(line), flush=True)
    print(json.dumps(measure_distance(b, s, peak, args.vector_rows, repeats=args.repeats,
                                      check_rows=0 if args.no_check else 262_144)), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
