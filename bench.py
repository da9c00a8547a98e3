#!/usr/bin/env python
"""Benchmark of the GPU operator path.

Headline workload (one step): `probe JOIN build ON fk = key WHERE qty > 10
GROUP BY attr` computing SUM(payload), SUM(qty), COUNT(*), AVG(payload), over
a 1M-row build side (unique int64 key, int32 attr U[0,1000)) and a 100M-row
probe side (int64 fk Zipf(1.1) over the build keys with 5% non-matching,
float64 payload U(0,100), int32 qty U[1,50]); seeded synthetic data.  One
step builds the join table on the device and runs the fused probe ->
filter -> aggregate pass, then reads the 1000-group result back.  The last
step's result is checked against the oracle over all 100M probe rows (that
run is also the CPU baseline), and the line says "parity": "ok" or
"mismatch"; a mismatch exits non-zero.

On one GPU the line also carries `per_config`: each other configured
workload measured once, with its roofline fraction, end-to-end time, the
oracle on the host cores and a parity check at the measured size:
  config1  SELECT k, SUM(v), COUNT(*) WHERE k >= 2 AND v < 4.0 GROUP BY k, 1M rows
  config3  200M rows in uneven batches, 10M distinct Int64 keys, SUM/MIN/MAX/COUNT
           of a nullable Int32 under WHERE f < s, s = 1, 50, 99 %
  config4  top-10 of 256 queries over 10M x 768 FP32 rows, WHERE f < 30 (30 %),
           l2 and cosine (parity on 16 of the 256 queries over every row)
  config5  the served mixed stream against the plain one-query-at-a-time path
  plain_operators  filter_project, probe_join + hash_join over the headline's
           100M-row probe, vector_distance over 4M x 768 rows, each against
           the measured HBM bandwidth (parity: whole results; a distance slice)

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--configs 1,3,4,5,ops]

N > 1 (one process per GPU under torchrun): weak scaling, each rank its own
100M-row probe shard and the same build side; the per-rank group partials are
exchanged with NCCL all_gather and merged.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

BUILD_ROWS = 1_000_000
PROBE_ROWS = 100_000_000
PROBE_ROW_BYTES = 8 + 8 + 4  # fk, payload, qty
BUILD_ROW_BYTES = 8 + 4  # key, attr
GROUP_OUT_BYTES = 4 + 8 + 8 + 8 + 8  # attr, SUM(payload), SUM(qty), COUNT(*), AVG
WORKLOAD = "hash join + aggregate: build 1M (unique i64 key, i32 attr), probe 100M (i64 fk Zipf 1.1, 5% misses; f64 payload; i32 qty), WHERE qty > 10 GROUP BY attr: SUM, SUM, COUNT(*), AVG"


def algorithmic_bytes(build_rows: int, probe_rows: int, groups: int = 1000) -> int:
    """Bytes the query must move at least once: the probe and build columns
    it reads and the groups it writes."""
    return probe_rows * PROBE_ROW_BYTES + build_rows * BUILD_ROW_BYTES + groups * GROUP_OUT_BYTES


def peaks(kind: str = "hbm"):
    """(peak, "measured" | "fallback"): HBM copy GB/s, or dense bf16 TFLOP/s
    (the burst figure, for a kernel timed on its own)."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return (float(d["hbm_gbs"]) if kind == "hbm" else float(d["bf16_tflops"])), "measured"
    return (6650.0 if kind == "hbm" else 1590.0), "fallback"


def profiled_traffic(kernel: str):
    """DRAM bytes per launch from the committed ncu summary, if one exists."""
    for f in sorted((ROOT / "profiles").glob(f"{kernel}*.md")):
        for line in f.read_text().splitlines():
            if line.strip().startswith("traffic_bytes_per_launch:"):
                try:
                    return float(line.split(":", 1)[1].strip())
                except ValueError:
                    return None
    return None


def profile_kernel(variant_name: str) -> str:
    """The kernel a join-aggregate variant name (as last_kernel_time reports
    it) launches, which names its committed ncu summary."""
    if "lean4" in variant_name:
        return "agg_lean4_join_kernel"
    if "lean" in variant_name:
        return "agg_lean_join_kernel"
    if "stream" in variant_name:
        return "agg_fstream_join_kernel"
    if "vec" in variant_name:
        return "agg_fusedv_join_kernel"
    if "fused" in variant_name:
        return "agg_fused_join_kernel"
    return "agg_join_kernel"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons read from NVML every 2 ms
    by a thread while the timed region runs (read-only queries; no setting of
    the GPU is touched)."""

    REASONS = {
        "hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
        "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
        "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
        "sw_power_cap": "nvmlClocksEventReasonSwPowerCap",
        "hw_power_brake_slowdown": "nvmlClocksEventReasonHwPowerBrakeSlowdown",
    }

    def __init__(self, index: int):
        self.index = index
        self.samples = []  # (sm_mhz, reasons bitmask)
        self.max_mhz = None
        self.handle = None
        self.stop = threading.Event()
        self.thread = None

    def __enter__(self):
        try:
            import pynvml as nv
            import torch

            nv.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            if not uuid.startswith("GPU-"):
                uuid = "GPU-" + uuid
            self.nv = nv
            self.handle = nv.nvmlDeviceGetHandleByUUID(uuid)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(self.handle, nv.NVML_CLOCK_SM))
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
        except Exception as e:  # NVML missing: no clock record
            self.error = repr(e)
            self.handle = None
        return self

    def _poll(self):
        nv = self.nv
        while not self.stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM)
                why = nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
                self.samples.append((float(mhz), int(why)))
            except Exception:
                pass
            time.sleep(0.002)

    def __exit__(self, *exc):
        self.stop.set()
        if self.thread:
            self.thread.join(timeout=5)

    def summary(self):
        if not self.samples:
            return None
        reasons = set()
        for _, why in self.samples:
            for name, const in self.REASONS.items():
                if why & getattr(self.nv, const, 0):
                    reasons.add(name)
        return {
            "sm_mhz": float(np.median([m for m, _ in self.samples])),
            "sm_max_mhz": self.max_mhz,
            "reasons": sorted(reasons),
            "samples": len(self.samples),
            "source": "NVML, every 2 ms during the timed steps",
        }


def gen_data(rank: int, build_rows: int, probe_rows: int):
    from datagen import config2

    # The build side is the same on every rank; each rank probes its own shard.
    build, _ = config2(build_rows, 0, seed=0x0A11CE + 2)
    _, probe = config2(build_rows, probe_rows, seed=0x0A11CE + 2 + 1000 * (rank + 1))
    return build, probe


CONFIG2_CONFIG = {
    "workload": WORKLOAD,
    "build_rows": BUILD_ROWS,
    "probe_rows_per_gpu": PROBE_ROWS,
    "l2": "inputs (2.0 GB per GPU) larger than L2; no flush",
}
JOIN_AGGS = ((0, 0, 1), (0, 0, 2), (5, 0, 0), (4, 0, 1))  # SUM(payload), SUM(qty), COUNT(*), AVG(payload)
QTY_GT_10 = [(2, 3, 3, 10)]  # oracle leaf: qty > 10 (Int32 literal)


def oracle_join_aggregate(build, probe, threads: int):
    """The oracle's result over every probe row, and its wall time."""
    import oracle

    t0 = time.perf_counter()
    res = oracle.join_aggregate(probe, build, 0, 0, QTY_GT_10, (1, 1), list(JOIN_AGGS), threads=threads)
    return res, time.perf_counter() - t0


def parity(got, want, float_cols=(), scale=None) -> dict:
    """Bit-exact except `float_cols` (1e-12 of max(|result|, scale))."""
    from compare import assert_batches_equal

    try:
        assert_batches_equal(got, want, float_sum_cols=float_cols, scale=scale)
        return {"result": "ok", "groups": want.num_rows}
    except AssertionError as e:
        return {"result": "mismatch", "detail": str(e)[:300]}


def run_reference(args) -> None:
    """The reference's CPU path for the same query over the same 100M probe
    rows: the oracle port of cpu/kernels.rs (JoinTable + JoinMatches +
    GroupedAggregator), run as DataFusion would over partitions — one thread
    per host core, partials merged."""
    import oracle

    threads = oracle.cpu_threads()
    build, probe = gen_data(0, args.build_rows, args.probe_rows)
    times = []
    res = None
    for i in range(args.warmup + args.steps):
        res, dt = oracle_join_aggregate(build, probe, threads)
        if i >= args.warmup:
            times.append(dt)
    ms = 1e3 * float(np.mean(times))
    gbs = algorithmic_bytes(args.build_rows, probe.num_rows) / (ms / 1e3) / 1e9
    sample = f"the whole workload each step: probe {probe.num_rows} rows x build {args.build_rows} rows"
    config = dict(CONFIG2_CONFIG, build_rows=args.build_rows, probe_rows_per_gpu=args.probe_rows,
                  groups=res.num_rows, parallelism="single")
    line = {
        "impl": "reference",
        "metric": "GB/s",
        "value": round(gbs, 3),
        "unit": "GB/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int64/f64",
        "data": "synthetic",
        "config": config,
        "rows_per_s": round(probe.num_rows / (ms / 1e3)),
        "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config1_block(backend, stream, threads: int) -> dict:
    """Config 1: SELECT k, SUM(v), COUNT(*) WHERE k >= 2 AND v < 4.0 GROUP BY k, 1M rows."""
    import oracle
    from datagen import config1

    from oxidelake_b200 import bench_filter_agg

    batch = config1(1_000_000)
    m = bench_filter_agg.measure(backend, stream, batch, repeats=20)
    leaves = [(1, 4, 1, 2), (2, 1, 2, 4.0)]
    times = []
    for _ in range(5):
        t0 = time.perf_counter()
        want = oracle.aggregate(batch, 1, [(0, 2), (5, 0)], leaves)
        times.append(time.perf_counter() - t0)
    peak, kind = peaks("hbm")
    gb = m["algorithmic_bytes"]
    achieved = gb / (m["kernel_ms"] / 1e3) / 1e9
    return {
        "workload": bench_filter_agg.QUERY + " (1M rows: id i64, k i64 U[0,10), v f64 U[0,10), emb f32[8])",
        "roofline": {"bound": "hbm (16 MB input sits in L2: launch- and latency-bound)", "kernel": m["kernel"],
                     "kernel_ms": round(m["kernel_ms"], 4), "algorithmic_bytes_per_launch": gb,
                     "achieved": round(achieved, 1), "peak": peak, "peak_kind": kind, "unit": "GB/s",
                     "frac": round(achieved / peak, 4)},
        "call_ms": round(m["call_ms"], 4),
        "two_step_call_ms": round(m["two_step_call_ms"], 4),
        "e2e": {"value": round(gb / (m["e2e_ms"] / 1e3) / 1e9, 2), "unit": "GB/s", "ms": round(m["e2e_ms"], 4),
                "h2d_bytes_per_step": m["e2e_h2d_bytes"], "d2h_bytes_per_step": m["e2e_d2h_bytes"],
                "from": "page-locked host columns (k, v)",
                "pageable_ms": round(m["e2e_pageable_ms"], 4)},
        "cpu_baseline": {"value": round(gb / min(times) / 1e9, 3), "unit": "GB/s", "cores": 1, "kind": "port",
                         "sample": "the whole 1M-row query, best of 5, one thread"},
        "parity": parity(m["result"], want, float_cols=(1,)),
    }


def config3_block(backend, stream, threads: int, rows: int = 200_000_000, distinct: int = 10_000_000) -> dict:
    """Config 3: 200M rows as uneven batches, 10M keys, SUM/MIN/MAX/COUNT of a
    nullable Int32 under WHERE f < s."""
    import oracle
    import pyarrow as pa

    from oxidelake_b200 import bench_batches
    from oxidelake_b200.benchkit import config3_device, host_copy, pinned_batch

    devs = config3_device(backend, rows, distinct)
    host = [host_copy(d) for d in devs]
    whole = pa.Table.from_batches(host).combine_chunks().to_batches()[0]
    peak, kind = peaks("hbm")
    out = {"workload": f"{rows} rows in {len(devs)} uneven batches (8K-1M rows), g i64 uniform over {distinct} "
                       "values, x i32 U[-1e6,1e6] with 2% NULLs, f i32 U[0,100); SELECT g, SUM(x), MIN(x), MAX(x), "
                       "COUNT(x) WHERE f < s GROUP BY g; one persistent launch",
           "l2": "inputs (3.2 GB) larger than L2; no flush",
           "selectivity": {}}
    aggs = [(0, 1), (2, 1), (3, 1), (1, 1)]
    for sel in (1, 50, 99):
        m = bench_batches.measure(backend, stream, devs, sel, repeats=2, download=True)
        t0 = time.perf_counter()
        want = oracle.aggregate(whole, 0, aggs, [(2, 1, 3, sel)], threads=threads)
        dt = time.perf_counter() - t0
        achieved = m["kernel_bytes"] / (m["kernel_ms"] / 1e3) / 1e9
        out["selectivity"][f"{sel}%"] = {
            "roofline": {"bound": "hbm", "kernel": m["kernel"], "kernel_ms": round(m["kernel_ms"], 3),
                         "algorithmic_bytes_per_launch": round(m["kernel_bytes"]), "achieved": round(achieved, 1),
                         "peak": peak, "peak_kind": kind, "unit": "GB/s", "frac": round(achieved / peak, 4)},
            "call_ms": round(m["call_ms"], 3),
            "groups": m["groups"],
            "cpu_baseline": {"value": round(m["kernel_bytes"] / dt / 1e9, 3), "unit": "GB/s", "cores": threads,
                             "kind": "port", "sample": f"the whole {rows}-row input, groups split over threads by key"},
            "parity": parity(m["result"], want),
        }
        del m
    del whole
    pinned, keep = [], []
    for h in host:
        pb, k = pinned_batch(backend, h)
        pinned.append(pb)
        keep.append(k)
    del host
    e = bench_batches.measure_e2e(backend, stream, pinned, 99, repeats=1)
    gb = bench_batches.kernel_bytes(rows, 99)
    out["e2e_99%"] = {"value": round(gb / (e["e2e_ms"] / 1e3) / 1e9, 2), "unit": "GB/s", "ms": round(e["e2e_ms"], 1),
                      "h2d_bytes_per_step": e["h2d_bytes"], "d2h_bytes_per_step": e["d2h_bytes"],
                      "from": "page-locked host batches, one upload call per batch"}
    del pinned, keep, devs
    return out


def _order_key(dist: np.ndarray) -> np.ndarray:
    """FP32 distances as signed integers in IEEE totalOrder (the oracle's
    ORDER BY distance)."""
    k = dist.view(np.int32).astype(np.int64)
    return np.where(k < 0, k ^ 0x7FFFFFFF, k)


def oracle_topk_kept(x, f, lit: int, queries: np.ndarray, k: int, metric: int, threads: int, chunk: int = 500_000):
    """The oracle's top-k over the rows with f < lit, read from the device
    table in chunks of kept rows; chunk results merge by (distance in
    totalOrder, row id), as one pass over the table orders them.  Returns
    (ids, dist, seconds of oracle compute)."""
    import oracle
    import pyarrow as pa
    import torch

    kept = torch.nonzero(f < lit).squeeze(1)
    nq, dim = queries.shape
    best_ids = np.full((nq, 0), -1, np.int64)
    best_d = np.zeros((nq, 0), np.float32)
    compute = 0.0
    for start in range(0, kept.numel(), chunk):
        idx = kept[start:start + chunk]
        xs = x.index_select(0, idx).cpu().numpy()
        rows = idx.cpu().numpy()
        batch = pa.RecordBatch.from_arrays(
            [pa.FixedSizeListArray.from_arrays(pa.array(xs.reshape(-1)), dim)], names=["emb"])
        t0 = time.perf_counter()
        ids, dist = oracle.vector_topk(batch, 0, queries, k, metric, None, threads=threads)
        compute += time.perf_counter() - t0
        gids = np.where(ids >= 0, rows[np.clip(ids, 0, None)], -1)
        cat_i = np.concatenate([best_ids, gids], axis=1)
        cat_d = np.concatenate([best_d, dist], axis=1)
        order = np.lexsort((cat_i, _order_key(cat_d)), axis=1)[:, :k]
        best_ids = np.take_along_axis(cat_i, order, axis=1)
        best_d = np.take_along_axis(cat_d, order, axis=1)
    return best_ids, best_d, compute, int(kept.numel())


def config4_block(backend, stream, threads: int, rows: int = 10_000_000, dim: int = 768, nq: int = 256,
                  check_every: int = 16) -> dict:
    """Config 4: top-10 of 256 queries over 10M x 768 FP32 rows, WHERE f < 30."""
    import torch

    from oxidelake_b200 import bench_topk
    from oxidelake_b200.benchkit import unit_queries, vector_table
    from oxidelake_b200.params import Comparison as Cmp
    from oxidelake_b200.params import DistanceMetric, Literal, compare

    batch, x, f = vector_table(backend, rows, dim, bench_topk.SEED, 100)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ix = backend.vector_index(stream, batch, 1)
    build_s = time.perf_counter() - t0
    q = unit_queries(nq, dim, 5)
    pred = compare(0, Cmp.Lt, Literal.int64(30))
    peak, kind = peaks("bf16")
    sub = np.arange(0, nq, check_every)
    out = {"workload": f"{rows} rows x {dim} f32 (L2-normalised), f i64 U[0,100); {nq} queries, top-10, "
                       "WHERE f < 30; BF16 tcgen05 scan, FP32 accumulate, FP32 re-rank",
           "index_build_s": round(build_s, 3), "metric": {}}
    for metric in (DistanceMetric.L2, DistanceMetric.Cosine):
        m = bench_topk.measure(backend, stream, ix, batch, q, 10, metric, pred, repeats=3)
        want_ids, want_d, cpu_s, kept = oracle_topk_kept(x, f, 30, q[sub], 10, int(metric), threads)
        flops = 2.0 * nq * kept * dim
        achieved = flops / (m["scan_ms"] / 1e3) / 1e12
        got_ids, got_d = m["ids"][sub], m["dist"][sub]
        same = bool((got_ids == want_ids).all() and (got_d.view(np.uint32) == want_d.view(np.uint32)).all())
        st = m["stats"]
        out["metric"][metric.name.lower()] = {
            "roofline": {"bound": "tensor", "kernel": "compaction + topk_scan_kernel", "kernel_ms": round(m["scan_ms"], 3),
                         "algorithmic_flops_per_launch": flops, "achieved": round(achieved, 1), "peak": peak,
                         "peak_kind": kind + " (bf16 dense, burst)", "unit": "TFLOP/s", "frac": round(achieved / peak, 4)},
            "kept_rows": kept,
            "call_ms": round(m["call_ms"], 3),
            "e2e": {"value": round(flops / (m["call_ms"] / 1e3) / 1e12, 1), "unit": "TFLOP/s",
                    "ms": round(m["call_ms"], 3), "h2d_bytes_per_step": m["h2d_bytes"],
                    "d2h_bytes_per_step": m["d2h_bytes"],
                    "from": "queries in host memory, ids and distances back to host memory; the table resident"},
            "exact_queries": st["exact_queries"], "reranked": st["reranked"],
            "bf16_score_error_vs_fp64": {"max": st["max_score_error"], "mean": st["mean_score_error"]},
            "cpu_baseline": {"value": round(2.0 * len(sub) * kept * dim / cpu_s / 1e12, 4), "unit": "TFLOP/s",
                             "cores": min(threads, len(sub)), "kind": "port",
                             "sample": f"{len(sub)} of {nq} queries over every kept row (one thread per query)"},
            "parity": {"result": "ok" if same else "mismatch",
                       "checked": f"queries {sub[0]}, {sub[1]}, ... {sub[-1]} ({len(sub)} of {nq}): ids and distance bits"},
        }
    del ix, batch, x, f
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return out


def ops_block(backend, stream, build, probe, bdev, pdev) -> dict:
    """The plain drop-in operators (filter_project, probe_join, hash_join,
    vector_distance) at HBM-bound sizes, each against the measured HBM
    copy bandwidth and checked against the oracle."""
    from oxidelake_b200 import bench_ops

    peak, kind = peaks("hbm")
    out = {}
    for line in bench_ops.measure_filter_join(backend, stream, build, probe, bdev, pdev, peak, repeats=5):
        out[line.pop("op")] = dict(line, peak_kind=kind)
    line = bench_ops.measure_distance(backend, stream, peak, repeats=5)
    out[line.pop("op")] = dict(line, peak_kind=kind)
    return out


def config5_block(backend, stream, build, probe, seconds: float = 2.0) -> dict:
    """Config 5: the served mixed stream against the plain path."""
    from oxidelake_b200 import bench_serve

    ctx = bench_serve.Stream(backend, stream, 10_000_000, 768, probe.num_rows, build, probe)
    m = bench_serve.measure(ctx, seconds)
    del ctx
    return {"workload": "HBM-resident 10M x 768 vector table (f U[0,1e6)) and the 1M-build / 100M-probe join "
                        "tables; Poisson arrivals, 70% top-k (k in {5,10,100}, selectivity log-uniform 0.1%-100%), "
                        "30% join+aggregate over probe slices of 1K-1M rows; budget 150 GB",
            **m["summary"], "runs": m["runs"]}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--probe-rows", type=int, default=PROBE_ROWS)
    ap.add_argument("--build-rows", type=int, default=BUILD_ROWS)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--configs", default="1,3,4,5,ops",
                    help="other configurations measured on one GPU ('' for none; 'ops': the plain operators)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--agg-variant", type=int, default=-1,
                    help="pin the join-aggregate kernel variant as oxb_set_agg_variant does (-1: tuned)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return 0

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    from oxidelake_b200.backend import CudaBackend
    from oxidelake_b200.benchkit import pinned_batch
    from oxidelake_b200.params import AggregateFunction as F
    from oxidelake_b200.params import Comparison as Cmp
    from oxidelake_b200.params import Literal, compare

    build, probe = gen_data(rank, args.build_rows, args.probe_rows)
    backend = CudaBackend(local)
    if args.agg_variant >= 0:
        backend.set_agg_variant(args.agg_variant, 0)
    stream = backend.create_stream()
    tstream = torch.cuda.ExternalStream(stream.cuda_handle())
    bdev = backend.upload(stream, build)
    pdev = backend.upload(stream, probe)
    pred = compare(2, Cmp.Gt, Literal.int32(10))
    aggs = [(F.Sum, 0, 1), (F.Sum, 0, 2), (F.CountStar, 0, 0), (F.Avg, 0, 1)]

    def barrier():
        if dist is not None:
            dist.barrier()

    # On more than one GPU each rank folds its shard into partial groups (AVG
    # as SUM and COUNT); one exchange merges them into the query's result.
    from oxidelake_b200.distributed import exchange_and_merge, partial_aggregates

    partial, finish = partial_aggregates(aggs)
    names = ["attr", "SUM(payload)", "SUM(qty)", "COUNT(*)", "AVG(payload)"]

    def exchange(res):
        if dist is None:
            return res
        return exchange_and_merge(res, partial, finish, names)

    def step():
        table = backend.prepare_join_build(stream, bdev, 0)
        out = backend.join_aggregate(stream, pdev, 0, table, pred, (1, 1), partial if dist is not None else aggs)
        return exchange(backend.download(stream, out))

    # warm-up
    for _ in range(args.warmup):
        res = step()
    torch.cuda.synchronize()

    # The kernel's own time (CUDA events around it on its stream) in steps of
    # their own: the library's kernel timing records events and reads them
    # back each call, which is instrumentation, not the step's work, so the
    # timed steps below run with it off.
    kernel_ms = []
    kernel_name = None
    backend.set_kernel_timing(True)
    for _ in range(args.steps):
        res = step()
        kernel_name, kms_step = backend.last_kernel_time()
        kernel_ms.append(kms_step)
    backend.set_kernel_timing(False)
    torch.cuda.synchronize()

    launches0 = backend.kernel_launches()
    with ClockSampler(local) as clocks:
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(tstream)
        for _ in range(args.steps):
            res = step()
        e1.record(tstream)
        torch.cuda.synchronize()
        barrier()
    launches = backend.kernel_launches() - launches0
    ms = e0.elapsed_time(e1) / args.steps
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    step_bytes = algorithmic_bytes(args.build_rows, args.probe_rows)
    value = world * step_bytes / (ms / 1e3) / 1e9

    # End to end through the public API with host buffers: pinned H2D of the
    # step's inputs, the query, the result read back.
    pin_build, keep_b = pinned_batch(backend, build)
    pin_probe, keep_p = pinned_batch(backend, probe)
    h2d = sum(pin_build.column(i).nbytes for i in range(pin_build.num_columns)) + sum(
        pin_probe.column(i).nbytes for i in range(pin_probe.num_columns)
    )
    d2h = sum(res.column(i).nbytes for i in range(res.num_columns))

    def e2e_step():
        bd = backend.upload(stream, pin_build)
        pd = backend.upload(stream, pin_probe)
        table = backend.prepare_join_build(stream, bd, 0)
        out = backend.download(stream, backend.join_aggregate(stream, pd, 0, table, pred, (1, 1),
                                                              partial if dist is not None else aggs))
        return exchange(out)

    e2e_step()
    barrier()
    torch.cuda.synchronize()
    e0.record(tstream)
    for _ in range(args.e2e_steps):
        e2e_step()
    e1.record(tstream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.e2e_steps
    if dist is not None:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * step_bytes / (e2e_ms / 1e3) / 1e9
    del keep_b, keep_p, pin_build, pin_probe

    rc = 0
    if rank == 0:
        peak, peak_kind = peaks()
        kms = float(np.mean(kernel_ms)) if kernel_ms else None
        kernel_bytes = args.probe_rows * PROBE_ROW_BYTES + args.build_rows * BUILD_ROW_BYTES
        achieved = kernel_bytes / (kms / 1e3) / 1e9 if kms else None
        config = dict(CONFIG2_CONFIG, build_rows=args.build_rows, probe_rows_per_gpu=args.probe_rows,
                      groups=res.num_rows, parallelism=f"dp{world}" if world > 1 else "single")
        line = {
            "metric": "GB/s",
            "value": round(value, 2),
            "unit": "GB/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms, 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "int64/f64",
            "data": "synthetic",
            "config": config,
            "rows_per_s": round(world * args.probe_rows / (ms / 1e3)),
            "roofline": {
                "bound": "hbm",
                "kernel": kernel_name,
                "timed": "the query's probe-table pre-pass and fused probe/filter/aggregate kernel, CUDA events on its stream, in as many steps of their own as the timed ones (which run without the events)",
                "achieved": round(achieved, 1) if achieved else None,
                "peak": peak,
                "peak_kind": peak_kind,
                "unit": "GB/s",
                "frac": round(achieved / peak, 4) if achieved else None,
                "kernel_ms": round(kms, 4) if kms else None,
                "traffic": profiled_traffic(profile_kernel(kernel_name or "")),
                "traffic_source": f"profiles/{profile_kernel(kernel_name or '')}_config2.md",
                "algorithmic_bytes_per_launch": kernel_bytes,
            },
            "e2e": {
                "value": round(e2e_value, 2),
                "unit": "GB/s",
                "ms_per_step": round(e2e_ms, 3),
                "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h),
            },
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
        }
        checks = []
        if world == 1 and not args.no_cpu_baseline:
            import oracle

            threads = oracle.cpu_threads()
            want, dt = oracle_join_aggregate(build, probe, threads)
            line["cpu_baseline"] = {
                "value": round(step_bytes / dt / 1e9, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                "sample": f"the whole workload: probe {probe.num_rows} rows x build {build.num_rows} rows, {dt:.1f} s",
            }
            p = parity(res, want, float_cols=(1, 4))
            p["checked"] = "the last timed step's 1000 groups against the oracle over all probe rows"
            line["parity_detail"] = p
            checks.append(p["result"])
            configs = [c.strip() for c in args.configs.split(",") if c.strip()]
            per = {}
            backend.set_kernel_timing(True)  # the blocks read each call's kernel time
            blocks = {
                "1": lambda: config1_block(backend, stream, threads),
                "3": lambda: config3_block(backend, stream, threads),
                "4": lambda: config4_block(backend, stream, threads),
                "5": lambda: config5_block(backend, stream, build, probe),
                "ops": lambda: ops_block(backend, stream, build, probe, bdev, pdev),
            }
            for c in configs:
                if c not in blocks:
                    continue
                t0 = time.perf_counter()
                try:
                    blk = blocks[c]()
                except Exception as e:  # recorded in the line; the headline still prints
                    blk = {"error": repr(e)[:300]}
                blk["seconds"] = round(time.perf_counter() - t0, 1)
                per[f"config{c}" if c != "ops" else "plain_operators"] = blk
                if c == "1" and "parity" in blk:
                    checks.append(blk["parity"]["result"])
                if c == "ops":
                    checks += [v["parity"]["result"] for v in blk.values() if isinstance(v, dict) and "parity" in v]
                for sub in ("selectivity", "metric"):
                    checks += [v["parity"]["result"] for v in blk.get(sub, {}).values()]
            if per:
                line["per_config"] = per
        line["parity"] = ("ok" if all(c == "ok" for c in checks) else "mismatch") if checks else "not checked (N > 1)"
        print(json.dumps(line), flush=True)
        rc = 0 if line["parity"] != "mismatch" else 1
    if dist is not None:
        dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
