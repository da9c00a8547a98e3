#!/usr/bin/env python
"""Benchmark of the GPU operator path on the hash join + aggregate workload.

Workload (one step): `probe JOIN build ON fk = key WHERE qty > 10 GROUP BY
attr` computing SUM(payload), SUM(qty), COUNT(*), AVG(payload), over a
1M-row build side (unique int64 key, int32 attr U[0,1000)) and a 100M-row
probe side (int64 fk Zipf(1.1) over the build keys with 5% non-matching,
float64 payload U(0,100), int32 qty U[1,50]); seeded synthetic data.  One
step builds the join table on the device and runs the fused probe ->
filter -> aggregate pass, then reads the 1000-group result back.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

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


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


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


def to_pinned(backend, batch):
    """The batch's columns copied into page-locked host memory (kept alive)."""
    import pyarrow as pa

    arrays, keep = [], []
    for i in range(batch.num_columns):
        a = batch.column(i)
        np_vals = np.ascontiguousarray(a.to_numpy(zero_copy_only=False))
        hb = backend.alloc_pinned_host(np_vals.nbytes)
        view = hb.view()
        view[:] = np_vals.view(np.uint8).reshape(-1)
        keep.append(hb)
        buf = pa.foreign_buffer(hb.view().ctypes.data, np_vals.nbytes, base=hb)
        arrays.append(pa.Array.from_buffers(a.type, len(a), [None, buf]))
    return pa.RecordBatch.from_arrays(arrays, schema=batch.schema), keep


def run_reference(args) -> None:
    """The reference's CPU path for the same query: the oracle port of
    cpu/kernels.rs (JoinTable + JoinMatches + GroupedAggregator), run as
    DataFusion would over partitions — one thread per host core, partials
    merged — on a bounded sample of the probe side each step."""
    import oracle
    from oxidelake_b200.params import AggregateFunction as F

    threads = oracle.cpu_threads()
    build, probe = gen_data(0, args.build_rows, min(args.probe_rows, args.ref_sample_rows))
    aggs = [(int(F.Sum), 0, 1), (int(F.Sum), 0, 2), (int(F.CountStar), 0, 0), (int(F.Avg), 0, 1)]
    leaves = [(2, 3, 3, 10)]  # qty > 10
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.join_aggregate(probe, build, 0, 0, leaves, (1, 1), aggs, threads=threads)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    ms = 1e3 * float(np.mean(times))
    gbs = algorithmic_bytes(args.build_rows, probe.num_rows) / (ms / 1e3) / 1e9
    sample = f"probe {probe.num_rows} rows x build {args.build_rows} rows per step"
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
        "config": {"workload": WORKLOAD, "build_rows": args.build_rows, "probe_rows_per_step": probe.num_rows},
        "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(build, probe, target_s: float):
    """The oracle port timed on this host's cores over a bounded probe sample."""
    import oracle
    from oxidelake_b200.params import AggregateFunction as F

    threads = oracle.cpu_threads()
    aggs = [(int(F.Sum), 0, 1), (int(F.Sum), 0, 2), (int(F.CountStar), 0, 0), (int(F.Avg), 0, 1)]
    leaves = [(2, 3, 3, 10)]
    n = min(probe.num_rows, 2_000_000)
    t0 = time.perf_counter()
    oracle.join_aggregate(probe.slice(0, n), build, 0, 0, leaves, (1, 1), aggs, threads=threads)
    dt = time.perf_counter() - t0
    n2 = int(min(probe.num_rows, max(n, n * target_s / max(dt, 1e-3))))
    t0 = time.perf_counter()
    oracle.join_aggregate(probe.slice(0, n2), build, 0, 0, leaves, (1, 1), aggs, threads=threads)
    dt = time.perf_counter() - t0
    gbs = algorithmic_bytes(build.num_rows, n2) / dt / 1e9
    return {
        "value": round(gbs, 3),
        "unit": "GB/s",
        "cores": threads,
        "kind": "port",
        "sample": f"probe {n2} of {probe.num_rows} rows x build {build.num_rows} rows, {dt:.1f} s",
    }


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--probe-rows", type=int, default=PROBE_ROWS)
    ap.add_argument("--build-rows", type=int, default=BUILD_ROWS)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--ref-sample-rows", type=int, default=20_000_000)
    ap.add_argument("--cpu-baseline-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
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

    import pyarrow as pa

    from oxidelake_b200.backend import CudaBackend
    from oxidelake_b200.params import AggregateFunction as F
    from oxidelake_b200.params import Comparison as Cmp
    from oxidelake_b200.params import Literal, compare

    build, probe = gen_data(rank, args.build_rows, args.probe_rows)
    backend = CudaBackend(local)
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
    backend.set_kernel_timing(True)
    for _ in range(args.warmup):
        res = step()
    torch.cuda.synchronize()

    kernel_ms = []
    kernel_name = None
    launches0 = backend.kernel_launches()
    with ClockSampler(local) as clocks:
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(tstream)
        for _ in range(args.steps):
            res = step()
            kernel_name, kms_step = backend.last_kernel_time()
            kernel_ms.append(kms_step)
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
    pin_build, keep_b = to_pinned(backend, build)
    pin_probe, keep_p = to_pinned(backend, probe)
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

    if rank == 0:
        peak, peak_kind = peaks()
        kms = float(np.mean(kernel_ms)) if kernel_ms else None
        kernel_bytes = args.probe_rows * PROBE_ROW_BYTES + args.build_rows * BUILD_ROW_BYTES
        achieved = kernel_bytes / (kms / 1e3) / 1e9 if kms else None
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
            "config": {
                "workload": WORKLOAD,
                "build_rows": args.build_rows,
                "probe_rows_per_gpu": args.probe_rows,
                "groups": res.num_rows,
                "rows_per_s": round(world * args.probe_rows / (ms / 1e3)),
                "l2": "inputs (2.0 GB per GPU) larger than L2; no flush",
                "parallelism": f"dp{world}" if world > 1 else "single",
            },
            "roofline": {
                "bound": "hbm",
                "kernel": kernel_name,
                "timed": "the query's probe-table pre-pass and fused probe/filter/aggregate kernel, CUDA events on its stream",
                "achieved": round(achieved, 1) if achieved else None,
                "peak": peak,
                "peak_kind": peak_kind,
                "unit": "GB/s",
                "frac": round(achieved / peak, 4) if achieved else None,
                "kernel_ms": round(kms, 4) if kms else None,
                "traffic": profiled_traffic("agg_fused_join_kernel"),
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
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(build, probe, args.cpu_baseline_seconds)
        print(json.dumps(line), flush=True)
    del keep_b, keep_p
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
