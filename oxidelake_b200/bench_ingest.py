"""Ingest rate of oxb_upload: the hash join's probe columns (100M rows of
fk i64, payload f64, qty i32 = 2.0 GB) copied from host memory into HBM.

Prints one JSON line per case, each the best of --repeats uploads (wall
clock around oxb_upload and the stream synchronize):
- "pageable, driver copy": staging off, one cudaMemcpyAsync per column from
  pageable memory, staged by the driver itself;
- "pageable, staged T threads": the page-locked ring filled by T host threads;
- "page-locked source": the same columns in page-locked memory, one copy per
  column (the copy engine's own rate, the ceiling of the two above);
- the same three cases the other way, from HBM into host memory
  (oxb_download_column, which returns once the bytes are on the host).

    python -m oxidelake_b200.bench_ingest [--rows N] [--repeats R]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=100_000_000)
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--threads", default="0,1,2,4,8")
    args = ap.parse_args()

    import numpy as np
    import torch

    from oxidelake_b200 import _abi
    from oxidelake_b200.backend import CudaBackend

    n = args.rows
    rng = np.random.default_rng(0x0A11CE + 2)
    fk = rng.integers(0, 1_000_000, size=n, dtype=np.int64)
    payload = rng.random(n) * 100.0
    qty = rng.integers(1, 51, size=n, dtype=np.int32)
    host_bytes = fk.nbytes + payload.nbytes + qty.nbytes

    b = CudaBackend(0)
    s = b.create_stream()
    lib = _abi.lib()

    def upload(cols) -> float:
        desc = (_abi.Column * len(cols))(*[_abi.Column(t, 1, n, a.ctypes.data, None) for t, a in cols])
        h = C.c_void_p()
        t0 = time.perf_counter()
        _abi.check(lib.oxb_upload(b.handle, s.handle, desc, len(cols), n, C.byref(h)))
        b.synchronize(s)
        dt = time.perf_counter() - t0
        lib.oxb_batch_free(h)
        return dt

    def best(cols) -> float:
        upload(cols)  # warm-up: pool growth, ring allocation
        return min(upload(cols) for _ in range(args.repeats))

    pageable = [(_abi.TYPE_INT64, fk), (_abi.TYPE_FLOAT64, payload), (_abi.TYPE_INT32, qty)]
    cases = []
    for t in [int(x) for x in args.threads.split(",")]:
        b.set_upload_staging(t)
        cases.append(("pageable, driver copy" if t == 0 else f"pageable, staged {t} threads", t, best(pageable)))
    b.set_upload_staging(max(1, min(8, (os.cpu_count() or 2) // 2)))  # the default

    pinned = []
    for t, a in pageable:
        p = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True).numpy().view(a.dtype)
        p[:] = a
        pinned.append((t, p))
    cases.append(("page-locked source", 0, best(pinned)))

    # The way back: the same columns from HBM into host memory.
    desc = (_abi.Column * 3)(*[_abi.Column(t, 1, n, a.ctypes.data, None) for t, a in pageable])
    h = C.c_void_p()
    _abi.check(lib.oxb_upload(b.handle, s.handle, desc, 3, n, C.byref(h)))
    b.synchronize(s)
    has = C.c_int32(0)

    def download(outs) -> float:
        t0 = time.perf_counter()
        for i, o in enumerate(outs):
            _abi.check(lib.oxb_download_column(b.handle, s.handle, h, i, o.ctypes.data, None, C.byref(has)))
        return time.perf_counter() - t0

    def best_down(outs) -> float:
        download(outs)
        return min(download(outs) for _ in range(args.repeats))

    outs = [np.empty_like(a) for _, a in pageable]
    for o in outs:
        o.fill(0)  # touch every page before timing
    down = []
    for t in (0, max(1, min(8, (os.cpu_count() or 2) // 2))):
        b.set_upload_staging(t)
        down.append(("download to pageable, driver copy" if t == 0 else f"download to pageable, staged {t} threads", t, best_down(outs)))
    down.append(("download to page-locked", 0, best_down([p for _, p in pinned])))
    for o, (_, a) in zip(outs, pageable):
        assert np.array_equal(o, a)
    lib.oxb_batch_free(h)
    cases += down

    for name, t, sec in cases:
        print(json.dumps({
            "workload": "ingest of the hash join's probe columns", "case": name, "staging_threads": t,
            "rows": n, "bytes": host_bytes, "ms": round(sec * 1e3, 2), "gbs": round(host_bytes / sec / 1e9, 2),
            "host_cores": os.cpu_count(), "data": "synthetic",
        }), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
