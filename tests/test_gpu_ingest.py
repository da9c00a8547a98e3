"""Upload of pageable host columns through the page-locked staging ring
(oxb_set_upload_staging) against the driver's own pageable copy: the device
holds the same bytes either way, for ragged chunk counts, every column type,
validity bitmaps, and any number of staging threads.  Downloads into
pageable memory run the ring the other way and are checked the same way."""
import ctypes as C
import os

import numpy as np
import pyarrow as pa
import pytest

from oxidelake_b200 import _abi
from oxidelake_b200.backend import DeviceBatch
from oxidelake_b200.errors import Plan

pytestmark = pytest.mark.gpu

# 8 MiB slots: 2_100_003 rows give 3 chunks of Int64 (the last one ragged),
# 2 of Int32 and 9 of an 8-wide vector; the validity bitmaps stay below the
# 4 MiB threshold and take the single copy.
ROWS = 2_100_003
DEFAULT_THREADS = max(1, min(8, (os.cpu_count() or 2) // 2))


def make_batch(rows: int, seed: int) -> pa.RecordBatch:
    rng = np.random.default_rng(seed)
    i64 = rng.integers(-(2**62), 2**62, size=rows, dtype=np.int64)
    f64 = rng.standard_normal(rows)
    null = rng.random(rows) < 0.1
    i32 = rng.integers(-(2**31), 2**31 - 1, size=rows, dtype=np.int32)
    vec = rng.standard_normal(rows * 8).astype(np.float32)
    emb = pa.FixedSizeListArray.from_arrays(pa.array(vec), 8)
    return pa.record_batch(
        [pa.array(i64), pa.array(f64, mask=null), pa.array(i32), emb], names=["a", "b", "c", "emb"]
    )


@pytest.mark.parametrize("threads", [0, 1, 4, 7, 8])
def test_staged_upload_is_byte_exact(backend, stream, threads):
    batch = make_batch(ROWS, 11 + threads)
    backend.set_upload_staging(threads)
    try:
        dev = backend.upload(stream, batch)
        out = backend.download(stream, dev)
    finally:
        backend.set_upload_staging(DEFAULT_THREADS)
    assert out.num_rows == ROWS
    for i in range(batch.num_columns):
        assert out.column(i).equals(batch.column(i)), batch.schema.field(i).name


@pytest.mark.parametrize("rows", [1, 524_287, 524_288, 1_048_577])
def test_sizes_around_the_threshold_and_one_chunk(backend, stream, rows):
    # Int64: 4 MiB is exactly 524_288 rows, 8 MiB (one slot) 1_048_576 rows.
    data = np.arange(rows, dtype=np.int64) * 7919 - 3
    batch = pa.record_batch([pa.array(data)], names=["a"])
    out = backend.download(stream, backend.upload(stream, batch))
    assert out.column(0).equals(batch.column(0))


def test_staged_source_may_change_once_upload_returns(backend, stream):
    # A staged buffer is fully in page-locked slots or on the device when
    # oxb_upload returns, so the caller may overwrite it before the stream
    # is synchronized.
    rows = 3_000_001
    src = np.arange(rows, dtype=np.int64) * 3 + 1
    keep = src.copy()
    schema = pa.schema([("a", pa.int64())])
    desc = (_abi.Column * 1)(_abi.Column(_abi.TYPE_INT64, 1, rows, src.ctypes.data, None))
    h = C.c_void_p()
    _abi.check(_abi.lib().oxb_upload(backend.handle, stream.handle, desc, 1, rows, C.byref(h)))
    src[:] = -1
    backend.synchronize(stream)
    out = backend.download(stream, DeviceBatch(h.value, schema))
    assert np.array_equal(out.column(0).to_numpy(), keep)


@pytest.mark.parametrize("threads", [0, 1, 8])
def test_staged_download_of_a_device_result(backend, stream, threads):
    # A filter's output is produced on the device and downloaded into
    # pageable memory: through the ring (threads > 0) or the driver's copy.
    from oxidelake_b200.params import Comparison as Cmp
    from oxidelake_b200.params import Literal, compare

    rows = 9_000_001
    rng = np.random.default_rng(5)
    a = rng.integers(0, 100, size=rows, dtype=np.int64)
    v = rng.standard_normal(rows)
    batch = pa.record_batch([pa.array(a), pa.array(v, mask=rng.random(rows) < 0.05)], names=["a", "v"])
    keep = a < 90
    want = batch.filter(pa.array(keep))
    dev = backend.upload(stream, batch)
    backend.set_upload_staging(threads)
    try:
        out = backend.download(stream, backend.filter_project(stream, dev, compare(0, Cmp.Lt, Literal.int64(90)), [0, 1]))
    finally:
        backend.set_upload_staging(DEFAULT_THREADS)
    assert out.num_rows == want.num_rows
    for i in range(2):
        assert out.column(i).equals(want.column(i))


def test_staging_threads_out_of_range(backend):
    with pytest.raises(Plan):
        backend.set_upload_staging(-1)
    with pytest.raises(Plan):
        backend.set_upload_staging(33)
    backend.set_upload_staging(DEFAULT_THREADS)


def test_concurrent_staged_uploads_and_downloads_on_two_streams(backend):
    """Two host threads stage pageable columns of at least 40 MiB on their
    own streams at the same time, each downloading into pageable memory
    right after its upload, while one of them swaps the staging pool
    between its rounds: every device buffer and every downloaded column is
    byte-exact."""
    import threading

    rows = 5_500_007  # 42 MiB of Int64, 44 MiB of Float64: six slots each
    errors = []

    def worker(seed, swap):
        try:
            s = backend.create_stream()
            for round_ in range(3):
                rng = np.random.default_rng(seed * 10 + round_)
                a = rng.integers(-(2**62), 2**62, size=rows, dtype=np.int64)
                v = rng.standard_normal(rows)
                batch = pa.record_batch([pa.array(a), pa.array(v)], names=["a", "v"])
                dev = backend.upload(s, batch)
                out = backend.download(s, dev)
                if not (out.column(0).equals(batch.column(0)) and out.column(1).equals(batch.column(1))):
                    errors.append(f"thread {seed} round {round_}: bytes differ")
                if swap:
                    backend.set_upload_staging(3 if round_ % 2 == 0 else DEFAULT_THREADS)
        except Exception as e:  # reported below
            errors.append(f"thread {seed}: {e!r}")

    threads = [threading.Thread(target=worker, args=(1, True)), threading.Thread(target=worker, args=(2, False))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    backend.set_upload_staging(DEFAULT_THREADS)
    assert not errors, errors
