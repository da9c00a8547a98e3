"""Telemetry through the C ABI: after a filter and a join on the B200, the
counters oxb_last_call_stats and oxb_operator_stats_get report are the
ones OperatorStats records (core/src/telemetry.rs:99-190): rows in and out,
bytes moved each way, batches, elapsed time, and no CPU fallback."""
import numpy as np
import pyarrow as pa
import pytest

from oxidelake_b200 import _abi
from oxidelake_b200.errors import Unsupported
from oxidelake_b200.params import Comparison as Cmp
from oxidelake_b200.params import Literal, compare

pytestmark = pytest.mark.gpu


def test_filter_and_join_counters(backend, stream):
    for op in range(5):
        backend.operator_stats(op, reset=True)
    rng = np.random.default_rng(1)
    n = 200_000
    k = rng.integers(0, 1000, n)
    v = rng.standard_normal(n)
    batch = pa.RecordBatch.from_arrays([pa.array(k), pa.array(v, mask=rng.random(n) < 0.1)], names=["k", "v"])
    dev = backend.upload(stream, batch)
    up = backend.last_call_stats()
    assert up["op"] == _abi.OP_TRANSFER and up["status"] == 0
    assert up["bytes_h2d"] == n * 8 + n * 8 + (n + 7) // 8 and up["rows_in"] == n

    out = backend.filter_project(stream, dev, compare(0, Cmp.Lt, Literal.int64(300)), [1])
    st = backend.last_call_stats()
    kept = int((k < 300).sum())
    assert st["op"] == _abi.OP_FILTER and st["status"] == 0
    assert (st["rows_in"], st["rows_out"], st["batches"]) == (n, kept, 1)
    assert st["bytes_h2d"] == st["bytes_d2h"] == 0  # device-resident in and out
    assert st["elapsed_ns"] > 0
    host = backend.download(stream, out)
    dn = backend.last_call_stats()
    assert dn["op"] == _abi.OP_TRANSFER and dn["bytes_d2h"] == kept * 8 + (kept + 7) // 8
    assert host.num_rows == kept

    build = pa.RecordBatch.from_arrays([pa.array(np.arange(0, 2000, 2, dtype=np.int64))], names=["key"])
    bdev = backend.upload(stream, build)
    table = backend.prepare_join_build(stream, bdev, 0)
    assert backend.last_call_stats()["rows_in"] == 1000
    matches = backend.probe_join(stream, dev, 0, table)
    pj = backend.last_call_stats()
    assert pj["op"] == _abi.OP_JOIN and pj["rows_in"] == n and pj["rows_out"] == int((k % 2 == 0).sum())
    joined = backend.hash_join(stream, dev, bdev, table, matches, 0, len(matches))
    hj = backend.last_call_stats()
    assert hj["op"] == _abi.OP_JOIN and hj["rows_out"] == joined.num_rows() == len(matches)

    filt = backend.operator_stats(_abi.OP_FILTER)
    assert (filt["calls"], filt["batches"], filt["rows_in"], filt["rows_out"]) == (1, 1, n, kept)
    assert filt["fallback_batches"] == 0 and filt["unsupported"] == 0 and filt["failed"] == 0
    join = backend.operator_stats(_abi.OP_JOIN)
    assert join["calls"] == 3 and join["rows_out"] == 2 * len(matches)
    xfer = backend.operator_stats(_abi.OP_TRANSFER, reset=True)
    assert xfer["bytes_h2d"] == up["bytes_h2d"] + 1000 * 8 and xfer["bytes_d2h"] == dn["bytes_d2h"]
    assert backend.operator_stats(_abi.OP_TRANSFER)["calls"] == 0  # reset


def test_unsupported_is_counted_not_run_on_the_cpu(backend, stream):
    backend.operator_stats(_abi.OP_FILTER, reset=True)
    batch = pa.RecordBatch.from_arrays([pa.array(["a", "b"])], names=["s"])
    with pytest.raises(Unsupported):
        backend.upload(stream, batch)
    n = 1000
    dev = backend.upload(stream, pa.RecordBatch.from_arrays([pa.array(np.arange(n, dtype=np.int64))], names=["k"]))
    with pytest.raises(Exception):
        backend.filter_project(stream, dev, compare(5, Cmp.Lt, Literal.int64(3)), [0])  # no column 5
    st = backend.operator_stats(_abi.OP_FILTER)
    assert st["calls"] == 1 and st["failed"] + st["unsupported"] == 1 and st["fallback_batches"] == 0
