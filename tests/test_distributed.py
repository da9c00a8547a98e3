"""The exchange step of the operator path on more than one GPU, run as two
gloo ranks on the CPU: each rank folds its own probe shard into partial
groups (the oracle stands in for its GPU here), the partials are gathered
and merged, and the merged result equals the oracle over every probe row."""
import os
import socket

import numpy as np
import pyarrow as pa
import pytest
import torch.multiprocessing as mp

AGGS = [(5, 0, 0), (0, 0, 1), (4, 0, 1), (0, 0, 2), (2, 0, 2), (3, 0, 1), (1, 0, 1)]  # COUNT(*), SUM, AVG, SUM, MIN, MAX, COUNT
NAMES = ["attr", "COUNT(*)", "SUM(payload)", "AVG(payload)", "SUM(qty)", "MIN(qty)", "MAX(payload)", "COUNT(payload)"]


def _data():
    from datagen import config2

    build, probe = config2(3_000, 120_000, seed=11)
    rng = np.random.default_rng(12)
    # NULL payloads and NULL group keys on the build side
    pay = probe.column(1).to_numpy(zero_copy_only=False)
    probe = pa.RecordBatch.from_arrays(
        [probe.column(0), pa.array(pay, mask=rng.random(len(pay)) < 0.05), probe.column(2)], names=probe.schema.names
    )
    attr = build.column(1).to_numpy(zero_copy_only=False)
    build = pa.RecordBatch.from_arrays([build.column(0), pa.array(attr, mask=rng.random(len(attr)) < 0.02)],
                                       names=build.schema.names)
    return build, probe


def _rank(rank, world, port, shares, out):
    import sys

    sys.path[:0] = [os.path.dirname(os.path.abspath(__file__)), os.path.dirname(os.path.dirname(os.path.abspath(__file__)))]
    import torch.distributed as dist

    import oracle
    from oxidelake_b200.distributed import exchange_and_merge, partial_aggregates

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        build, probe = _data()
        lo, hi = shares[rank]
        shard = probe.slice(lo, hi - lo)
        leaves = [(2, 3, 3, 10)]  # qty > 10
        partial, finish = partial_aggregates(AGGS)
        local = oracle.join_aggregate(shard, build, 0, 0, leaves, (1, 1), [tuple(int(x) for x in a) for a in partial])
        merged = exchange_and_merge(local, partial, finish, NAMES)
        if rank == 0:
            sink = pa.BufferOutputStream()
            with pa.ipc.new_stream(sink, merged.schema) as w:
                w.write_batch(merged)
            out.put(sink.getvalue().to_pybytes())
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("shares", [[(0, 70_000), (70_000, 120_000)], [(0, 0), (0, 120_000)]], ids=["split", "empty-rank"])
def test_two_gloo_ranks_merge_to_the_whole(shares):
    import oracle
    from compare import assert_batches_equal

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, shares, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = pa.ipc.open_stream(out.get(timeout=120)).read_next_batch()
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    build, probe = _data()
    want = oracle.join_aggregate(probe, build, 0, 0, [(2, 3, 3, 10)], (1, 1), AGGS)
    assert_batches_equal(got, want, float_sum_cols=(2, 3))
