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


def _vectors():
    rng = np.random.default_rng(21)
    n, d = 6_000, 16
    v = rng.integers(-3, 4, (n, d)).astype(np.float32)
    v[2990:3010] = v[5]  # ties across the shard boundary, broken by row id
    f = rng.integers(0, 100, n)
    q = rng.standard_normal((7, d)).astype(np.float32)
    batch = pa.RecordBatch.from_arrays([pa.array(f), pa.FixedSizeListArray.from_arrays(pa.array(v.reshape(-1)), d)],
                                       names=["f", "emb"])
    return batch, q


def _topk_rank(rank, world, port, metric, out):
    import sys

    sys.path[:0] = [os.path.dirname(os.path.abspath(__file__)), os.path.dirname(os.path.dirname(os.path.abspath(__file__)))]
    import torch.distributed as dist

    import oracle
    from oxidelake_b200.distributed import exchange_topk

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        batch, q = _vectors()
        lo = batch.num_rows * rank // world
        hi = batch.num_rows * (rank + 1) // world
        shard = batch.slice(lo, hi - lo)
        ids, d = oracle.vector_topk(shard, 1, q, 12, metric, [(0, 1, 1, 60)])  # each rank's exact top-k
        gi, gd = exchange_topk(ids, d, lo, 12)
        if rank == 0:
            out.put((gi, gd))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("metric", [0, 1], ids=["l2", "cosine"])
def test_two_gloo_ranks_topk_equals_one_pass(metric):
    """The top-k over a table sharded by rows: each rank's exact top-k,
    gathered and merged by (distance, row id), equals one pass over the
    whole table, ties across the shard boundary included."""
    import oracle

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_topk_rank, args=(r, 2, port, metric, out)) for r in range(2)]
    for p in procs:
        p.start()
    gi, gd = out.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    batch, q = _vectors()
    want_i, want_d = oracle.vector_topk(batch, 1, q, 12, metric, [(0, 1, 1, 60)])
    assert (gi == want_i).all()
    assert (gd.view(np.uint32) == want_d.view(np.uint32)).all()


AGGS3 = [(0, 1), (2, 1), (3, 1), (1, 1), (4, 1)]  # SUM, MIN, MAX, COUNT, AVG of x
NAMES3 = ["g", "SUM(x)", "MIN(x)", "MAX(x)", "COUNT(x)", "AVG(x)"]


def _groups_data():
    from datagen import config3_batches

    batches = config3_batches(90_000, 7_000, seed=23, min_rows=5_000, max_rows=20_000)
    whole = pa.Table.from_batches(batches).combine_chunks().to_batches()[0]
    rng = np.random.default_rng(24)
    g = whole.column(0).to_numpy(zero_copy_only=False)
    return pa.RecordBatch.from_arrays([pa.array(g, mask=rng.random(len(g)) < 0.01), whole.column(1), whole.column(2)],
                                      names=["g", "x", "f"])


def _groups_rank(rank, world, port, out):
    import sys

    sys.path[:0] = [os.path.dirname(os.path.abspath(__file__)), os.path.dirname(os.path.dirname(os.path.abspath(__file__)))]
    import torch.distributed as dist

    import oracle
    from oxidelake_b200.distributed import exchange_partitioned, partial_aggregates

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        whole = _groups_data()
        lo = whole.num_rows * rank // world
        hi = whole.num_rows * (rank + 1) // world
        partial, finish = partial_aggregates([(f, 0, c) for f, c in AGGS3])
        local = oracle.aggregate(whole.slice(lo, hi - lo), 0, [(int(a[0]), a[2]) for a in partial], [(2, 1, 3, 60)])
        mine = exchange_partitioned(local, partial, finish, NAMES3)
        sink = pa.BufferOutputStream()
        with pa.ipc.new_stream(sink, mine.schema) as w:
            w.write_batch(mine)
        out.put((rank, sink.getvalue().to_pybytes()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_hash_partitioned_exchange():
    """Many groups: each rank sends its partial groups to the rank their key
    hashes to and merges those it owns; the ranks' disjoint results together
    equal the oracle over every row (NULL group included)."""
    import oracle
    from compare import assert_batches_equal

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_groups_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    parts = dict(out.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got = [pa.ipc.open_stream(parts[r]).read_next_batch() for r in range(2)]
    assert got[0].num_rows > 0 and got[1].num_rows > 0
    keys = [set(b.column(0).drop_null().to_pylist()) for b in got]
    assert not (keys[0] & keys[1])  # each group merged on one rank
    both = pa.Table.from_batches(got).combine_chunks()
    both = both.sort_by([("g", "ascending")], null_placement="at_end").to_batches()[0]
    want = oracle.aggregate(_groups_data(), 0, AGGS3, [(2, 1, 3, 60)])
    assert_batches_equal(both, pa.RecordBatch.from_arrays(want.columns, names=NAMES3), float_sum_cols=(5,))
