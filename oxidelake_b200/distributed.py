"""Grouped results of several ranks merged into one: the exchange step of the
operator path on more than one GPU.

Each rank folds its own shard of the input (its probe rows) into partial
group states on its GPU; the partials (a few thousand groups at most for the
join + aggregate workload) are exchanged once and merged on the host.  AVG
cannot be merged from finished averages, so each rank computes it as SUM and
COUNT (partial_aggregates) and the merge finishes it; the merge rules are the
reference's GroupedAggregator::merge (crates/oxidelake-device/src/cpu/
kernels.rs:679-811): counts add, integer sums add wrapping, Float64 sums add,
MIN/MAX take the smaller/larger non-NULL value, a group with no values stays
NULL; groups come out sorted by key with the NULL group last.
"""
from __future__ import annotations

import math
from typing import List, Sequence, Tuple

import numpy as np
import pyarrow as pa

from .params import AggregateFunction as F


def partial_aggregates(aggregates: Sequence[Tuple]) -> Tuple[List[Tuple], List[Tuple]]:
    """The per-rank aggregate list (AVG replaced by SUM and COUNT of its
    column) and, per requested aggregate, how to finish it from the merged
    partial columns: ("col", i) or ("avg", sum_i, count_i)."""
    partial: List[Tuple] = []
    finish: List[Tuple] = []

    def slot(agg):
        if agg not in partial:
            partial.append(agg)
        return partial.index(agg)

    for agg in aggregates:
        f, rest = F(agg[0]), tuple(agg[1:])
        if f == F.Avg:
            finish.append(("avg", slot((F.Sum, *rest)), slot((F.Count, *rest))))
        else:
            finish.append(("col", slot((f, *rest))))
    return partial, finish


def _merge_column(func: F, arrays: List[pa.Array], groups: np.ndarray, ngroups: int) -> pa.Array:
    vals = [a for a in arrays]
    typ = vals[0].type
    valid = np.concatenate([a.is_valid().to_numpy(zero_copy_only=False) for a in vals]) if vals else np.zeros(0, bool)
    if pa.types.is_floating(typ):
        x = np.concatenate([a.fill_null(0.0).to_numpy(zero_copy_only=False) for a in vals]).astype(np.float64)
    else:
        x = np.concatenate([a.fill_null(0).to_numpy(zero_copy_only=False) for a in vals]).astype(np.int64)
    has = np.zeros(ngroups, bool)
    np.logical_or.at(has, groups[valid], True)
    if func in (F.Count, F.CountStar):
        out = np.zeros(ngroups, np.int64)
        np.add.at(out, groups, x)
        return pa.array(out, pa.int64())
    if func == F.Sum:
        if pa.types.is_floating(typ):
            # each group's partial sums added exactly, then rounded once
            parts: List[List[float]] = [[] for _ in range(ngroups)]
            for gi, v, ok in zip(groups, x, valid):
                if ok:
                    parts[gi].append(float(v))
            out = np.array([math.fsum(p) for p in parts], np.float64)
            return pa.array(out, typ, mask=~has)
        out = np.zeros(ngroups, np.uint64)
        np.add.at(out, groups[valid], x[valid].view(np.uint64))  # wraps like wrapping_add
        return pa.array(out.view(np.int64), typ, mask=~has)
    # MIN / MAX over non-NULL values (Float64 by totalOrder through its key)
    if pa.types.is_floating(typ):
        bits = x.view(np.int64)
        key = bits ^ ((bits >> 63) & 0x7FFFFFFFFFFFFFFF)
    else:
        key = x
    fill = np.iinfo(np.int64).max if func == F.Min else np.iinfo(np.int64).min
    best = np.full(ngroups, fill, np.int64)
    (np.minimum if func == F.Min else np.maximum).at(best, groups[valid], key[valid])
    if pa.types.is_floating(typ):
        back = best ^ ((best >> 63) & 0x7FFFFFFFFFFFFFFF)
        out = back.view(np.float64)
    else:
        out = best
    return pa.array(out, typ, mask=~has)


def merge_partials(parts: Sequence[pa.RecordBatch], partial: Sequence[Tuple], finish: Sequence[Tuple],
                   names: Sequence[str]) -> pa.RecordBatch:
    """Merges per-rank partial results (key, then one column per partial
    aggregate) into the final grouped result."""
    parts = [p for p in parts if p is not None]
    keys = [p.column(0) for p in parts]
    key_type = keys[0].type
    kvalid = np.concatenate([k.is_valid().to_numpy(zero_copy_only=False) for k in keys])
    kv = np.concatenate([k.fill_null(0).to_numpy(zero_copy_only=False) for k in keys]).astype(np.int64)
    uniq = np.unique(kv[kvalid])
    has_null = bool((~kvalid).any())
    ngroups = len(uniq) + (1 if has_null else 0)
    groups = np.where(kvalid, np.searchsorted(uniq, kv), len(uniq))
    merged = [
        _merge_column(F(partial[j][0]), [p.column(1 + j) for p in parts], groups, ngroups)
        for j in range(len(partial))
    ]
    cols = [pa.array(np.concatenate([uniq, np.zeros(1 if has_null else 0, np.int64)]).astype(key_type.to_pandas_dtype()),
                     key_type, mask=np.arange(ngroups) == len(uniq) if has_null else None)]
    for fin in finish:
        if fin[0] == "col":
            cols.append(merged[fin[1]])
        else:
            s = merged[fin[1]].fill_null(0.0).to_numpy(zero_copy_only=False).astype(np.float64)
            c = merged[fin[2]].to_numpy(zero_copy_only=False).astype(np.int64)
            with np.errstate(divide="ignore", invalid="ignore"):
                avg = s / c
            cols.append(pa.array(avg, pa.float64(), mask=c == 0))
    return pa.RecordBatch.from_arrays(cols, names=list(names))


def exchange_and_merge(local: pa.RecordBatch, partial, finish, names, group=None) -> pa.RecordBatch:
    """All ranks' partial results gathered (torch.distributed, one
    all_gather of Arrow IPC bytes: NCCL between GPUs, gloo on CPUs) and
    merged; every rank gets the final result."""
    import torch.distributed as dist

    sink = pa.BufferOutputStream()
    with pa.ipc.new_stream(sink, local.schema) as w:
        w.write_batch(local)
    payload = sink.getvalue().to_pybytes()
    gathered: List[bytes] = [b""] * dist.get_world_size(group)
    dist.all_gather_object(gathered, payload, group=group)
    parts = [pa.ipc.open_stream(b).read_next_batch() for b in gathered]
    return merge_partials(parts, partial, finish, names)


# ---- top-k over row shards ------------------------------------------------

def _order_key(dist: np.ndarray) -> np.ndarray:
    """FP32 distances as signed integers in IEEE totalOrder (NaN last), the
    order of ORDER BY distance."""
    k = dist.view(np.int32).astype(np.int64)
    return np.where(k < 0, k ^ 0x7FFFFFFF, k)


def merge_topk(ids: Sequence[np.ndarray], dist: Sequence[np.ndarray], k: int) -> Tuple[np.ndarray, np.ndarray]:
    """Per query, the k best of several ranks' candidate lists ([Q, m_r] ids
    with global row numbers, -1 padding) by (distance in totalOrder, row id):
    the order one pass over the whole table gives.  Each rank's list is its
    shard's exact top-k, and the global top-k is drawn from their union."""
    cat_i = np.concatenate(list(ids), axis=1)
    cat_d = np.concatenate(list(dist), axis=1)
    pad = cat_i < 0
    key = _order_key(cat_d)
    key = np.where(pad, np.iinfo(np.int64).max, key)
    rid = np.where(pad, np.iinfo(np.int64).max, cat_i)
    order = np.lexsort((rid, key), axis=1)[:, :k]
    out_i = np.take_along_axis(cat_i, order, axis=1)
    out_d = np.take_along_axis(cat_d, order, axis=1)
    return out_i, out_d


def exchange_topk(local_ids: np.ndarray, local_dist: np.ndarray, row_offset: int, k: int,
                  group=None) -> Tuple[np.ndarray, np.ndarray]:
    """The top-k of a table sharded by rows over the ranks: each rank's exact
    local top-k (shard row numbers) made global by its shard's first row,
    gathered once, and merged; every rank gets the result."""
    import torch.distributed as dist

    gids = np.where(local_ids >= 0, local_ids + row_offset, -1)
    gathered: List[Tuple[np.ndarray, np.ndarray]] = [None] * dist.get_world_size(group)
    dist.all_gather_object(gathered, (gids, local_dist), group=group)
    return merge_topk([g[0] for g in gathered], [g[1] for g in gathered], k)


# ---- many groups: a hash-partitioned exchange -----------------------------

def key_owner(keys: pa.Array, world: int) -> np.ndarray:
    """The rank that merges each group: a hash of the key (the NULL group to
    rank 0), the same on every rank."""
    valid = keys.is_valid().to_numpy(zero_copy_only=False)
    k = keys.fill_null(0).to_numpy(zero_copy_only=False).astype(np.int64).view(np.uint64)
    with np.errstate(over="ignore"):
        z = k * np.uint64(0x9E3779B97F4A7C15)
        z ^= z >> np.uint64(29)
    return np.where(valid, (z % np.uint64(world)).astype(np.int64), 0)


def exchange_partitioned(local: pa.RecordBatch, partial, finish, names, group=None) -> pa.RecordBatch:
    """The exchange for many groups: each rank sends every partial group to
    the rank its key hashes to (an all-to-all of Arrow IPC pieces), merges
    the groups it owns, and returns them (sorted by key, NULL last).  The
    ranks' results are disjoint; together they are the query's result.  A
    rank holds only its share of the groups, where exchange_and_merge
    gathers all of them everywhere."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    owner = key_owner(local.column(0), world)
    pieces = []
    for r in range(world):
        part = local.filter(pa.array(owner == r))
        sink = pa.BufferOutputStream()
        with pa.ipc.new_stream(sink, local.schema) as w:
            w.write_batch(part)
        pieces.append(sink.getvalue().to_pybytes())
    # all-to-all through one gather of every rank's pieces (gloo and NCCL both carry it)
    gathered: List[List[bytes]] = [None] * world
    dist.all_gather_object(gathered, pieces, group=group)
    me = dist.get_rank(group)
    mine = [pa.ipc.open_stream(g[me]).read_next_batch() for g in gathered]
    return merge_partials(mine, partial, finish, names)
