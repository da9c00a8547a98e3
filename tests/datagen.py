"""Seeded synthetic inputs for the tests and the benchmark.

* ``splitmix64`` and ``demo_table``: the reference's demo generator
  (crates/oxidelake-storage/src/datagen.rs:89-95, 125-182), pinned by its
  digest known-answer test (datagen.rs:348-354).
* ``conformance_*``: the shapes of the reference's conformance suite
  (crates/oxidelake-compute/tests/conformance.rs:34-75, 1405-1430); its Rust
  StdRng streams cannot be reproduced here, so numpy's seeded generator
  draws the same distributions.
* ``config*``: the benchmark configurations, at any scale.
"""
from __future__ import annotations

import math

import numpy as np
import pyarrow as pa

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def splitmix64_stream(state: int, count: int):
    """`count` successive splitmix64 outputs from `state` (datagen.rs:89-95);
    returns (outputs, final state)."""
    with np.errstate(over="ignore"):
        s = (np.uint64(state) + GOLDEN * np.arange(1, count + 1, dtype=np.uint64)).astype(np.uint64)
        z = s.copy()
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    final = (state + 0x9E3779B97F4A7C15 * count) & 0xFFFFFFFFFFFFFFFF
    return z, final


EMBEDDING_DIM = 8
KEY_CARDINALITY = 100
CHUNK_ROWS = 65_536
S_VALUES = [f"s{i}" for i in range(13)]


def _demo_chunk(first_id: int, rows: int, seed: int):
    with np.errstate(over="ignore"):
        state = int((np.uint64(seed) ^ (np.uint64(first_id) * np.uint64(0xA0761D6478BD642F))) & M64)
    per_row = 2 + EMBEDDING_DIM
    r, _ = splitmix64_stream(state, rows * per_row)
    r = r.reshape(rows, per_row)
    rk, rv, re = r[:, 0], r[:, 1], r[:, 2:]
    ids = np.arange(first_id, first_id + rows, dtype=np.int64)
    k = ((rk >> np.uint64(8)).astype(np.int64) % KEY_CARDINALITY).astype(np.int64)
    k_valid = (rk % np.uint64(50)) != 0
    v = (((rv >> np.uint64(8)) & np.uint64(0xFFFFFFFF)) % np.uint64(100)).astype(np.float64) / 4.0
    v_valid = (rv % np.uint64(40)) != 0
    emb = ((re % np.uint64(2000)).astype(np.uint16).astype(np.float32) / np.float32(100.0)) - np.float32(10.0)
    s = [S_VALUES[(first_id + i) % 13] for i in range(rows)]
    return ids, k, k_valid, v, v_valid, s, emb.astype(np.float32)


def demo_table(rows: int, seed: int = 42) -> pa.RecordBatch:
    """The `oxide gen-data` demo table (datagen.rs:125-182) as one batch."""
    parts = [_demo_chunk(f, min(CHUNK_ROWS, rows - f), seed) for f in range(0, rows, CHUNK_ROWS)]
    ids = np.concatenate([p[0] for p in parts]) if parts else np.zeros(0, np.int64)
    k = np.concatenate([p[1] for p in parts]) if parts else np.zeros(0, np.int64)
    kv = np.concatenate([p[2] for p in parts]) if parts else np.zeros(0, bool)
    v = np.concatenate([p[3] for p in parts]) if parts else np.zeros(0)
    vv = np.concatenate([p[4] for p in parts]) if parts else np.zeros(0, bool)
    s = sum((p[5] for p in parts), [])
    emb = np.concatenate([p[6] for p in parts]) if parts else np.zeros((0, EMBEDDING_DIM), np.float32)
    emb_arr = pa.FixedSizeListArray.from_arrays(pa.array(emb.reshape(-1), pa.float32()), EMBEDDING_DIM)
    schema = pa.schema(
        [
            pa.field("id", pa.int64(), False),
            pa.field("k", pa.int64(), True),
            pa.field("v", pa.float64(), True),
            pa.field("s", pa.utf8(), False),
            pa.field("emb", pa.list_(pa.field("item", pa.float32(), False), EMBEDDING_DIM), False),
        ]
    )
    return pa.RecordBatch.from_arrays(
        [
            pa.array(ids, pa.int64()),
            pa.array(k, pa.int64(), mask=~kv),
            pa.array(v, pa.float64(), mask=~vv),
            pa.array(s, pa.utf8()),
            emb_arr.cast(schema.field("emb").type),
        ],
        schema=schema,
    )


def demo_digest(batch: pa.RecordBatch) -> int:
    """FNV-1a over every value, NULL as b"null" (datagen.rs:300-330)."""
    h = 0xCBF29CE484222325
    mask = (1 << 64) - 1
    data = bytearray()
    ids = batch.column(0).to_numpy()
    k = batch.column(1)
    v = batch.column(2)
    s = batch.column(3).to_pylist()
    emb = batch.column(4).values.to_numpy().view(np.uint32).reshape(-1, EMBEDDING_DIM)
    kv = k.is_valid().to_numpy(zero_copy_only=False)
    kk = k.fill_null(0).to_numpy()
    vvld = v.is_valid().to_numpy(zero_copy_only=False)
    vbits = v.fill_null(0.0).to_numpy().view(np.uint64)
    for row in range(batch.num_rows):
        data += int(ids[row]).to_bytes(8, "little", signed=True)
        data += int(kk[row]).to_bytes(8, "little", signed=True) if kv[row] else b"null"
        data += int(vbits[row]).to_bytes(8, "little") if vvld[row] else b"null"
        data += s[row].encode()
        data += emb[row].astype("<u4").tobytes()
    for byte in bytes(data):
        h = ((h ^ byte) * 0x100000001B3) & mask
    return h


# --------------------------------------------------------------- conformance shapes

def _mask(rng, n, p=0.1):
    return rng.random(n) < p


def conformance_left(seed: int, rows: int, dim: int = 4) -> pa.RecordBatch:
    """`k Int64?`, `v Float64?` (multiples of 0.25), `s Utf8`, `vec
    FixedSizeList<Float32, 4>?` (conformance.rs:38-75)."""
    rng = np.random.default_rng(seed)
    k = rng.integers(0, 10, rows)
    v = rng.integers(0, 40, rows) / 4.0
    vals = rng.uniform(-5.0, 5.0, rows * dim).astype(np.float32)
    vec = pa.FixedSizeListArray.from_arrays(pa.array(vals, pa.float32()), dim, mask=pa.array(_mask(rng, rows)))
    return pa.RecordBatch.from_arrays(
        [
            pa.array(k, pa.int64(), mask=_mask(rng, rows)),
            pa.array(v, pa.float64(), mask=_mask(rng, rows)),
            pa.array([f"s{i % 13}" for i in range(rows)], pa.utf8()),
            vec,
        ],
        names=["k", "v", "s", "vec"],
    )


def conformance_right(seed: int, rows: int) -> pa.RecordBatch:
    """`rk Int64?`, `name Utf8` (conformance.rs:77-98)."""
    rng = np.random.default_rng(seed ^ 0xDEADBEEF)
    rk = rng.integers(0, 10, rows)
    return pa.RecordBatch.from_arrays(
        [pa.array(rk, pa.int64(), mask=_mask(rng, rows)), pa.array([f"n{i}" for i in range(rows)], pa.utf8())],
        names=["rk", "name"],
    )


SPECIAL_VALUES = [float("nan"), -float("nan"), math.inf, -math.inf, 0.0, -0.0, 4.0, 4.5, -1.0, 0.25]


def special_floats(seed: int, rows: int) -> pa.RecordBatch:
    """`k Int64?`, `v Float64?` over the special values, `s Utf8`
    (conformance.rs:1405-1430)."""
    rng = np.random.default_rng(seed ^ 0x5BEC1A1F)
    bits = np.array([np.float64(x).view(np.uint64) for x in SPECIAL_VALUES], dtype=np.uint64)
    bits[1] = np.uint64(0xFFF8000000000000)  # -NaN with its sign bit
    bits[0] = np.uint64(0x7FF8000000000000)
    v = bits[rng.integers(0, len(bits), rows)].view(np.float64)
    k = rng.integers(0, 10, rows)
    return pa.RecordBatch.from_arrays(
        [
            pa.array(k, pa.int64(), mask=_mask(rng, rows)),
            pa.array(v, pa.float64(), mask=_mask(rng, rows)),
            pa.array([f"r{i}" for i in range(rows)], pa.utf8()),
        ],
        names=["k", "v", "s"],
    )


# --------------------------------------------------------------- benchmark configs

def config1(n: int, seed: int = 0x0A11CE + 1) -> pa.RecordBatch:
    """id = 0..N-1, k U[0,10), v U[0,10), emb f32[8] ~ N(0,1)."""
    rng = np.random.default_rng(seed)
    emb = rng.standard_normal(n * 8).astype(np.float32)
    return pa.RecordBatch.from_arrays(
        [
            pa.array(np.arange(n, dtype=np.int64)),
            pa.array(rng.integers(0, 10, n, dtype=np.int64)),
            pa.array(rng.uniform(0.0, 10.0, n)),
            pa.FixedSizeListArray.from_arrays(pa.array(emb), 8),
        ],
        names=["id", "k", "v", "emb"],
    )


def zipf_ranks(rng, n: int, universe: int, s: float = 1.1) -> np.ndarray:
    """n draws of Zipf(s) ranks in [0, universe): inverse-CDF over the exact
    finite distribution."""
    w = np.arange(1, universe + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    u = rng.random(n)
    return np.searchsorted(cdf, u, side="right").clip(0, universe - 1)


def config2(build_rows: int, probe_rows: int, seed: int = 0x0A11CE + 2):
    """Build: key = a permutation of 0..B-1, attr i32 U[0,1000).  Probe: fk
    Zipf(1.1) over build keys with 5% non-matching keys (>= B), payload f64
    U(0,100), qty i32 U[1,50]."""
    rng = np.random.default_rng(seed)
    key = rng.permutation(build_rows).astype(np.int64)
    attr = rng.integers(0, 1000, build_rows, dtype=np.int32)
    ranks = zipf_ranks(rng, probe_rows, build_rows)
    fk = key[ranks]
    miss = rng.random(probe_rows) < 0.05
    fk = np.where(miss, build_rows + rng.integers(0, build_rows, probe_rows), fk).astype(np.int64)
    payload = rng.uniform(0.0, 100.0, probe_rows)
    qty = rng.integers(1, 51, probe_rows, dtype=np.int32)
    build = pa.RecordBatch.from_arrays([pa.array(key), pa.array(attr)], names=["key", "attr"])
    probe = pa.RecordBatch.from_arrays([pa.array(fk), pa.array(payload), pa.array(qty)], names=["fk", "payload", "qty"])
    return build, probe


def config3_batches(total_rows: int, distinct: int, seed: int = 0x0A11CE + 3, min_rows: int = 8192,
                    max_rows: int = 1 << 20):
    """High-cardinality input as uneven RecordBatches: g i64 uniform over
    `distinct` values, x i32 U(-1e6, 1e6) with 2% NULLs, f i32 U[0,100) (the
    filter column: `f < s` keeps s %).  Batch sizes are seeded in
    [min_rows, max_rows]."""
    rng = np.random.default_rng(seed)
    batches = []
    left = total_rows
    while left > 0:
        n = int(min(left, rng.integers(min_rows, max_rows + 1)))
        g = rng.integers(0, distinct, n, dtype=np.int64)
        x = rng.integers(-1_000_000, 1_000_001, n, dtype=np.int32)
        f = rng.integers(0, 100, n, dtype=np.int32)
        batches.append(
            pa.RecordBatch.from_arrays(
                [pa.array(g), pa.array(x, mask=rng.random(n) < 0.02), pa.array(f)], names=["g", "x", "f"]
            )
        )
        left -= n
    return batches
