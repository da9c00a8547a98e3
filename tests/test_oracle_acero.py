"""The oracle's aggregate semantics that no reference test pins, checked
against Arrow C++'s own engine (pyarrow.acero) on the same inputs.  CPU only.

The reference's CPU path is DataFusion 55.3 (its Cargo.lock), which this
image cannot run.  Its documented semantics for the functions the north-star
queries add beyond the reference's tests are also Arrow's:
  * AVG(Float64) and AVG(Int32) -> Float64, NULL for a group with no values
    (datafusion-functions-aggregate `Avg`; Arrow `hash_mean`);
  * COUNT(*) counts every row of the group, NULL inputs included
    (`count(*)` -> `hash_count` with mode "all");
  * SUM(Int32) -> Int64 (DataFusion widens; Arrow `hash_sum` of int32 gives
    int64), NULL when the group has no values;
  * MIN/MAX(Int32) -> Int32;
  * COUNT(col) counts non-NULL values;
  * an inner equi-join drops NULL keys on either side and multiplies
    duplicate matches.
The oracle (a C restatement of crates/oxidelake-device/src/cpu/kernels.rs
plus those widened functions) must agree with acero on all of them:
integers, counts and keys exactly, Float64 within 1e-12 of
max(|result|, mean of |x|) — Arrow's float sums are pairwise, not sequential.
Acero does not order its groups; both sides are sorted by key, NULL last,
as GpuAggregateExec emits them (compute/src/exec/aggregate.rs:35-66).
"""
import numpy as np
import pyarrow as pa
import pyarrow.acero as ac
import pyarrow.compute as pc
import pytest

import oracle
from datagen import config1, config2, config3_batches

SUM, COUNT, MIN, MAX, AVG, COUNT_STAR = 0, 1, 2, 3, 4, 5
ACERO = {SUM: "hash_sum", COUNT: "hash_count", MIN: "hash_min", MAX: "hash_max", AVG: "hash_mean"}
RTOL = 1e-12


def _source(table):
    return ac.Declaration("table_source", ac.TableSourceNodeOptions(table))


def acero_group_by(table: pa.Table, key: str, aggs, where=None, input_names=None) -> pa.Table:
    """GROUP BY `key` over `table` in acero, optionally after a filter
    expression; `aggs` are (function, column name) pairs.  Output columns:
    the key, then one per aggregate, rows sorted by key with NULL last."""
    names = []
    specs = []
    for j, (f, col) in enumerate(aggs):
        name = f"a{j}"
        names.append(name)
        if f == COUNT_STAR:
            specs.append(((key,), "hash_count", pc.CountOptions(mode="all"), name))
        elif f == COUNT:
            specs.append(((col,), "hash_count", pc.CountOptions(mode="only_valid"), name))
        else:
            specs.append(((col,), ACERO[f], None, name))
    steps = [_source(table)]
    if where is not None:
        steps.append(ac.Declaration("filter", ac.FilterNodeOptions(where)))
    steps.append(ac.Declaration("aggregate", ac.AggregateNodeOptions(specs, keys=[key])))
    out = ac.Declaration.from_sequence(steps).to_table()
    out = out.select([key] + names)
    return out.sort_by([(key, "ascending")], null_placement="at_end") if out.num_rows else out


def acero_join(probe: pa.Table, build: pa.Table, probe_key: str, build_key: str) -> pa.Table:
    """probe INNER JOIN build ON probe_key = build_key, in acero."""
    opts = ac.HashJoinNodeOptions("inner", left_keys=[probe_key], right_keys=[build_key])
    return ac.Declaration("hashjoin", opts, inputs=[_source(probe), _source(build)]).to_table()


def _arr(c):
    return c.combine_chunks() if isinstance(c, pa.ChunkedArray) else c


def assert_same(got: pa.RecordBatch, want: pa.Table, float_cols=(), scale=None) -> None:
    """`got` (the oracle) against `want` (acero): the same groups, types and
    values; the columns in `float_cols` to RTOL of max(|want|, scale)."""
    assert got.num_rows == want.num_rows, (got.num_rows, want.num_rows)
    assert got.num_columns == want.num_columns
    for i in range(got.num_columns):
        g, w = _arr(got.column(i)), _arr(want.column(i))
        assert g.type == w.type, (got.schema.field(i).name, g.type, w.type)
        gv = g.is_valid().to_numpy(zero_copy_only=False)
        wv = w.is_valid().to_numpy(zero_copy_only=False)
        assert (gv == wv).all(), f"{got.schema.field(i).name}: validity differs"
        if pa.types.is_floating(g.type):
            gx = g.fill_null(0.0).to_numpy(zero_copy_only=False)
            wx = w.fill_null(0.0).to_numpy(zero_copy_only=False)
            if i in float_cols:
                mag = np.abs(wx) if scale is None else np.maximum(np.abs(wx), scale[i])
                bad = ~((np.abs(gx - wx) <= RTOL * mag) | (gx == wx))
            else:
                bad = gx.view(np.uint64) != wx.view(np.uint64)
        else:
            bad = g.fill_null(0).to_numpy(zero_copy_only=False) != w.fill_null(0).to_numpy(zero_copy_only=False)
        bad &= gv
        assert not bad.any(), f"{got.schema.field(i).name}: differs at groups {np.nonzero(bad)[0][:5].tolist()}"


def _mean_abs(table: pa.Table, key: str, col: str, where=None) -> np.ndarray:
    """Per group (sorted as acero_group_by sorts), the mean of |col|: the
    scale of an AVG's rounding."""
    t = table.append_column("__abs", pc.abs(table.column(col)))
    m = acero_group_by(t, key, [(AVG, "__abs")], where)
    return m.column(1).fill_null(0.0).to_numpy(zero_copy_only=False)


def _with_nulls(n, rng, p):
    return rng.random(n) < p


def test_config1_shape_sum_avg_count_star():
    """SELECT k, SUM(v), AVG(v), COUNT(*), COUNT(v), MIN(v), MAX(v)
    WHERE k >= 2 AND v < 4.0 GROUP BY k over config-1-shaped data with NULL
    keys and values."""
    rng = np.random.default_rng(101)
    b = config1(200_000)
    n = b.num_rows
    k = pa.array(b.column(1).to_numpy(), pa.int64(), mask=_with_nulls(n, rng, 0.03))
    v = pa.array(b.column(2).to_numpy(), pa.float64(), mask=_with_nulls(n, rng, 0.05))
    batch = pa.RecordBatch.from_arrays([b.column(0), k, v], names=["id", "k", "v"])
    aggs = [(SUM, 2), (AVG, 2), (COUNT_STAR, 0), (COUNT, 2), (MIN, 2), (MAX, 2)]
    leaves = [(1, 4, 1, 2), (2, 1, 2, 4.0)]  # k >= 2, v < 4.0
    got = oracle.aggregate(batch, 1, aggs, leaves)
    table = pa.Table.from_batches([batch])
    where = (pc.field("k") >= 2) & (pc.field("v") < 4.0)
    want = acero_group_by(table, "k", [(f, batch.schema.names[c]) for f, c in aggs], where)
    assert_same(got, want, float_cols=(1, 2))


def test_config1_shape_without_where_keeps_the_null_group():
    rng = np.random.default_rng(102)
    n = 100_000
    k = pa.array(rng.integers(0, 10, n), pa.int64(), mask=_with_nulls(n, rng, 0.1))
    v = pa.array(rng.uniform(-10, 10, n), pa.float64(), mask=_with_nulls(n, rng, 0.1))
    batch = pa.RecordBatch.from_arrays([k, v], names=["k", "v"])
    aggs = [(AVG, 1), (COUNT_STAR, 0), (SUM, 1), (COUNT, 1)]
    got = oracle.aggregate(batch, 0, aggs)
    table = pa.Table.from_batches([batch])
    want = acero_group_by(table, "k", [(f, batch.schema.names[c]) for f, c in aggs])
    assert not want.column(0).combine_chunks().is_valid().to_numpy(zero_copy_only=False)[-1]
    # AVG's and SUM's values cancel: the rounding scale is the mean (sum) of |v|.
    mabs = _mean_abs(table, "k", "v")
    counts = want.column(4).to_numpy()
    scale = np.zeros((5, want.num_rows))
    scale[1] = mabs
    scale[3] = mabs * counts
    assert_same(got, want, float_cols=(1, 3), scale=scale)


def test_int32_widening_sum_min_max_avg():
    """SUM(Int32) -> Int64, MIN/MAX(Int32) -> Int32, AVG(Int32) -> Float64,
    COUNT(Int32), under WHERE f < 50, over config-3-shaped batches with an
    Int32 group key too."""
    batches = config3_batches(400_000, 20_000, seed=103, min_rows=5000, max_rows=90_000)
    table = pa.Table.from_batches(batches).combine_chunks()
    whole = table.to_batches()[0]
    aggs = [(SUM, 1), (MIN, 1), (MAX, 1), (COUNT, 1), (AVG, 1), (COUNT_STAR, 0)]
    leaves = [(2, 1, 3, 50)]  # f < 50 (Int32 literal)
    got = oracle.aggregate(whole, 0, aggs, leaves)
    want = acero_group_by(table, "g", [(f, whole.schema.names[c]) for f, c in aggs], pc.field("f") < 50)
    assert got.schema.field(1).type == pa.int64() and got.schema.field(2).type == pa.int32()
    assert got.schema.field(5).type == pa.float64()
    assert_same(got, want, float_cols=(5,))

    # The same over an Int32 group key (the join's attr is one), with NULL keys.
    rng = np.random.default_rng(104)
    n = whole.num_rows
    g32 = pa.array((whole.column(0).to_numpy() % 997).astype(np.int32), pa.int32(), mask=_with_nulls(n, rng, 0.02))
    b32 = pa.RecordBatch.from_arrays([g32, whole.column(1), whole.column(2)], names=["g", "x", "f"])
    got = oracle.aggregate(b32, 0, aggs, leaves)
    want = acero_group_by(pa.Table.from_batches([b32]), "g", [(f, b32.schema.names[c]) for f, c in aggs],
                          pc.field("f") < 50)
    assert got.schema.field(0).type == pa.int32()
    assert_same(got, want, float_cols=(5,))


def test_groups_with_only_null_inputs():
    """SUM, MIN, MAX and AVG of a group whose inputs are all NULL are NULL;
    COUNT(col) is 0 and COUNT(*) the group's rows."""
    k = pa.array([1, 1, 2, 2, 2, None, 3], pa.int64())
    x = pa.array([None, None, 5, None, -7, None, 2**31 - 1], pa.int32())
    v = pa.array([None, None, 1.5, 2.5, None, None, -0.25], pa.float64())
    batch = pa.RecordBatch.from_arrays([k, x, v], names=["k", "x", "v"])
    aggs = [(SUM, 1), (MIN, 1), (MAX, 1), (AVG, 1), (COUNT, 1), (COUNT_STAR, 0), (AVG, 2), (SUM, 2)]
    got = oracle.aggregate(batch, 0, aggs)
    want = acero_group_by(pa.Table.from_batches([batch]), "k", [(f, batch.schema.names[c]) for f, c in aggs])
    assert_same(got, want, float_cols=(4, 7, 8))
    assert got.column(1).to_pylist() == [None, -2, 2**31 - 1, None]


@pytest.mark.parametrize("with_nulls", [False, True], ids=["config2", "nulls-and-duplicates"])
def test_join_aggregate_config2_shape(with_nulls):
    """probe JOIN build ON fk = key WHERE qty > 10 GROUP BY attr:
    SUM(payload), SUM(qty), COUNT(*), AVG(payload), MIN(qty), MAX(qty) —
    the oracle's fused join-aggregate against acero's hash join followed by
    its group-by."""
    build, probe = config2(20_000, 400_000, seed=105)
    if with_nulls:
        rng = np.random.default_rng(106)
        nb, npr = build.num_rows, probe.num_rows
        key = build.column(0).to_numpy().copy()
        key[rng.integers(0, nb, nb // 20)] = key[rng.integers(0, nb, nb // 20)]  # repeated build keys
        build = pa.RecordBatch.from_arrays(
            [pa.array(key, mask=_with_nulls(nb, rng, 0.02)),
             pa.array(build.column(1).to_numpy(), pa.int32(), mask=_with_nulls(nb, rng, 0.02))],
            names=["key", "attr"])
        probe = pa.RecordBatch.from_arrays(
            [pa.array(probe.column(0).to_numpy(), mask=_with_nulls(npr, rng, 0.02)),
             pa.array(probe.column(1).to_numpy(), mask=_with_nulls(npr, rng, 0.05)),
             pa.array(probe.column(2).to_numpy(), pa.int32(), mask=_with_nulls(npr, rng, 0.02))],
            names=["fk", "payload", "qty"])
    aggs = [(SUM, 0, 1), (SUM, 0, 2), (COUNT_STAR, 0, 0), (AVG, 0, 1), (MIN, 0, 2), (MAX, 0, 2)]
    got = oracle.join_aggregate(probe, build, 0, 0, [(2, 3, 3, 10)], (1, 1), aggs, threads=4)
    joined = acero_join(pa.Table.from_batches([probe]), pa.Table.from_batches([build]), "fk", "key")
    want = acero_group_by(joined, "attr", [(f, probe.schema.names[c]) for f, _, c in aggs], pc.field("qty") > 10)
    assert_same(got, want, float_cols=(1, 4))
