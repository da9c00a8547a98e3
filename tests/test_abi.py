"""The C ABI library without a GPU: it loads, exports exactly what
include/oxb200.h declares, and the ctypes structs match the C layouts.
No compute call runs here."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "oxb200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"OXB_API\s+[\w\s\*]+?\b(oxb_\w+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    from oxidelake_b200 import _abi

    lib = _abi.lib()
    syms = declared_symbols()
    assert len(syms) > 40
    for s in syms:
        assert hasattr(lib, s), s
    # Every declared entry point has a ctypes prototype, and no more.
    assert sorted(_abi.PROTOTYPES) == syms
    out = subprocess.run(["nm", "-D", "--defined-only", str(_abi.LIB_PATH)], capture_output=True, text=True).stdout
    exported = sorted(set(re.findall(r" T (oxb_\w+)", out)))
    assert exported == syms


def test_abi_version_and_kind_without_a_device():
    from oxidelake_b200 import _abi

    assert _abi.lib().oxb_abi_version() == 1
    assert _abi.lib().oxb_backend_kind(None) == b"cuda"


def test_errors_map_to_engine_error_kinds():
    from oxidelake_b200 import errors

    assert errors.error_for(1, "x").is_unsupported()
    assert isinstance(errors.error_for(7, "x"), errors.TableFull)
    assert not errors.error_for(4, "x").is_unsupported()


LAYOUT_PROBE = r"""
#include <stdio.h>
#include <stddef.h>
#include "oxb200.h"
#define S(t) printf(#t " %zu\n", sizeof(t));
#define O(t, f) printf(#t "." #f " %zu\n", offsetof(t, f));
int main(void) {
  S(oxb_column) S(oxb_leaf) S(oxb_memory_info) S(oxb_filter_project_args) S(oxb_join_index)
  S(oxb_join_build_args) S(oxb_join_probe_args) S(oxb_hash_join_args) S(oxb_aggregate_spec)
  S(oxb_aggregate_args) S(oxb_vector_distance_args) S(oxb_join_aggregate_args)
  S(oxb_call_stats) S(oxb_operator_stats)
  O(oxb_leaf, lit) O(oxb_call_stats, batches) O(oxb_operator_stats, fallback_batches) O(oxb_hash_join_args, projection) O(oxb_join_aggregate_args, funcs)
  O(oxb_join_aggregate_args, columns) O(oxb_vector_distance_args, query)
  return 0;
}
"""


def test_ctypes_structs_match_the_c_layout(tmp_path):
    from oxidelake_b200 import _abi

    src = tmp_path / "probe.c"
    src.write_text(LAYOUT_PROBE)
    exe = tmp_path / "probe"
    r = subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.skip("no C compiler: " + r.stderr[:200])
    got = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split("\n") if line)
    py = {
        "oxb_column": _abi.Column,
        "oxb_leaf": _abi.Leaf,
        "oxb_memory_info": _abi.MemoryInfo,
        "oxb_filter_project_args": _abi.FilterProjectArgs,
        "oxb_join_index": _abi.JoinIndex,
        "oxb_join_build_args": _abi.JoinBuildArgs,
        "oxb_join_probe_args": _abi.JoinProbeArgs,
        "oxb_hash_join_args": _abi.HashJoinArgs,
        "oxb_aggregate_spec": _abi.AggregateSpecC,
        "oxb_aggregate_args": _abi.AggregateArgs,
        "oxb_vector_distance_args": _abi.VectorDistanceArgs,
        "oxb_join_aggregate_args": _abi.JoinAggregateArgs,
        "oxb_call_stats": _abi.CallStats,
        "oxb_operator_stats": _abi.OperatorStats,
    }
    for name, cls in py.items():
        assert int(got[name]) == C.sizeof(cls), name
    assert int(got["oxb_leaf.lit"]) == _abi.Leaf.lit.offset
    assert int(got["oxb_hash_join_args.projection"]) == _abi.HashJoinArgs.projection.offset
    assert int(got["oxb_join_aggregate_args.funcs"]) == _abi.JoinAggregateArgs.funcs.offset
    assert int(got["oxb_join_aggregate_args.columns"]) == _abi.JoinAggregateArgs.columns.offset
    assert int(got["oxb_vector_distance_args.query"]) == _abi.VectorDistanceArgs.query.offset
    assert int(got["oxb_call_stats.batches"]) == _abi.CallStats.batches.offset
    assert int(got["oxb_operator_stats.fallback_batches"]) == _abi.OperatorStats.fallback_batches.offset


def test_call_stats_record_refused_calls_without_a_device():
    """Each operator entry point leaves its counters for
    oxb_last_call_stats even when it fails before any device work: a filter
    and a join given no backend are recorded under their operator with the
    PLAN status and no rows."""
    from oxidelake_b200 import _abi

    lib = _abi.lib()
    out = C.c_void_p()
    args = _abi.FilterProjectArgs(None, None, 0, None, 0)
    assert lib.oxb_filter_project(None, None, C.byref(args), C.byref(out)) == 4
    st = _abi.CallStats()
    assert lib.oxb_last_call_stats(C.byref(st)) == 0
    assert (st.op, st.status, st.rows_out, st.bytes_h2d) == (_abi.OP_FILTER, 4, 0, 0)
    jargs = _abi.JoinProbeArgs()
    assert lib.oxb_probe_join(None, None, C.byref(jargs), C.byref(out)) == 4
    assert lib.oxb_last_call_stats(C.byref(st)) == 0
    assert (st.op, st.status) == (_abi.OP_JOIN, 4)
    ops = _abi.OperatorStats()
    assert lib.oxb_operator_stats_get(None, _abi.OP_FILTER, C.byref(ops), 0) == 4


def test_backend_create_fails_loudly_without_a_gpu():
    """No silent CPU path: creating the backend on a machine with no CUDA
    device raises a Device error rather than returning something."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from oxidelake_b200.backend import CudaBackend
    from oxidelake_b200.errors import EngineError

    with pytest.raises(EngineError):
        CudaBackend(0)
