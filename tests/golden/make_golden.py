"""Writes tests/golden/reference_vectors.json: the golden vectors the
reference's own tests hold for the GPU operator path, transcribed case by
case with the file and line each comes from (paths inside the reference
project).  Floats are stored as their IEEE-754 bit patterns (hex), so NaN
signs and -0.0 survive.

    python tests/golden/make_golden.py

The reference is Rust and cannot run in this environment (no toolchain), so
these vectors are written out from its test sources; nothing here executes
reference code.
"""
from __future__ import annotations

import json
import math
import struct
from pathlib import Path

OUT = Path(__file__).resolve().parent / "reference_vectors.json"

I64_MAX = 2**63 - 1
I64_MIN = -(2**63)


def fbits(x: float) -> str:
    return "0x%016x" % struct.unpack("<Q", struct.pack("<d", x))[0]


NAN = "0x7ff8000000000000"      # f64::NAN
NEG_NAN = "0xfff8000000000000"  # -f64::NAN
INF = fbits(math.inf)
NEG_INF = fbits(-math.inf)
ZERO = fbits(0.0)
NEG_ZERO = fbits(-0.0)


def f(x):
    return None if x is None else (x if isinstance(x, str) else fbits(x))


def main() -> None:
    g = {}

    # cpu/kernels.rs:946-974 (batch) and :976-988
    g["filter_drops_null_predicates_and_projects"] = {
        "source": "crates/oxidelake-device/src/cpu/kernels.rs:976-988",
        "k": [1, 2, None, 2, 5],
        "v": [f(0.5), None, f(2.5), f(3.5), f(-1.0)],
        "s": ["a", "b", "c", None, "e"],
        "leaves": [[0, "GtEq", "Int64", 2], [1, "Lt", "Float64", f(4.0)]],
        "projection": [2, 0],
        "expect_names": ["s", "k"],
        "expect_k": [2, 5],
    }

    # cpu/kernels.rs:991-1021
    g["float_comparisons_order_as_datafusion_does"] = {
        "source": "crates/oxidelake-device/src/cpu/kernels.rs:991-1021",
        "values": [NAN, NEG_NAN, INF, NEG_INF, ZERO, NEG_ZERO, f(4.0)],
        "cases": [
            ["Gt", f(4.0), [0, 2]],
            ["Lt", NEG_INF, [1]],
            ["Eq", NAN, [0]],
            ["Eq", ZERO, [4, 5]],
            ["Eq", NEG_ZERO, [4, 5]],
            ["Lt", ZERO, [1, 3]],
            ["GtEq", NEG_ZERO, [0, 2, 4, 5, 6]],
        ],
    }

    # cpu/kernels.rs:1023-1031
    g["filter_type_mismatch_is_unsupported"] = {
        "source": "crates/oxidelake-device/src/cpu/kernels.rs:1023-1031",
        "leaf": [1, "Eq", "Int64", 1],
        "projection": [0],
    }

    # cpu/kernels.rs:1033-1058
    g["join_skips_null_keys_and_multiplies_matches"] = {
        "source": "crates/oxidelake-device/src/cpu/kernels.rs:1033-1058",
        "rk": [2, 2, None, 9],
        "name": ["two-a", "two-b", "null", "nine"],
        "expect_columns": 5,
        "expect_rows": 4,
        "expect_sorted_names": ["two-a", "two-a", "two-b", "two-b"],
    }

    # cpu/kernels.rs:1063-1121
    g["join_matches_gather_in_ranges_equal_one_gather"] = {
        "source": "crates/oxidelake-device/src/cpu/kernels.rs:1063-1121",
        "rk": [2, 2, None, 9, 2, 5],
        "name": ["a", "b", "null", "nine", "c", "five"],
        "expect_matches": 7,
        "projection": [0, 1, 3, 4],
        "chunks": [1, 2, 3, 4, 5, 6, 7, 8],
        # the pairs follow from probe order then build order (cpu/kernels.rs:303-318)
        "expect_pairs": [[1, 0], [1, 1], [1, 4], [3, 0], [3, 1], [3, 4], [4, 5]],
        "out_of_range": [[7, 1], [0, 18446744073709551615]],
    }

    # cpu/kernels.rs:1123-1158
    g["aggregate_groups_nulls_last_and_skips_null_values"] = {
        "source": "crates/oxidelake-device/src/cpu/kernels.rs:1123-1158",
        "aggregates": [["Sum", 1], ["Count", 1], ["Min", 1], ["Max", 0]],
        "expect_keys": [1, 2, 5, None],
        "expect_sums": [f(0.5), f(3.5), f(-1.0), f(2.5)],
        "expect_counts": [1, 1, 1, 1],
        "expect_name_1": "SUM(v)",
        "expect_name_4": "MAX(k)",
        "expect_maxk": [1, 2, 5, None],
    }

    # cpu/kernels.rs:1209-1288
    g["batch_by_batch_and_merged_partials_equal_one_pass"] = {
        "source": "crates/oxidelake-device/src/cpu/kernels.rs:1209-1288",
        "rows": [
            [1, I64_MAX - 1, f(1.0)],
            [2, 5, NAN],
            [None, I64_MAX, NEG_ZERO],
            [1, I64_MAX - 1, NAN],
            [3, None, None],
            [4, I64_MIN, NEG_NAN],
            [None, I64_MAX, ZERO],
            [1, -3, f(3.0)],
            [4, 7, NEG_INF],
            [2, -1, f(0.25)],
        ],
        "aggregates": [["Sum", 1], ["Count", 1], ["Min", 1], ["Max", 1], ["Sum", 2], ["Count", 2], ["Min", 2], ["Max", 2]],
        "expect_col1": [-7, 4, None, I64_MIN + 7, -2],
        "expect_col7_bits": [f(1.0), f(0.25), None, NEG_NAN, NEG_ZERO],
        "expect_col8_bits": [NAN, NAN, None, NEG_INF, ZERO],
    }

    # cpu/kernels.rs:1303-1313
    g["aggregate_over_empty_batch_has_no_groups"] = {
        "source": "crates/oxidelake-device/src/cpu/kernels.rs:1303-1313",
        "expect_rows": 0,
        "expect_columns": 2,
    }

    # cpu/kernels.rs:1318-1358
    g["total_order_keys"] = {
        "source": "crates/oxidelake-device/src/cpu/kernels.rs:1318-1358",
        "values_in_order": [
            "0xffffffffffffffff",
            NEG_NAN,
            NEG_INF,
            fbits(-1.7976931348623157e308),
            fbits(-1.0),
            "0x8000000000000001",
            NEG_ZERO,
            ZERO,
            "0x0000000000000001",
            fbits(2.2250738585072014e-308),
            fbits(1.0),
            fbits(1.7976931348623157e308),
            INF,
            "0x7ff0000000000001",
            NAN,
            "0x7fffffffffffffff",
        ],
        "from_key_max_bits": "0x7fffffffffffffff",
        "from_key_min_bits": "0xffffffffffffffff",
    }

    # cpu/kernels.rs:1360-1396
    g["vector_distances"] = {
        "source": "crates/oxidelake-device/src/cpu/kernels.rs:1360-1396",
        "dim": 2,
        "values": [1.0, 0.0, 0.0, 1.0, 3.0, 4.0],
        "valid": [True, False, True],
        "query": [1.0, 0.0],
        "expect_l2": [0.0, None, "sqrt20"],
        "expect_cosine_approx": [0.0, None, 1.0 - 3.0 / 5.0],
        "cosine_tolerance": 1e-6,
        "zero_norm_cosine_is_nan": [[0.0, 0.0], [1.0, 0.0]],
    }

    # crates/oxidelake-compute/tests/conformance.rs:306-356 and cuda/mod.rs:993-1065
    g["sum_overflow_wraps"] = {
        "source": "crates/oxidelake-compute/tests/conformance.rs:306-356",
        "rows": [
            [1, I64_MAX - 1],
            [2, 5],
            [1, I64_MAX - 1],
            [3, I64_MIN],
            [4, I64_MAX],
            [3, -1],
            [None, I64_MAX],
            [4, 1],
            [None, I64_MAX],
            [4, -2],
        ],
        "expect_rows": ["1|-4|2", "2|5|1", "3|9223372036854775807|2", "4|9223372036854775806|3", "NULL|-2|2"],
        "device_source": "crates/oxidelake-device/src/cuda/mod.rs:993-1065",
        "device_expect_sums": [-4, 5, I64_MAX, I64_MAX - 1, -2],
    }

    # conformance.rs:428-449 (groups) and cuda/mod.rs:1071-1153 (device bits)
    g["float_min_max_total_order"] = {
        "source": "crates/oxidelake-compute/tests/conformance.rs:428-449",
        "groups": [
            [1, [f(1.0), NAN, f(3.0)], [f(1.0), NAN]],
            [2, [NAN, NAN], [NAN, NAN]],
            [3, [ZERO, NEG_ZERO], [NEG_ZERO, ZERO]],
            [4, [NEG_ZERO, ZERO], [NEG_ZERO, ZERO]],
            [5, [INF, NAN], [INF, NAN]],
            [6, [NEG_INF], [NEG_INF, NEG_INF]],
            [7, [INF], [INF, INF]],
            [8, [f(1.0), NEG_NAN], [NEG_NAN, f(1.0)]],
            [None, [NAN, f(2.0)], [f(2.0), NAN]],
        ],
        "device_source": "crates/oxidelake-device/src/cuda/mod.rs:1071-1153",
        "device_rows": [
            [1, f(1.0)], [1, NAN], [1, f(3.0)], [2, NAN], [2, NAN], [3, ZERO], [3, NEG_ZERO], [4, NEG_ZERO],
            [4, ZERO], [5, INF], [5, NAN], [6, NEG_INF], [7, f(1.0)], [7, NEG_NAN], [None, NAN], [None, f(2.0)],
        ],
        "device_expect_min": [f(1.0), NAN, NEG_ZERO, NEG_ZERO, INF, NEG_INF, NEG_NAN, f(2.0)],
        "device_expect_max": [NAN, NAN, ZERO, ZERO, NAN, NEG_INF, f(1.0), NAN],
    }

    # conformance.rs:607-646
    g["signed_zeros"] = {
        "source": "crates/oxidelake-compute/tests/conformance.rs:607-646",
        "one_sign_rows": [
            [1, NEG_ZERO], [1, NEG_ZERO], [2, ZERO], [2, ZERO], [3, NEG_ZERO], [3, f(1.0)], [4, f(-1.0)], [4, ZERO], [None, NEG_ZERO],
        ],
        # stock DataFusion's order-free answers for one sign per group
        "one_sign_expect": [
            [1, NEG_ZERO, NEG_ZERO], [2, ZERO, ZERO], [3, NEG_ZERO, f(1.0)], [4, f(-1.0), ZERO], [None, NEG_ZERO, NEG_ZERO],
        ],
        "both_zeros_expect": [NEG_ZERO, ZERO],
    }

    # conformance.rs:1405-1450 special-float filters (predicates only; rows by hand)
    g["special_float_filter_predicates"] = {
        "source": "crates/oxidelake-compute/tests/conformance.rs:1432-1456",
        "values": [NAN, NEG_NAN, INF, NEG_INF, ZERO, NEG_ZERO, f(4.0), f(4.5), f(-1.0), f(0.25)],
        "predicates": [
            [["v", "Gt", f(4.0)]],
            [["v", "GtEq", f(4.5)]],
            [["v", "Lt", ZERO]],
            [["v", "Gt", NEG_ZERO]],
            [["v", "LtEq", NEG_ZERO]],
            [["v", "Eq", ZERO]],
            [["v", "Eq", NEG_ZERO]],
            [["v", "GtEq", NAN]],
            [["v", "Eq", NAN]],
            [["v", "Gt", INF]],
            [["v", "Lt", NEG_INF]],
            [["k", "GtEq", 2], ["v", "Gt", f(4.0)]],
        ],
        "shapes": {"seeds": [1, 7, 42], "sizes": [0, 1, 7, 64, 1000], "null_fraction": 0.1, "k_range": [0, 10]},
    }

    # join_slots.rs:174-179
    g["slot_hash"] = {
        "source": "crates/oxidelake-device/src/join_slots.rs:174-179",
        "cases": [[0, 16, 0], [1, 16, 12], [-1, 1024, 801], [42, 131072, 22988], [I64_MIN, 1 << 20, 107667]],
    }

    # storage/src/datagen.rs:348-354
    g["demo_table_digest"] = {
        "source": "crates/oxidelake-storage/src/datagen.rs:348-354",
        "rows": 65536 + 1000,
        "seed": 42,
        "chunk_rows": 65536,
        "digest": 13955388935552808329,
    }

    # cuda/mod.rs:1161-1260 (device group-numbering cases, generated by splitmix64 from state 29)
    g["aggregate_numbering_cases"] = {
        "source": "crates/oxidelake-device/src/cuda/mod.rs:1161-1260",
        "state": 29,
        "cases": ["no rows", "only NULL keys", "a group per row", "extreme keys", "100 keys in one GPU batch"],
    }

    # conformance.rs:34-75 shapes (StdRng cannot be reproduced; shapes only)
    g["conformance_shapes"] = {
        "source": "crates/oxidelake-compute/tests/conformance.rs:34-75",
        "dim": 4,
        "sizes": [0, 1, 7, 64, 1000],
        "seeds": [1, 7, 42],
        "null_fraction": 0.1,
        "k_range": [0, 10],
        "v_quarters": [0, 40],
        "vec_range": [-5.0, 5.0],
    }

    OUT.write_text(json.dumps(g, indent=1) + "\n")
    print(OUT)


if __name__ == "__main__":
    main()
