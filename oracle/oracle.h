/*
 * oracle.h — CPU restatement of OxideLake's reference semantics for the GPU
 * operator path.  TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check
 * and the CPU-baseline leg of the benchmark call it as the checker; the
 * product (liboxb200.so) never links, loads or calls it.
 *
 * Follows crates/oxidelake-device/src/cpu/kernels.rs of the reference (file
 * and line cited per function in oracle.c).  Parity is pinned against the
 * reference's own golden vectors (tests/golden/, generated by
 * tests/golden/make_golden.py from the reference's test files).
 *
 * Column and leaf structs have the same layout as oxb_column / oxb_leaf in
 * include/oxb200.h, so one descriptor serves both.
 */
#ifndef OXB_ORACLE_H
#define OXB_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_INT64 = 1, ORC_FLOAT64 = 2, ORC_INT32 = 3, ORC_FLOAT32 = 4, ORC_VECTOR_F32 = 5 };
enum { ORC_EQ = 0, ORC_LT = 1, ORC_LTEQ = 2, ORC_GT = 3, ORC_GTEQ = 4 };
enum { ORC_SUM = 0, ORC_COUNT = 1, ORC_MIN = 2, ORC_MAX = 3, ORC_AVG = 4, ORC_COUNT_STAR = 5 };
enum { ORC_L2 = 0, ORC_COSINE = 1 };
/* Return codes (negative): EngineError kinds. */
enum { ORC_OK = 0, ORC_ERR_UNSUPPORTED = -1, ORC_ERR_PLAN = -4, ORC_ERR_EXECUTION = -3 };

typedef struct orc_column {
    int32_t type;
    int32_t dim;
    int64_t length;
    const void* values;
    const uint8_t* validity;
} orc_column;

typedef struct orc_leaf {
    int32_t column;
    int32_t op;
    int32_t lit_type;
    int32_t reserved;
    union {
        int64_t i;
        double f;
    } lit;
} orc_leaf;

#define ORC_MAX_AGGREGATES 16
typedef struct orc_agg_spec {
    int32_t group_by;
    int32_t naggregates;
    int32_t funcs[ORC_MAX_AGGREGATES];
    int32_t columns[ORC_MAX_AGGREGATES];
} orc_agg_spec;

/* ---- scalar helpers ---- */
int64_t orc_total_order_key(double x);
double orc_from_total_order_key(int64_t key);
int64_t orc_filter_order_key(double x);
uint32_t orc_slot_hash(int64_t key, uint32_t capacity);
float orc_l2(const float* a, const float* b, int64_t dim);
float orc_cosine(const float* a, const float* b, int64_t dim);

/* ---- filter ---- */
/* Selected rows (ascending) into out_rows; returns their number or an error. */
int64_t orc_filter(const orc_column* cols, int32_t ncols, const orc_leaf* leaves, int32_t nleaves,
                   uint32_t* out_rows);

/* ---- join ---- */
typedef struct orc_join_table orc_join_table;
int32_t orc_join_build(const orc_column* key, orc_join_table** out);
void orc_join_free(orc_join_table* t);
int64_t orc_join_distinct(const orc_join_table* t);
int64_t orc_join_nrows(const orc_join_table* t);
/* Runs (key, start, count), in the table's own order, and the row array. */
void orc_join_export(const orc_join_table* t, int64_t* keys, uint32_t* starts, uint32_t* counts,
                     uint32_t* rows);
/* offsets: nprobe + 1 entries; starts: nprobe entries.  Returns total. */
int64_t orc_join_probe(const orc_join_table* t, const orc_column* key, uint64_t* offsets,
                       uint32_t* starts);
int32_t orc_join_pairs(const orc_join_table* t, const uint64_t* offsets, const uint32_t* starts,
                       int64_t nprobe, uint64_t first, uint64_t rows, uint32_t* left,
                       uint32_t* right);

/* ---- grouped aggregation (GroupedAggregator) ---- */
typedef struct orc_agg orc_agg;
int32_t orc_agg_new(const orc_column* schema_cols, int32_t ncols, const orc_agg_spec* spec,
                    orc_agg** out);
int32_t orc_agg_update(orc_agg* a, const orc_column* cols, int32_t ncols, const orc_leaf* leaves,
                       int32_t nleaves);
/* Folds a partial laid out as this aggregation's output (key, then one
 * column per aggregate; AVG partials are not mergeable and are refused). */
int32_t orc_agg_merge(orc_agg* a, const orc_column* partial, int32_t ncols);
int64_t orc_agg_groups(const orc_agg* a);
/* Writes the finished groups sorted by key, NULL last: key values (as
 * int64) and validity (1 byte per group), then per aggregate 8-byte values
 * (int64 or double bits; Int32 MIN/MAX widened) and 1-byte validity. */
void orc_agg_finish(const orc_agg* a, int64_t* keys, uint8_t* key_valid, int64_t* values,
                    uint8_t* valid);
void orc_agg_free(orc_agg* a);
/* A new aggregation of one batch (WHERE `leaves`), its groups split over
 * `threads` by key hash; bit-identical to orc_agg_new + orc_agg_update. */
int32_t orc_aggregate_parallel(const orc_column* cols, int32_t ncols, const orc_agg_spec* spec,
                               const orc_leaf* leaves, int32_t nleaves, int32_t threads,
                               orc_agg** out);

/* ---- join + filter + grouped aggregation over one probe batch ----
 * Inner join probe.key = build.key; `leaves` filter the probe side; the
 * group key and each aggregate input name a side (0 probe, 1 build) and a
 * column.  Sequential in probe-row order, then build order. */
typedef struct orc_join_agg_query {
    int32_t probe_key;
    int32_t build_key;
    int32_t group_side;
    int32_t group_column;
    int32_t naggregates;
    int32_t funcs[ORC_MAX_AGGREGATES];
    int32_t sides[ORC_MAX_AGGREGATES];
    int32_t columns[ORC_MAX_AGGREGATES];
} orc_join_agg_query;
int32_t orc_join_aggregate(const orc_column* probe, int32_t nprobe_cols, const orc_column* build,
                           int32_t nbuild_cols, const orc_leaf* leaves, int32_t nleaves,
                           const orc_join_agg_query* q, int32_t threads, orc_agg** out);

/* ---- vectors ---- */
/* Distances per row (NaN-free rows get valid = 1; NULL rows valid = 0). */
int32_t orc_vector_distance(const orc_column* vec, const float* query, int32_t metric, float* out,
                            uint8_t* out_valid);
/* Top-k by (distance, row id) over rows passing `leaves` (evaluated over
 * `cols`) with a non-NULL vector; ids -1 / NaN pad when fewer rows pass. */
int32_t orc_vector_topk(const orc_column* cols, int32_t ncols, int32_t vec_column,
                        const orc_leaf* leaves, int32_t nleaves, const float* queries,
                        int32_t nqueries, int32_t k, int32_t metric, int32_t threads,
                        int64_t* out_ids, float* out_dist);

#ifdef __cplusplus
}
#endif
#endif
