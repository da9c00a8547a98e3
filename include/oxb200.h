/*
 * oxb200.h — C ABI of the B200 (sm_100a) GPU operator path of OxideLake.
 *
 * The entry points mirror, one to one, the object-safe `GpuBackend` trait of
 * the reference (crates/oxidelake-device/src/backend.rs:44-198) and its
 * argument bundles (crates/oxidelake-device/src/args.rs:10-86), so a Rust
 * `extern "C"` binding can implement the trait over this library without any
 * change to the `Gpu*Exec` plans above it.  Every signature uses plain C
 * types, pointers and sizes.
 *
 * Conventions (crates/oxidelake-device/src/columns.rs:28-40):
 *   - a column's values are tightly packed from row 0;
 *   - a validity bitmap is LSB-first, bit 0 = row 0, re-based to bit 0;
 *     a NULL validity pointer means "every row valid";
 *   - a FixedSizeList<Float32, dim> column stores dim floats per row.
 * Every call is synchronous towards the host unless it says otherwise (work
 * is ordered on the stream it is given); every call is thread-safe.  A call
 * that fails returns a status other than OXB_OK and leaves a message that
 * oxb_last_error() returns on the calling thread.  No entry point falls
 * back to the CPU: OXB_UNSUPPORTED is returned only for shapes outside
 * coverage, exactly where the reference's backend returns
 * EngineError::Unsupported (crates/oxidelake-core/src/error.rs:56-64).
 */
#ifndef OXB200_H
#define OXB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define OXB_API __attribute__((visibility("default")))
#else
#define OXB_API
#endif

#define OXB_ABI_VERSION 1

/* EngineError, crates/oxidelake-core/src/error.rs:17-73, plus the device-path
 * statuses the reference has no variant for. */
typedef enum oxb_status {
    OXB_OK = 0,
    OXB_UNSUPPORTED = 1,   /* EngineError::Unsupported: caller may take its CPU path */
    OXB_DEVICE = 2,        /* EngineError::Device: a CUDA call failed */
    OXB_EXECUTION = 3,     /* EngineError::Execution */
    OXB_PLAN = 4,          /* EngineError::Plan: bad column index, type, shape */
    OXB_ALLOCATION = 5,    /* EngineError::Allocation: device or pinned allocation failed */
    OXB_OOM_ADMISSION = 6, /* serving: a request's estimated memory exceeds the budget */
    OXB_TABLE_FULL = 7,    /* a device hash table ran out of slots */
    OXB_TIMEOUT = 8        /* a bounded device wait gave up */
} oxb_status;

/* Arrow types the path reads (crates/oxidelake-core/src/params.rs:170-182,
 * widened by Int32). */
typedef enum oxb_type {
    OXB_TYPE_INT64 = 1,
    OXB_TYPE_FLOAT64 = 2,
    OXB_TYPE_INT32 = 3,
    OXB_TYPE_FLOAT32 = 4,
    OXB_TYPE_VECTOR_F32 = 5 /* FixedSizeList<Float32, dim> */
} oxb_type;

/* Comparison, crates/oxidelake-core/src/params.rs:12-23. */
typedef enum oxb_cmp {
    OXB_CMP_EQ = 0,
    OXB_CMP_LT = 1,
    OXB_CMP_LTEQ = 2,
    OXB_CMP_GT = 3,
    OXB_CMP_GTEQ = 4
} oxb_cmp;

/* AggregateFunction, crates/oxidelake-core/src/params.rs:117-126, widened by
 * AVG and COUNT(*) (DataFusion semantics: AVG -> Float64, COUNT(*) counts rows). */
typedef enum oxb_agg_func {
    OXB_AGG_SUM = 0,
    OXB_AGG_COUNT = 1,
    OXB_AGG_MIN = 2,
    OXB_AGG_MAX = 3,
    OXB_AGG_AVG = 4,
    OXB_AGG_COUNT_STAR = 5
} oxb_agg_func;

/* DistanceMetric, crates/oxidelake-core/src/params.rs:151-156. */
typedef enum oxb_metric { OXB_METRIC_L2 = 0, OXB_METRIC_COSINE = 1 } oxb_metric;

/* One column, host- or device-resident (which one is said by the call). */
typedef struct oxb_column {
    int32_t type;            /* oxb_type */
    int32_t dim;             /* list size for OXB_TYPE_VECTOR_F32, else 1 */
    int64_t length;          /* rows */
    const void* values;      /* length * width bytes, width = 8, 4 or 4 * dim */
    const uint8_t* validity; /* ceil(length / 8) bytes, or NULL = all valid */
} oxb_column;

/* One comparison leaf of a predicate: `column <op> literal`.  A predicate is
 * the AND of its leaves (Predicate::And of Predicate::Compare,
 * crates/oxidelake-core/src/params.rs:60-72; a WHERE keeps a row only when
 * every leaf is true, so the AND-tree flattens exactly).  The literal type
 * must equal the column type, else the call returns OXB_UNSUPPORTED as the
 * reference's evaluate_predicate does (cpu/kernels.rs:110-119). */
typedef struct oxb_leaf {
    int32_t column;
    int32_t op;       /* oxb_cmp */
    int32_t lit_type; /* OXB_TYPE_INT64, OXB_TYPE_FLOAT64 or OXB_TYPE_INT32 */
    int32_t reserved;
    union {
        int64_t i;
        double f;
    } lit;
} oxb_leaf;

/* Most leaves one predicate may have (crates/oxidelake-compute/src/exec/mod.rs:31). */
#define OXB_MAX_PREDICATE_LEAVES 64
/* Most aggregates one grouped aggregation may compute. */
#define OXB_MAX_AGGREGATES 16

typedef struct oxb_backend oxb_backend;           /* CudaBackend: one device */
typedef struct oxb_stream oxb_stream;             /* DeviceStream */
typedef struct oxb_buffer oxb_buffer;             /* DeviceBuffer */
typedef struct oxb_host_buffer oxb_host_buffer;   /* HostBuffer */
typedef struct oxb_batch oxb_batch;               /* DeviceBatch */
typedef struct oxb_join_table oxb_join_table;     /* DeviceJoinTable */
typedef struct oxb_join_matches oxb_join_matches; /* DeviceJoinMatches */
typedef struct oxb_vector_index oxb_vector_index; /* resident BF16 copy for top-k */

/* MemoryInfo, crates/oxidelake-device/src/backend.rs:18-26. */
typedef struct oxb_memory_info {
    uint64_t total_bytes;
    uint64_t free_bytes;
    int32_t pinned_supported;
    int32_t reserved;
} oxb_memory_info;

/* ---- errors and version ------------------------------------------------ */

/* Message of the last failed call on this thread ("" when none). */
OXB_API const char* oxb_last_error(void);
OXB_API int32_t oxb_abi_version(void);

/* ---- backend lifecycle (HardwareDetector::select -> CudaBackend::new,
 *      crates/oxidelake-device/src/cuda/mod.rs:344) ---------------------- */

OXB_API oxb_status oxb_backend_create(int32_t device, oxb_backend** out);
OXB_API void oxb_backend_destroy(oxb_backend* backend);
/* GpuBackend::kind (backend.rs:46): "cuda". */
OXB_API const char* oxb_backend_kind(const oxb_backend* backend);
/* GpuBackend::device_id (backend.rs:49). */
OXB_API int32_t oxb_backend_device_id(const oxb_backend* backend);
/* GpuBackend::memory_info (backend.rs:52). */
OXB_API oxb_status oxb_memory_info_get(oxb_backend* backend, oxb_memory_info* out);

/* ---- memory (backend.rs:55-59) ---------------------------------------- */

/* GpuBackend::alloc_device: zeroed, 256-byte aligned (>= the 128 the
 * reference requires, crates/oxidelake-core/src/layout.rs:9). */
OXB_API oxb_status oxb_alloc_device(oxb_backend* backend, size_t bytes, oxb_buffer** out);
OXB_API void* oxb_buffer_device_ptr(const oxb_buffer* buffer);
OXB_API size_t oxb_buffer_len(const oxb_buffer* buffer);
OXB_API void oxb_buffer_free(oxb_buffer* buffer);
/* GpuBackend::alloc_pinned_host: page-locked when possible. */
OXB_API oxb_status oxb_alloc_pinned_host(oxb_backend* backend, size_t bytes, oxb_host_buffer** out);
OXB_API void* oxb_host_buffer_ptr(const oxb_host_buffer* buffer);
OXB_API size_t oxb_host_buffer_len(const oxb_host_buffer* buffer);
OXB_API int32_t oxb_host_buffer_is_pinned(const oxb_host_buffer* buffer);
OXB_API void oxb_host_buffer_free(oxb_host_buffer* buffer);

/* ---- streams and transfers (backend.rs:62-81) -------------------------- */

OXB_API oxb_status oxb_stream_create(oxb_backend* backend, oxb_stream** out);
/* Wraps a caller-owned cudaStream_t (not destroyed by oxb_stream_destroy). */
OXB_API oxb_status oxb_stream_wrap(oxb_backend* backend, void* cuda_stream, oxb_stream** out);
OXB_API void* oxb_stream_cuda_handle(const oxb_stream* stream);
OXB_API oxb_status oxb_stream_synchronize(oxb_backend* backend, oxb_stream* stream);
OXB_API void oxb_stream_destroy(oxb_stream* stream);
/* GpuBackend::copy_h2d / copy_d2h: whole buffers, min of the two lengths. */
OXB_API oxb_status oxb_copy_h2d(oxb_backend* backend, oxb_stream* stream, const oxb_host_buffer* src,
                        oxb_buffer* dst);
OXB_API oxb_status oxb_copy_d2h(oxb_backend* backend, oxb_stream* stream, const oxb_buffer* src,
                        oxb_host_buffer* dst);

/* ---- batches (backend.rs:84-95; handles.rs:130) ------------------------ */

/* GpuBackend::upload: copies `ncols` host columns of `rows` rows to the
 * device.  Queued on `stream`; the host buffers must stay alive until the
 * stream is synchronized (large pageable buffers are staged and released
 * earlier: oxb_set_upload_staging). */
OXB_API oxb_status oxb_upload(oxb_backend* backend, oxb_stream* stream, const oxb_column* columns,
                      int32_t ncols, int64_t rows, oxb_batch** out);
/* A batch over columns already in device memory (no copy; the caller keeps
 * the memory alive for the batch's lifetime). */
OXB_API oxb_status oxb_batch_from_device(oxb_backend* backend, const oxb_column* columns, int32_t ncols,
                                 int64_t rows, oxb_batch** out);
OXB_API int64_t oxb_batch_num_rows(const oxb_batch* batch);
OXB_API int32_t oxb_batch_num_columns(const oxb_batch* batch);
/* The device-side descriptor of column `index` (device pointers). */
OXB_API oxb_status oxb_batch_column(const oxb_batch* batch, int32_t index, oxb_column* out);
/* GpuBackend::download, column by column: copies column `index` into
 * caller-allocated host memory (values: length * width bytes; validity:
 * ceil(length / 8) bytes, written only when the column has a bitmap, which
 * *has_validity reports).  Synchronizes `stream`. */
OXB_API oxb_status oxb_download_column(oxb_backend* backend, oxb_stream* stream, const oxb_batch* batch,
                               int32_t index, void* values, uint8_t* validity,
                               int32_t* has_validity);
/* GpuBackend::download (backend.rs:91-95), the whole batch in one call:
 * column i into values[i] (length * width bytes) and, when it has a bitmap
 * (has_validity[i] = 1), validity[i] (ceil(length / 8) bytes; may be NULL
 * for a column without one).  The copies are queued together and the stream
 * is synchronized once, at the end.  ncols must equal the batch's. */
OXB_API oxb_status oxb_download(oxb_backend* backend, oxb_stream* stream, const oxb_batch* batch, int32_t ncols,
                                void* const* values, uint8_t* const* validity, int32_t* has_validity);
OXB_API void oxb_batch_free(oxb_batch* batch);

/* ---- Arrow C data interface (columns.rs:192-289 hands the backend the
 * same buffers) ------------------------------------------------------------
 * The structs are the Arrow project's stable C ABI ("The Arrow C data
 * interface"), declared under its own include guard so a program that also
 * includes Arrow's abi.h sees one definition. */
#ifndef ARROW_C_DATA_INTERFACE
#define ARROW_C_DATA_INTERFACE
#define ARROW_FLAG_DICTIONARY_ORDERED 1
#define ARROW_FLAG_NULLABLE 2
#define ARROW_FLAG_MAP_KEYS_SORTED 4
struct ArrowSchema {
    const char* format;
    const char* name;
    const char* metadata;
    int64_t flags;
    int64_t n_children;
    struct ArrowSchema** children;
    struct ArrowSchema* dictionary;
    void (*release)(struct ArrowSchema*);
    void* private_data;
};
struct ArrowArray {
    int64_t length;
    int64_t null_count;
    int64_t offset;
    int64_t n_buffers;
    int64_t n_children;
    const void** buffers;
    struct ArrowArray** children;
    struct ArrowArray* dictionary;
    void (*release)(struct ArrowArray*);
    void* private_data;
};
#endif

/* GpuBackend::upload of a RecordBatch exported through the Arrow C data
 * interface: a struct array ("+s") whose children are Int64 ("l"), Int32
 * ("i"), Float64 ("g"), Float32 ("f") or FixedSizeList<Float32, dim>
 * ("+w:dim" over "f", no nulls inside the lists).  Array and child offsets
 * are honoured (a validity bitmap at an odd bit offset is re-based on the
 * host).  The copies finish before the call returns; then `array` and
 * `schema` are released.  On an error neither is released (the caller
 * still owns them, e.g. to take its CPU path after OXB_UNSUPPORTED). */
OXB_API oxb_status oxb_import_arrow(oxb_backend* backend, oxb_stream* stream, struct ArrowArray* array,
                                    struct ArrowSchema* schema, oxb_batch** out);
/* GpuBackend::download into a RecordBatch exported through the Arrow C data
 * interface: `out_array` and `out_schema` (caller-provided structs, filled
 * here) describe a struct array whose children are the batch's columns,
 * named names[i] (or "c<i>" when `names` is NULL), in host memory this call
 * allocates.  The consumer releases them with their release callbacks.
 * Synchronizes `stream`. */
OXB_API oxb_status oxb_export_arrow(oxb_backend* backend, oxb_stream* stream, const oxb_batch* batch,
                                    const char* const* names, struct ArrowArray* out_array,
                                    struct ArrowSchema* out_schema);

/* ---- operators --------------------------------------------------------- */

/* FilterProjectArgs, args.rs:10-15 -> GpuBackend::filter_project
 * (backend.rs:98).  Rows where every leaf is true, projected columns in
 * projection order, row order kept. */
typedef struct oxb_filter_project_args {
    const oxb_batch* input;
    const oxb_leaf* leaves;
    int32_t nleaves;
    const int32_t* projection;
    int32_t nprojection;
} oxb_filter_project_args;
OXB_API oxb_status oxb_filter_project(oxb_backend* backend, oxb_stream* stream,
                              const oxb_filter_project_args* args, oxb_batch** out);

/* No counterpart in the reference: oxb_filter_project that allocates
 * nothing, neither device nor pinned memory.
 *
 * Why: some callers must not allocate per call.  An executor that admitted
 * a query against a fixed device-memory budget and reserved its output
 * buffers up front cannot let an operator take more memory in the middle of
 * the pipeline, where the allocation could fail or push the device past the
 * budget the admission promised; and a caller that manages its own buffer
 * pool wants the call's footprint known before the call, not drawn from the
 * stream-ordered pool behind its back.
 *
 * Output: projected column i goes to out_values[i] (device memory, room for
 * `capacity` rows of that column's width, 8-byte aligned for 8-byte and
 * wider rows, else 4-byte) and, when the source column has a validity
 * bitmap, to out_validity[i] (device memory, ceil(capacity / 32) 32-bit
 * words, LSB-first; this call clears the words it uses).  *out_rows receives
 * the selected row count; when it exceeds `capacity` the call writes no
 * output and returns OXB_EXECUTION, with *out_rows still set.
 *
 * Limit: at most OXB_NOALLOC_MAX_ROWS input rows (OXB_UNSUPPORTED beyond).
 * The mask, tile counts, tile offsets and scan partials live in one static
 * device array of about 2.2 MiB per device.  The first call on each device
 * looks that array's address up with cudaGetSymbolAddress (which can load
 * the module); make that first call before any stream capture begins.
 * Calls whose work overlaps on one device (other streams, other threads)
 * race on that array: the caller serialises them.  The call synchronizes
 * `stream` once (to read the selected count) and returns with the gather
 * still queued on it. */
#define OXB_NOALLOC_MAX_ROWS (1 << 24)
OXB_API oxb_status oxb_filter_project_noalloc(oxb_backend* backend, oxb_stream* stream,
                                              const oxb_filter_project_args* args, void* const* out_values,
                                              uint32_t* const* out_validity, int64_t capacity,
                                              int64_t* out_rows);

/* The host's index of a build side (cpu::kernels::JoinTable::runs and
 * row_indices, cpu/kernels.rs:245-255): `ndistinct` runs (key, start,
 * count) into `rows`, which groups the build rows with a non-NULL key by
 * key, in build order.  JoinBuildArgs::index (args.rs:21-30). */
typedef struct oxb_join_index {
    const int64_t* keys;
    const uint32_t* starts;
    const uint32_t* counts;
    int64_t ndistinct;
    const uint32_t* rows;
    int64_t nrows;
} oxb_join_index;

/* JoinBuildArgs -> GpuBackend::prepare_join_build (backend.rs:129).  With
 * `index` NULL the device builds the same index itself from the key column
 * (a stable sort by key keeps build order within a key). */
typedef struct oxb_join_build_args {
    const oxb_batch* build;
    int32_t key;
    int32_t reserved;
    const oxb_join_index* index;
} oxb_join_build_args;
OXB_API oxb_status oxb_prepare_join_build(oxb_backend* backend, oxb_stream* stream,
                                  const oxb_join_build_args* args, oxb_join_table** out);
OXB_API int64_t oxb_join_table_distinct_keys(const oxb_join_table* table);
OXB_API int64_t oxb_join_table_rows(const oxb_join_table* table);
OXB_API void oxb_join_table_free(oxb_join_table* table);

/* JoinProbeArgs -> GpuBackend::probe_join (backend.rs:153).  Matches are
 * numbered in probe-row order, then build order (backend.rs:148-152). */
typedef struct oxb_join_probe_args {
    const oxb_batch* probe;
    int32_t key;
    int32_t reserved;
    const oxb_join_table* table;
} oxb_join_probe_args;
OXB_API oxb_status oxb_probe_join(oxb_backend* backend, oxb_stream* stream,
                          const oxb_join_probe_args* args, oxb_join_matches** out);
OXB_API uint64_t oxb_join_matches_len(const oxb_join_matches* matches);
OXB_API int64_t oxb_join_matches_probe_rows(const oxb_join_matches* matches);
OXB_API void oxb_join_matches_free(oxb_join_matches* matches);

/* HashJoinArgs -> GpuBackend::hash_join (backend.rs:114): matches
 * first..first+rows as left columns ++ right columns, or the `projection`
 * subset of that concatenation (NULL = all). */
typedef struct oxb_hash_join_args {
    const oxb_batch* left;
    const oxb_batch* right;
    const oxb_join_table* table;
    const oxb_join_matches* matches;
    uint64_t first;
    uint64_t rows;
    const int32_t* projection;
    int32_t nprojection;
    int32_t reserved;
} oxb_hash_join_args;
OXB_API oxb_status oxb_hash_join(oxb_backend* backend, oxb_stream* stream,
                         const oxb_hash_join_args* args, oxb_batch** out);

/* AggregateSpec, params.rs:142-147 -> AggregateArgs, args.rs:64-69 ->
 * GpuBackend::aggregate (backend.rs:166).  Output: the key (nullable Int64
 * or Int32, as the key column) then one column per aggregate, groups sorted
 * by key with the NULL group last (crates/oxidelake-device/src/cuda/ops.rs:1037;
 * cpu/kernels.rs:793-811).  Types: SUM(Int64|Int32) -> Int64 (wrapping),
 * SUM(Float64) -> Float64, COUNT/COUNT(*) -> Int64, MIN/MAX keep the input
 * type, AVG -> Float64.  For OXB_AGG_COUNT_STAR the column is ignored. */
typedef struct oxb_aggregate_spec {
    int32_t group_by;
    int32_t naggregates;
    int32_t funcs[OXB_MAX_AGGREGATES];   /* oxb_agg_func */
    int32_t columns[OXB_MAX_AGGREGATES];
} oxb_aggregate_spec;
typedef struct oxb_aggregate_args {
    const oxb_batch* input;
    const oxb_aggregate_spec* spec;
    /* Optional fused WHERE over `input` (NULL/0 = every row). */
    const oxb_leaf* leaves;
    int32_t nleaves;
    int32_t reserved;
} oxb_aggregate_args;
OXB_API oxb_status oxb_aggregate(oxb_backend* backend, oxb_stream* stream,
                         const oxb_aggregate_args* args, oxb_batch** out);

/* Every RecordBatch of one GpuAggregateExec input partition folded into one
 * result (compute/src/exec/aggregate.rs:35-321 emits one batch at the end
 * of the stream; the reference merges per-batch device partials on the host,
 * operator.rs:994-1075).  The batches share a schema and may differ in row
 * count; one persistent launch takes their rows from one work queue into
 * one table sized by a distinct-count estimate of the keys.  Same output as
 * oxb_aggregate over the batches' concatenation. */
typedef struct oxb_aggregate_batches_args {
    const oxb_batch* const* inputs;
    int32_t ninputs;
    int32_t reserved;
    const oxb_aggregate_spec* spec;
    const oxb_leaf* leaves; /* WHERE over each batch, NULL/0 = every row */
    int32_t nleaves;
    int32_t reserved2;
} oxb_aggregate_batches_args;
OXB_API oxb_status oxb_aggregate_batches(oxb_backend* backend, oxb_stream* stream,
                                         const oxb_aggregate_batches_args* args, oxb_batch** out);

/* ORDER BY l2|cosine(vector, query) LIMIT k over the rows a WHERE keeps, for
 * a batch of queries: the reference's GpuVectorDistanceExec followed by its
 * CPU SortExec(fetch = k) (compute/src/exec/vector.rs:29-249,
 * cpu/kernels.rs:841-927), fused.  Rows with a NULL vector are left out; the
 * order is (distance in IEEE totalOrder, row id); when fewer than k rows
 * qualify, the rest of the row is id -1 and distance NaN.  Returned
 * distances are the reference's FP32 values bit for bit.
 *
 * oxb_vector_index_build keeps a BF16 copy of the vector column (and each
 * row's norm) resident for the tensor-core scan; the index refers to the
 * batch's FP32 vectors, so the batch outlives it.  Up to 2^32 - 1 rows. */
OXB_API oxb_status oxb_vector_index_build(oxb_backend* backend, oxb_stream* stream, const oxb_batch* input,
                                          int32_t column, oxb_vector_index** out);
OXB_API void oxb_vector_index_free(oxb_vector_index* index);

typedef struct oxb_vector_topk_args {
    const oxb_vector_index* index;
    const oxb_batch* input;  /* the batch the index was built over (WHERE columns) */
    const oxb_leaf* leaves;  /* WHERE over `input`, NULL/0 = every row */
    int32_t nleaves;
    int32_t nqueries;
    const float* queries;    /* host, nqueries x dim FP32 */
    int32_t dim;
    int32_t k;               /* 1..4096 */
    int32_t metric;          /* oxb_metric */
    int32_t overfetch;       /* re-ranked candidates per query = overfetch * k (0: 4) */
    int32_t exact;           /* 1: skip the BF16 scan, the exact FP32 path for every query */
    /* A leaf each query has with its own literal, so queries whose WHERE
     * differs share one scan: query q also needs
     * `qleaf_column <qleaf_op> qleaf_lits[q]` (qleaf_column -1: none). */
    int32_t qleaf_column;
    int32_t qleaf_op;        /* oxb_cmp */
    int32_t qleaf_type;      /* the column's oxb_type: INT64, INT32 or FLOAT64 */
    int32_t reserved;
    const int64_t* qleaf_lits; /* host, nqueries literals (a Float64 one as its bit pattern) */
} oxb_vector_topk_args;

typedef struct oxb_vector_topk_stats {
    int64_t reranked;          /* candidates re-ranked in FP32 */
    int64_t exact_queries;     /* queries the exact path answered */
    double max_score_error;    /* largest |BF16 score - FP64 score| among re-ranked candidates */
    double mean_score_error;
} oxb_vector_topk_stats;

/* out_ids: nqueries x k int64 (host), out_dist: nqueries x k float (host);
 * stats may be NULL.  Synchronizes `stream`. */
OXB_API oxb_status oxb_vector_topk(oxb_backend* backend, oxb_stream* stream, const oxb_vector_topk_args* args,
                                   int64_t* out_ids, float* out_dist, oxb_vector_topk_stats* stats);

/* VectorDistanceArgs, args.rs:72-84 -> GpuBackend::vector_distance
 * (backend.rs:173): the input columns plus a Float32 distance column with
 * the vector column's validity.  Distances follow cpu/kernels.rs:909-927
 * bit for bit (Float32, summed in index order). */
typedef struct oxb_vector_distance_args {
    const oxb_batch* input;
    int32_t column;
    int32_t metric; /* oxb_metric */
    const float* query; /* host pointer, dim floats */
    int32_t dim;
    int32_t reserved;
} oxb_vector_distance_args;
OXB_API oxb_status oxb_vector_distance(oxb_backend* backend, oxb_stream* stream,
                               const oxb_vector_distance_args* args, oxb_batch** out);

/* ---- new forms beside the drop-in path --------------------------------- */

/* One pass of `probe JOIN build ON probe.key = build.key WHERE <leaves on
 * probe columns> GROUP BY <one column of either side>` computing the listed
 * aggregates, over a join table prepared on `build`.  It has no counterpart
 * in the reference, where this query runs as GpuHashJoinExec (probe_join +
 * hash_join chunks, backend.rs:114-163) followed by an aggregate over the
 * joined rows (cpu/kernels.rs:679-811); the output equals that plan's:
 * groups sorted by key, NULL last, types as oxb_aggregate.  Sides: 0 =
 * probe, 1 = build. */
typedef struct oxb_join_aggregate_args {
    const oxb_batch* probe;
    int32_t probe_key;
    int32_t reserved;
    const oxb_join_table* table;
    const oxb_batch* build;
    const oxb_leaf* leaves;
    int32_t nleaves;
    int32_t group_side;
    int32_t group_column;
    int32_t naggregates;
    int32_t funcs[OXB_MAX_AGGREGATES];
    int32_t sides[OXB_MAX_AGGREGATES];
    int32_t columns[OXB_MAX_AGGREGATES];
} oxb_join_aggregate_args;
OXB_API oxb_status oxb_join_aggregate(oxb_backend* backend, oxb_stream* stream,
                              const oxb_join_aggregate_args* args, oxb_batch** out);
/* Several oxb_join_aggregate requests in one launch, where they differ only
 * in their probe batch (columns of the same types) and their WHERE literals:
 * the rows of every request are tiles of one work queue, and each request
 * folds into its own table.  out[i] is the result of args[i], equal to its
 * own oxb_join_aggregate call's; requests that cannot share the launch
 * (another shape, a column with a validity bitmap, more than two inputs)
 * run one at a time.  No reference counterpart: the reference runs one query
 * at a time (compute/src/operator.rs). */
OXB_API oxb_status oxb_join_aggregate_many(oxb_backend* backend, oxb_stream* stream,
                                           const oxb_join_aggregate_args* args, int32_t n, oxb_batch** out);

/* ---- serving (the request loop the reference lacks; its queries run one at
 *      a time through compute/src/operator.rs) ---------------------------- */

/* A request loop over resident tables: submit returns a ticket at once;
 * worker threads (one CUDA stream each) run admitted work concurrently, and
 * top-k requests that queue while others run are stacked into one scan when
 * they share the index, batch, metric and WHERE except for their own query
 * vector, k and per-query literal; join-aggregate requests of one shape
 * (oxb_join_aggregate_many) share one launch the same way.  Work is admitted while the estimated
 * device memory of what runs stays within the budget; a request that alone
 * exceeds it is refused with OXB_OOM_ADMISSION.  Results equal the direct
 * calls'.  The resident batches, indexes and join tables outlive the server. */
typedef struct oxb_server oxb_server;
typedef struct oxb_server_config {
    uint64_t memory_budget; /* bytes (0: 150 GB) */
    int32_t workers;        /* concurrent work items (0: 2) */
    int32_t max_batch;      /* queries stacked into one top-k scan (0: 256; 1: no batching) */
} oxb_server_config;
OXB_API oxb_status oxb_server_create(oxb_backend* backend, const oxb_server_config* config, oxb_server** out);
/* Finishes the submitted work, then stops the workers. */
OXB_API void oxb_server_destroy(oxb_server* server);

typedef struct oxb_topk_request {
    const oxb_vector_index* index;
    const oxb_batch* input;
    const oxb_leaf* leaves; /* the WHERE */
    int32_t nleaves;
    int32_t qleaf;          /* 1: leaves[nleaves - 1] is this query's own literal (see oxb_vector_topk) */
    const float* query;     /* dim floats, copied at submit */
    int32_t dim;
    int32_t k;
    int32_t metric;
    int32_t reserved;
} oxb_topk_request;
OXB_API oxb_status oxb_server_submit_topk(oxb_server* server, const oxb_topk_request* request, uint64_t* ticket);
/* The arguments (and leaves) are copied at submit. */
OXB_API oxb_status oxb_server_submit_join_aggregate(oxb_server* server, const oxb_join_aggregate_args* request,
                                                    uint64_t* ticket);
/* Blocks until the request is done.  Top-k: k ids and distances into
 * caller buffers; join-aggregate: the result batch.  latency_us (may be
 * NULL): submit to completion. */
OXB_API oxb_status oxb_server_wait_topk(oxb_server* server, uint64_t ticket, int64_t* ids, float* dist,
                                        double* latency_us);
OXB_API oxb_status oxb_server_wait_batch(oxb_server* server, uint64_t ticket, oxb_batch** out, double* latency_us);

typedef struct oxb_server_stats {
    int64_t completed;
    int64_t rejected;
    int64_t dispatches;      /* work items run */
    int64_t batched_queries; /* requests that shared a launch: top-k scans, join-aggregate folds */
    int64_t peak_bytes;      /* largest admitted estimate in flight */
    double p50_us, p99_us;   /* submit-to-result latency */
    double qps;              /* completed / (last completion - first submit) */
} oxb_server_stats;
/* reset: 1 starts a new measurement window. */
OXB_API oxb_status oxb_server_stats_get(oxb_server* server, oxb_server_stats* out, int32_t reset);

/* ---- instrumentation (no counterpart in the reference) ------------------ */

/* When enabled, each operator records CUDA events on its stream around its
 * main kernel; oxb_last_kernel_time returns that kernel's name and duration
 * for the last operator call on this thread. */
OXB_API oxb_status oxb_set_kernel_timing(oxb_backend* backend, int32_t enabled);
OXB_API oxb_status oxb_last_kernel_time(oxb_backend* backend, char* name, int32_t name_len,
                                        float* ms);
/* Kernels this library has launched in this process. */
OXB_API uint64_t oxb_kernel_launches(void);
/* Ingest of pageable host memory by oxb_upload, and oxb_download_column into
 * pageable memory: a column buffer of at least
 * 4 MiB that is not page-locked is copied by `threads` host threads (the
 * calling thread included) into a ring of four page-locked 8 MiB chunks, and
 * each chunk's host-to-device copy overlaps the filling of the next (a
 * download drains one chunk while the next ones are copied).  Such a
 * buffer is no longer read when oxb_upload returns.  0 = off: the driver
 * copies pageable memory itself.  Default: half the host's cores, at most
 * 8; the setter takes at most 32.  The ring (32 MiB
 * page-locked) is allocated on the first staged copy. */
OXB_API oxb_status oxb_set_upload_staging(oxb_backend* backend, int32_t threads);
/* When enabled, the first call of each query shape times every compiled
 * variant of its main kernel (warp combining on/off, rows per thread) on
 * that call's data and keeps the fastest for later calls in this process. */
OXB_API oxb_status oxb_set_autotune(oxb_backend* backend, int32_t enabled);
/* Pins the aggregation kernels' variant instead of the tuned one: combine
 * -1 (automatic), 0 (per-row atomics), 1 (warp combining and caches), 2
 * (tile sort-reduce), 3 (columns streamed by bulk copies), 4 (streamed
 * tile sort-reduce), 5 (join-aggregate only: the fused probe table, for a
 * build-side group key with a small span; its dense form when the build
 * keys fill at least a quarter of their range), 6 (the fused probe table,
 * hashed form), 7 or 8 (5 or 6 interpreted a vector of rows per thread at
 * a time), 9 or 10 (oxb_aggregate_batches only: the hash-partitioned
 * passes with the planned partitions, or with their fewest; there 0..8 pin
 * the single persistent kernel), 11 or 12 (join-aggregate only: 5 or 6 with
 * the probe columns streamed into shared memory by bulk copies), 13 or 14
 * (join-aggregate only: 5 or 6 compiled for the accumulator shape, when the
 * inputs are at most two sums and no column has a validity bitmap), 15 or
 * 16 (13 or 14 reading each column two rows per vector load, when every
 * column starts on a 16-byte boundary; otherwise 13 or 14), 17
 * (oxb_aggregate_batches only: the dense-range passes, partitioned by the
 * key's offset in the sampled key range, when every aggregate is COUNT,
 * SUM, MIN or MAX of one Int32 column and the range holds at most 2^25
 * keys; otherwise the single persistent kernel);
 * rows_per_thread 0 (automatic), 1, 2, 4 or 8 (the row loops take
 * 1 or 2, the fused kernels 2 or 4, the compiled ones 1, 2 or 4, the vector
 * ones 4 or 8; other values round to the nearest the kernel has). */
OXB_API oxb_status oxb_set_agg_variant(oxb_backend* backend, int32_t combine, int32_t rows_per_thread);

/* ---- telemetry: the counters of OperatorStats
 *      (crates/oxidelake-core/src/telemetry.rs:38-66, 99-190) ------------- */

/* The operator a call counts under.  Uploads and downloads count as
 * transfers; the fused join-aggregate and the many-batch fold count as
 * aggregates; top-k and vector distance as vector. */
typedef enum oxb_operator {
    OXB_OP_TRANSFER = 0,
    OXB_OP_FILTER = 1,
    OXB_OP_JOIN = 2,
    OXB_OP_AGGREGATE = 3,
    OXB_OP_VECTOR = 4,
    OXB_OP_COUNT = 5
} oxb_operator;

/* One call, as OperatorStats::record_batch / record_transfer take it
 * (telemetry.rs:140-152): rows in and out (for an aggregate the groups it
 * emits; for a top-k the queries x k it returns), host wall time of the
 * call, bytes the call itself moved between host and device memory.
 * batches: the input batches the call consumed (oxb_aggregate_batches: its
 * batch count; otherwise 1).  device_ns: the main kernel's CUDA-event time
 * when oxb_set_kernel_timing is on, else 0.  status: the call's return. */
typedef struct oxb_call_stats {
    int32_t op;        /* oxb_operator */
    int32_t status;    /* oxb_status */
    uint64_t batches;
    uint64_t rows_in;
    uint64_t rows_out;
    uint64_t elapsed_ns;
    uint64_t device_ns;
    uint64_t bytes_h2d;
    uint64_t bytes_d2h;
} oxb_call_stats;
/* The last operator or transfer call made on the calling thread.  Replaces
 * the Rust-side measurement around a trait call in GpuOperator::record_rows
 * (crates/oxidelake-compute/src/operator.rs:508-520). */
OXB_API oxb_status oxb_last_call_stats(oxb_call_stats* out);

/* A backend's totals per operator since it was created (or last reset):
 * the sums of its calls' counters, plus
 *   unsupported       calls that returned OXB_UNSUPPORTED (where the
 *                     reference's operator takes its CPU path and counts a
 *                     fallback, operator.rs:573-586);
 *   failed            calls that returned another error;
 *   fallback_batches  batches this library ran on the CPU: always 0, it has
 *                     no CPU path (record_fallback, telemetry.rs:162-175). */
typedef struct oxb_operator_stats {
    uint64_t calls;
    uint64_t batches;
    uint64_t rows_in;
    uint64_t rows_out;
    uint64_t elapsed_ns;
    uint64_t device_ns;
    uint64_t bytes_h2d;
    uint64_t bytes_d2h;
    uint64_t unsupported;
    uint64_t failed;
    uint64_t fallback_batches;
} oxb_operator_stats;
/* reset: 1 zeroes this operator's totals after reading them. */
OXB_API oxb_status oxb_operator_stats_get(oxb_backend* backend, int32_t op, oxb_operator_stats* out,
                                          int32_t reset);

/* GpuBackend::supports_predicate / supports_hash_join / supports_aggregate
 * (backend.rs:182-197): 1 when the call runs on the device. */
OXB_API int32_t oxb_supports_predicate(const oxb_backend* backend, const oxb_leaf* leaves,
                               int32_t nleaves);
OXB_API int32_t oxb_supports_hash_join(const oxb_backend* backend);
OXB_API int32_t oxb_supports_aggregate(const oxb_backend* backend);

#ifdef __cplusplus
}
#endif

#endif /* OXB200_H */
