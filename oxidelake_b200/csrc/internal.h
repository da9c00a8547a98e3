// Host-side runtime of liboxb200: handles behind the C ABI, the device
// allocator, per-call error state and the operator entry points the ABI
// layer (api.cu) dispatches to.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <atomic>
#include <cstring>
#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/oxb200.h"
#include "common.cuh"

namespace oxb {

// ---- errors ---------------------------------------------------------------

// A failed call: the status the ABI returns and the message oxb_last_error
// reports.  Operators throw it; the ABI layer catches it at the boundary,
// so no C++ exception ever crosses into the caller.
struct Error {
    oxb_status status;
    std::string message;
};

[[noreturn]] void fail(oxb_status status, const std::string& message);
void check_cuda(cudaError_t err, const char* what);
#define OXB_CUDA(call) ::oxb::check_cuda((call), #call)

// ---- streams and memory -------------------------------------------------

struct StreamState {
    cudaStream_t stream = nullptr;
    bool owned = false;
    int device = 0;
    ~StreamState();
};
using StreamRef = std::shared_ptr<StreamState>;

// One device allocation from the stream-ordered pool, freed on the stream
// it was allocated on once the last reference goes away.
struct DevAlloc {
    void* ptr = nullptr;
    size_t bytes = 0;
    StreamRef stream;
    ~DevAlloc();
};
using AllocRef = std::shared_ptr<DevAlloc>;

AllocRef dev_alloc(const StreamRef& s, size_t bytes, bool zero);

// Scratch memory that lives for one call, on that call's stream.
template <typename T>
struct Scratch {
    AllocRef a;
    T* ptr = nullptr;
    Scratch() = default;
    Scratch(const StreamRef& s, size_t n, bool zero = false) {
        a = dev_alloc(s, n * sizeof(T) + 16, zero);
        ptr = (T*)a->ptr;
    }
    T* get() const { return ptr; }
};

class Stager;  // page-locked staging ring for pageable uploads (ingest.cu)

struct Backend {
    int device = 0;
    int sms = 148;
    size_t smem_optin = 0;
    std::string name;
    bool timing = false;    // oxb_set_kernel_timing
    bool autotune = false;  // oxb_set_autotune
    int force_combine = -1;  // oxb_set_agg_variant: -1 = tuned/default
    int force_rpt = 0;
    int stage_threads = 8;            // oxb_set_upload_staging: 0 = off
    std::shared_ptr<Stager> stager;   // made on the first staged upload
    std::shared_ptr<struct SmallDownloads> small_dl;  // made on the first gathered download
};

// Queues the copy of n host bytes to device memory on s.  A large pageable
// source goes through the backend's page-locked staging ring (and is no
// longer read on return); any other source is one cudaMemcpyAsync.
void upload_bytes(Backend& b, const StreamRef& s, void* dst, const void* src, size_t n);
// The way back: a large pageable `dst` is filled through the same ring and
// holds every byte on return; any other `dst` is one queued cudaMemcpyAsync.
void download_bytes(Backend& b, const StreamRef& s, void* dst, const void* src, size_t n);
// Copies every piece (device src -> host dst, n bytes) and returns once all
// are in host memory (one stream synchronization).  Small pageable pieces
// go through one page-locked buffer of the backend, so their copies queue
// without waiting on each other; large ones through download_bytes.
struct DownloadPiece {
    void* dst;
    const void* src;
    size_t n;
};
void download_pieces(Backend& b, const StreamRef& s, const std::vector<DownloadPiece>& pieces);
void set_upload_staging(Backend& b, int threads);

// Counts every kernel this library launches (oxb_kernel_launches).
void note_launch();

// Times an operator's main kernel with CUDA events recorded on the stream it
// is launched on, when timing is switched on; the elapsed time is read after
// the stop event completes and kept for oxb_last_kernel_time on this thread.
class KernelTimer {
  public:
    KernelTimer(const Backend& b, const StreamRef& s, const char* name);
    ~KernelTimer();
    // Each begin()/end() pair is one timed segment; the recorded time is
    // the sum of the segments (host work between them is not counted).
    void begin();
    void end();
    void rename(const char* name) { name_ = name; }

  private:
    bool on_;
    const char* name_;
    cudaStream_t stream_;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> segs_;
    bool ended_ = false;
};

// ---- batches ----------------------------------------------------------------

struct Column {
    int type = 0;
    int dim = 1;
    long long length = 0;
    void* values = nullptr;
    uint8_t* validity = nullptr;
    AllocRef owner_values;    // null when the memory belongs to the caller
    AllocRef owner_validity;  // ditto
    int width() const { return type_width(type, dim); }
};

}  // namespace oxb

namespace oxb {
// Per-operator totals of a backend (oxb_operator_stats), one atomic word per
// field, added to by every call that names the backend.
struct Telemetry {
    static constexpr int kFields = 11;
    std::atomic<uint64_t> v[OXB_OP_COUNT][kFields];
    Telemetry() {
        for (auto& op : v)
            for (auto& f : op) f.store(0, std::memory_order_relaxed);
    }
};
}  // namespace oxb

struct oxb_backend {
    oxb::Backend b;
    oxb::Telemetry tel;
};
struct oxb_stream {
    oxb::StreamRef s;
};
struct oxb_buffer {
    oxb::AllocRef a;
};
struct oxb_host_buffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    bool pinned = false;
};
struct oxb_batch {
    long long rows = 0;
    std::vector<oxb::Column> cols;
};

namespace oxb {

// The build side of a hash join as the device probes it: an open-addressing
// table of one slot per distinct key (key, start, count) into `rows`, the
// build rows with a non-NULL key grouped by key, in build order.
struct JoinSlot {
    long long key;
    unsigned int start;
    unsigned int count;
};
struct JoinTableDev {
    JoinSlot* slots = nullptr;  // capacity slots
    unsigned int capacity = 0;  // power of two
    // rows[start] of each slot's run, beside the slots: indexed by the same
    // slot number, so a probe loads it in parallel with the slot and a
    // unique key needs no second dependent load to find its build row.
    unsigned int* first_row = nullptr;  // capacity + 1 entries
    unsigned int* rows = nullptr;
    long long nrows = 0;
    long long ndistinct = 0;
    // The run of the key equal to kEmptyKey, which cannot live in a slot.
    unsigned int special_start = 0;
    unsigned int special_count = 0;
    int key_type = kInt64;
    // Smallest and largest key placed in the slots (key_lo > key_hi: none).
    long long key_lo = 0;
    long long key_hi = -1;
    // Unique keys that fill their range (the dense build): the run start of
    // key dense_lo + d at dense[d], or kNoRun for a key the build lacks;
    // null otherwise.  A probe then reads 4 bytes instead of a 16-byte slot.
    const unsigned int* dense = nullptr;
    long long dense_lo = 0;
    unsigned long long dense_n = 0;
};
constexpr unsigned int kNoRun = 0xffffffffu;

}  // namespace oxb

// A vector column prepared for the tensor-core top-k scan (topk.cu).
struct oxb_vector_index {
    oxb::Column vec;  // the FP32 vectors (shares the batch's memory)
    long long n = 0;
    int dim = 0;
    int dp = 0;  // dim rounded up to 64
    oxb::AllocRef bf16, norm2, inv;
    float xmax = 0.0f;  // largest row norm
    CUtensorMap xmap;
};

struct oxb_join_table {
    oxb::JoinTableDev t;
    oxb::AllocRef slots_mem, rows_mem, dense_mem;
    const oxb_batch* build = nullptr;
    long long build_rows = 0;
};

struct oxb_join_matches {
    oxb::AllocRef offsets_mem;  // u64, probe_rows + 1
    oxb::AllocRef starts_mem;   // u32, probe_rows
    long long probe_rows = 0;
    unsigned long long total = 0;
    const oxb_join_table* table = nullptr;
};

namespace oxb {

// ---- helpers shared by the operators --------------------------------------

// The dynamic shared memory `kernel` may use on the current device: the
// device's opt-in maximum less the kernel's static shared memory.  The
// function's limit is raised to it on the first call for a kernel and device
// (under a lock, so no launch of that kernel precedes it) and never set to
// one call's size: host threads launching the same kernel with different
// sizes at once (the serving loop's workers) would otherwise lower it
// between another thread's setting and its launch, which then fails with
// "invalid argument".
int allow_smem_cap(const void* kernel);

template <typename K>
void allow_smem(K kernel, size_t smem) {
    if (smem <= 48 * 1024) return;
    const int cap = allow_smem_cap((const void*)kernel);
    if (smem > (size_t)cap)
        fail(OXB_UNSUPPORTED, std::to_string(smem) + " bytes of dynamic shared memory exceed the " +
                                  std::to_string(cap) + " the device leaves this kernel");
}

inline int grid_for(const Backend& b, long long work, int threads, int per_sm = 4) {
    long long blocks = (work + threads - 1) / threads;
    long long cap = (long long)b.sms * per_sm;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    return (int)blocks;
}

DevPredicate make_predicate(const oxb_batch& in, const oxb_leaf* leaves, int nleaves);

// ---- the Arrow C data interface (arrow_c.cu) ---------------------------------
// Host column descriptors over an exported struct array's buffers (bitmaps
// at an odd bit offset re-based into `rebased`).
struct ArrowImport {
    std::vector<oxb_column> cols;
    std::vector<std::vector<uint8_t>> rebased;
};
ArrowImport arrow_import_columns(const ArrowArray* array, const ArrowSchema* schema);
// A device batch copied to host memory and described as a struct array.
void arrow_export_batch(Backend& b, const StreamRef& s, const oxb_batch& batch, const char* const* names,
                        ArrowArray* out_array, ArrowSchema* out_schema, oxb_call_stats& st);
void check_status_word(uint32_t status, const char* what);

// Exclusive scan of n u32 counts into n + 1 u64 offsets (offsets[n] = total).
void scan_u32_to_u64(const StreamRef& s, const Backend& b, const unsigned int* counts,
                     unsigned long long* offsets, long long n);
// The same scan with its block partials in caller memory
// (scan_partials_needed(n) entries): it allocates nothing.
long long scan_partials_needed(long long n);
void scan_u32_to_u64_into(const StreamRef& s, const unsigned int* counts, unsigned long long* offsets, long long n,
                          unsigned long long* partials);
// The scan when the producer of the counts already wrote each block's total
// (block b: counts [b * scan_block_rows(), (b + 1) * scan_block_rows())) into
// partials[b]: the reduce pass is skipped.
long long scan_block_rows();
void scan_u32_to_u64_from_totals(const StreamRef& s, const unsigned int* counts, unsigned long long* offsets,
                                 long long n, unsigned long long* partials);

// Stable LSD radix sort of (key, value) pairs on bits [0, bits) of the key.
void radix_sort_pairs(const StreamRef& s, const Backend& b, unsigned long long* keys,
                      unsigned int* values, long long n, int bits);
// Orders n distinct keys in [0, span] and their values by key, into
// keys_out / values_out, without a sort: a span under 32768 in one launch (a
// presence bitmap and its ranks in shared memory), a span the keys fill to
// at least a quarter by presence flags in HBM and their scan.  False, with
// nothing launched, for a wider span.
bool order_distinct_keys(const StreamRef& s, const Backend& b, const unsigned long long* keys,
                          const unsigned int* values, long long n, unsigned long long span,
                          unsigned long long* keys_out, unsigned int* values_out);

// Minimum and maximum valid int key (as int64) of a column; false when none.
bool key_range(const StreamRef& s, const Backend& b, const Column& key, long long n,
               long long* lo, long long* hi, long long* count = nullptr);

// Operators.
oxb_batch* filter_project(const StreamRef& s, const Backend& b, const oxb_filter_project_args& a);
AllocRef predicate_bits(const StreamRef& s, const Backend& b, const DevPredicate& pred, long long n);
oxb_batch* aggregate_batches(const StreamRef& s, const Backend& b, const oxb_aggregate_batches_args& a);
oxb_server* server_create(oxb_backend* backend, const oxb_server_config& cfg);
void server_destroy(oxb_server* srv);
uint64_t server_submit_topk(oxb_server* srv, const oxb_topk_request& q);
uint64_t server_submit_join_aggregate(oxb_server* srv, const oxb_join_aggregate_args& a);
double server_wait(oxb_server* srv, uint64_t ticket, int64_t* ids, float* dist, oxb_batch** out);
void server_stats(oxb_server* srv, oxb_server_stats* out, bool reset);
oxb_vector_index* vector_index_build(const StreamRef& s, const Backend& b, const oxb_batch& in, int column);
void vector_topk(const StreamRef& s, const Backend& b, const oxb_vector_topk_args& a, int64_t* out_ids,
                 float* out_dist, oxb_vector_topk_stats* stats);
void filter_project_noalloc(const StreamRef& s, const Backend& b, const oxb_filter_project_args& a,
                            void* const* out_values, uint32_t* const* out_validity, long long capacity,
                            long long* out_rows);
oxb_join_table* prepare_join_build(const StreamRef& s, const Backend& b,
                                   const oxb_join_build_args& a);
oxb_join_matches* probe_join(const StreamRef& s, const Backend& b, const oxb_join_probe_args& a);
oxb_batch* hash_join(const StreamRef& s, const Backend& b, const oxb_hash_join_args& a);
oxb_batch* aggregate(const StreamRef& s, const Backend& b, const oxb_aggregate_args& a);
oxb_batch* vector_distance(const StreamRef& s, const Backend& b,
                           const oxb_vector_distance_args& a);
oxb_batch* join_aggregate(const StreamRef& s, const Backend& b, const oxb_join_aggregate_args& a);
// Requests of one shape (same_join_shape) in one launch; each result equals
// its own join_aggregate call's.
bool same_join_shape(const oxb_join_aggregate_args& a, const oxb_join_aggregate_args& z);
std::vector<oxb_batch*> join_aggregate_many(const StreamRef& s, const Backend& b, const oxb_join_aggregate_args* a,
                                            int n);
void launch_vector_distance(const StreamRef& s, const Backend& b, const Column& vec, long long n,
                            const float* dquery, int metric, float* out);

}  // namespace oxb
