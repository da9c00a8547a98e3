// The C ABI of liboxb200 (include/oxb200.h): handle lifetimes, memory,
// streams, transfers, and the operator entry points.  Every entry point
// catches the runtime's errors at the boundary, records the message for
// oxb_last_error() and returns the status; nothing throws across the ABI
// and nothing falls back to the CPU.
#include <chrono>
#include <cstdio>
#include <map>
#include <new>
#include <thread>

#include "internal.h"

namespace oxb {

namespace {
thread_local std::string g_last_error;
thread_local std::string g_last_kernel;
thread_local float g_last_kernel_ms = 0.0f;
thread_local uint64_t g_kernel_times = 0;  // kernel times recorded on this thread
thread_local oxb_call_stats g_last_call{};
std::atomic<unsigned long long> g_launches{0};
}  // namespace

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

KernelTimer::KernelTimer(const Backend& b, const StreamRef& s, const char* name)
    : on_(b.timing), name_(name), stream_(s->stream) {}

void KernelTimer::begin() {
    if (!on_) return;
    cudaEvent_t a = nullptr, z = nullptr;
    OXB_CUDA(cudaEventCreate(&a));
    if (cudaEventCreate(&z) != cudaSuccess) {
        cudaEventDestroy(a);
        fail(OXB_DEVICE, "cudaEventCreate failed");
    }
    segs_.emplace_back(a, z);
    OXB_CUDA(cudaEventRecord(a, stream_));
}

void KernelTimer::end() {
    if (on_ && !segs_.empty()) {
        OXB_CUDA(cudaEventRecord(segs_.back().second, stream_));
        ended_ = true;
    }
}

KernelTimer::~KernelTimer() {
    if (!on_) return;
    if (ended_ && cudaEventSynchronize(segs_.back().second) == cudaSuccess) {
        float total = 0.0f;
        bool ok = true;
        for (auto& sg : segs_) {
            float ms = 0.0f;
            ok = ok && cudaEventElapsedTime(&ms, sg.first, sg.second) == cudaSuccess;
            total += ms;
        }
        if (ok) {
            g_last_kernel = name_;
            g_last_kernel_ms = total;
            g_kernel_times++;
        }
    }
    cudaGetLastError();
    for (auto& sg : segs_) {
        cudaEventDestroy(sg.first);
        cudaEventDestroy(sg.second);
    }
}

void fail(oxb_status status, const std::string& message) { throw Error{status, message}; }

void check_cuda(cudaError_t err, const char* what) {
    if (err == cudaSuccess) return;
    cudaGetLastError();  // clear a non-sticky error so the context stays usable
    fail(err == cudaErrorMemoryAllocation ? OXB_ALLOCATION : OXB_DEVICE,
         std::string(what) + ": " + cudaGetErrorString(err));
}

void check_status_word(uint32_t status, const char* what) {
    if (status & kStatusTableFull) fail(OXB_TABLE_FULL, std::string(what) + ": device hash table full");
    if (status & kStatusTimeout) fail(OXB_TIMEOUT, std::string(what) + ": a bounded device wait gave up");
    if (status & kStatusBounds) fail(OXB_EXECUTION, std::string(what) + ": an index failed its bounds check");
}

StreamState::~StreamState() {
    if (owned && stream) {
        cudaSetDevice(device);
        cudaStreamDestroy(stream);
    }
}

DevAlloc::~DevAlloc() {
    if (ptr) {
        cudaSetDevice(stream->device);
        cudaFreeAsync(ptr, stream->stream);
    }
}

int allow_smem_cap(const void* kernel) {
    int dev = 0;
    OXB_CUDA(cudaGetDevice(&dev));
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> caps;
    std::lock_guard<std::mutex> l(mu);
    const auto it = caps.find({kernel, dev});
    if (it != caps.end()) return it->second;
    int optin = 0;
    OXB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa{};
    OXB_CUDA(cudaFuncGetAttributes(&fa, kernel));
    const int cap = optin - (int)fa.sharedSizeBytes;
    if (cap > 48 * 1024) OXB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, cap));
    caps[{kernel, dev}] = cap;
    return cap;
}

AllocRef dev_alloc(const StreamRef& s, size_t bytes, bool zero) {
    auto a = std::make_shared<DevAlloc>();
    a->stream = s;
    a->bytes = bytes;
    size_t rounded = ((bytes ? bytes : 1) + 255) & ~size_t(255);
    cudaError_t e = cudaMallocAsync(&a->ptr, rounded, s->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        a->ptr = nullptr;
        fail(OXB_ALLOCATION, "allocation of " + std::to_string(bytes) + " device bytes failed: " +
                                 cudaGetErrorString(e));
    }
    if (((uintptr_t)a->ptr & 255) != 0) fail(OXB_DEVICE, "device allocation is not 256-byte aligned");
    if (zero) OXB_CUDA(cudaMemsetAsync(a->ptr, 0, rounded, s->stream));
    return a;
}

}  // namespace oxb

using namespace oxb;

namespace {

// One entry point's counters: filled in by the call, then kept as the
// thread's last call and added to the backend's totals for its operator.
class CallRecord {
  public:
    CallRecord(oxb_backend* be, int op) : be_(be), t0_(std::chrono::steady_clock::now()), timed0_(g_kernel_times) {
        st.op = op;
        st.batches = 1;
    }
    void finish(oxb_status status) {
        st.status = status;
        st.elapsed_ns = (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                            std::chrono::steady_clock::now() - t0_)
                            .count();
        if (status != OXB_OK) st.rows_out = 0;
        st.device_ns = status == OXB_OK && g_kernel_times != timed0_ ? (uint64_t)(g_last_kernel_ms * 1e6) : 0;
        g_last_call = st;
        if (!be_ || st.op < 0 || st.op >= OXB_OP_COUNT) return;
        std::atomic<uint64_t>* t = be_->tel.v[st.op];
        const uint64_t add[Telemetry::kFields] = {
            1, status == OXB_OK ? st.batches : 0, st.rows_in, st.rows_out, st.elapsed_ns, st.device_ns,
            st.bytes_h2d, st.bytes_d2h, status == OXB_UNSUPPORTED ? 1u : 0u,
            status != OXB_OK && status != OXB_UNSUPPORTED ? 1u : 0u, 0u /* no CPU path: never a fallback */};
        for (int i = 0; i < Telemetry::kFields; i++)
            if (add[i]) t[i].fetch_add(add[i], std::memory_order_relaxed);
    }
    oxb_call_stats st{};

  private:
    oxb_backend* be_;
    std::chrono::steady_clock::time_point t0_;
    uint64_t timed0_;
};

// Runs an entry point's body, turning the runtime's errors into its status
// (the message kept for oxb_last_error) and recording the call's counters.
template <typename F>
oxb_status counted(oxb_backend* backend, int op, F&& body) {
    CallRecord rec(backend, op);
    oxb_status status = OXB_OK;
    try {
        body(rec.st);
    } catch (const Error& e) {
        g_last_error = e.message;
        status = e.status;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        status = OXB_ALLOCATION;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        status = OXB_EXECUTION;
    }
    rec.finish(status);
    return status;
}

uint64_t column_bytes(const Column& c) {
    return (uint64_t)c.length * c.width() + (c.validity ? ((uint64_t)c.length + 7) / 8 : 0);
}

}  // namespace

#define OXB_TRY try {
#define OXB_CATCH                                                                \
    }                                                                            \
    catch (const Error& e) {                                                     \
        g_last_error = e.message;                                                \
        return e.status;                                                         \
    }                                                                            \
    catch (const std::bad_alloc&) {                                              \
        g_last_error = "host allocation failed";                                 \
        return OXB_ALLOCATION;                                                   \
    }                                                                            \
    catch (const std::exception& e) {                                            \
        g_last_error = e.what();                                                 \
        return OXB_EXECUTION;                                                    \
    }                                                                            \
    return OXB_OK;

namespace {

void use_device(const oxb_backend* b) {
    if (!b) fail(OXB_PLAN, "backend is null");
    OXB_CUDA(cudaSetDevice(b->b.device));
}

const StreamRef& stream_of(const oxb_stream* s) {
    if (!s) fail(OXB_PLAN, "stream is null");
    return s->s;
}

}  // namespace

extern "C" {

const char* oxb_last_error(void) { return g_last_error.c_str(); }

int32_t oxb_abi_version(void) { return OXB_ABI_VERSION; }

oxb_status oxb_backend_create(int32_t device, oxb_backend** out) {
    OXB_TRY
    if (!out) fail(OXB_PLAN, "out is null");
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        fail(OXB_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    }
    if (device < 0 || device >= count) fail(OXB_PLAN, "device " + std::to_string(device) + " does not exist");
    OXB_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop{};
    OXB_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
        fail(OXB_UNSUPPORTED, std::string("device ") + prop.name + " is not sm_100 (this library is built for sm_100a)");
    OXB_CUDA(cudaFree(nullptr));
    cudaMemPool_t pool;
    OXB_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t threshold = UINT64_MAX;  // keep freed blocks cached in the pool
    OXB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
    auto b = new oxb_backend();
    b->b.device = device;
    b->b.sms = prop.multiProcessorCount;
    b->b.smem_optin = prop.sharedMemPerBlockOptin;
    b->b.name = prop.name;
    // Half the host's cores, at most 8: 8 threads fill the staging ring at
    // about the copy engine's rate from page-locked memory.
    b->b.stage_threads = std::clamp(int(std::thread::hardware_concurrency() / 2), 1, 8);
    *out = b;
    OXB_CATCH
}

void oxb_backend_destroy(oxb_backend* backend) { delete backend; }

const char* oxb_backend_kind(const oxb_backend* backend) {
    (void)backend;
    return "cuda";
}

int32_t oxb_backend_device_id(const oxb_backend* backend) { return backend ? backend->b.device : -1; }

oxb_status oxb_memory_info_get(oxb_backend* backend, oxb_memory_info* out) {
    OXB_TRY
    use_device(backend);
    if (!out) fail(OXB_PLAN, "out is null");
    size_t free_b = 0, total_b = 0;
    OXB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    out->total_bytes = total_b;
    out->free_bytes = free_b;
    out->pinned_supported = 1;
    out->reserved = 0;
    OXB_CATCH
}

oxb_status oxb_stream_create(oxb_backend* backend, oxb_stream** out) {
    OXB_TRY
    use_device(backend);
    if (!out) fail(OXB_PLAN, "out is null");
    auto st = std::make_shared<StreamState>();
    st->device = backend->b.device;
    st->owned = true;
    OXB_CUDA(cudaStreamCreateWithFlags(&st->stream, cudaStreamNonBlocking));
    *out = new oxb_stream{st};
    OXB_CATCH
}

oxb_status oxb_stream_wrap(oxb_backend* backend, void* cuda_stream, oxb_stream** out) {
    OXB_TRY
    use_device(backend);
    if (!out) fail(OXB_PLAN, "out is null");
    auto st = std::make_shared<StreamState>();
    st->device = backend->b.device;
    st->owned = false;
    st->stream = (cudaStream_t)cuda_stream;
    *out = new oxb_stream{st};
    OXB_CATCH
}

void* oxb_stream_cuda_handle(const oxb_stream* stream) { return stream ? (void*)stream->s->stream : nullptr; }

oxb_status oxb_stream_synchronize(oxb_backend* backend, oxb_stream* stream) {
    OXB_TRY
    use_device(backend);
    OXB_CUDA(cudaStreamSynchronize(stream_of(stream)->stream));
    OXB_CATCH
}

void oxb_stream_destroy(oxb_stream* stream) { delete stream; }

oxb_status oxb_alloc_device(oxb_backend* backend, size_t bytes, oxb_buffer** out) {
    OXB_TRY
    use_device(backend);
    if (!out) fail(OXB_PLAN, "out is null");
    // Allocations made outside any call's stream live on a backend-wide stream.
    static thread_local StreamRef alloc_stream;
    if (!alloc_stream || alloc_stream->device != backend->b.device) {
        alloc_stream = std::make_shared<StreamState>();
        alloc_stream->device = backend->b.device;
        alloc_stream->owned = true;
        OXB_CUDA(cudaStreamCreateWithFlags(&alloc_stream->stream, cudaStreamNonBlocking));
    }
    AllocRef a = dev_alloc(alloc_stream, bytes, true);
    OXB_CUDA(cudaStreamSynchronize(alloc_stream->stream));
    auto buf = new oxb_buffer{a};
    buf->a->bytes = bytes;
    *out = buf;
    OXB_CATCH
}

void* oxb_buffer_device_ptr(const oxb_buffer* buffer) { return buffer ? buffer->a->ptr : nullptr; }
size_t oxb_buffer_len(const oxb_buffer* buffer) { return buffer ? buffer->a->bytes : 0; }
void oxb_buffer_free(oxb_buffer* buffer) { delete buffer; }

oxb_status oxb_alloc_pinned_host(oxb_backend* backend, size_t bytes, oxb_host_buffer** out) {
    OXB_TRY
    use_device(backend);
    if (!out) fail(OXB_PLAN, "out is null");
    auto h = new oxb_host_buffer();
    h->bytes = bytes;
    if (cudaMallocHost(&h->ptr, bytes ? bytes : 1) == cudaSuccess) {
        h->pinned = true;
    } else {
        cudaGetLastError();
        h->ptr = std::malloc(bytes ? bytes : 1);
        h->pinned = false;
        if (!h->ptr) {
            delete h;
            fail(OXB_ALLOCATION, "host allocation of " + std::to_string(bytes) + " bytes failed");
        }
    }
    *out = h;
    OXB_CATCH
}

void* oxb_host_buffer_ptr(const oxb_host_buffer* buffer) { return buffer ? buffer->ptr : nullptr; }
size_t oxb_host_buffer_len(const oxb_host_buffer* buffer) { return buffer ? buffer->bytes : 0; }
int32_t oxb_host_buffer_is_pinned(const oxb_host_buffer* buffer) { return buffer && buffer->pinned ? 1 : 0; }
void oxb_host_buffer_free(oxb_host_buffer* buffer) {
    if (!buffer) return;
    if (buffer->pinned) cudaFreeHost(buffer->ptr);
    else std::free(buffer->ptr);
    delete buffer;
}

oxb_status oxb_copy_h2d(oxb_backend* backend, oxb_stream* stream, const oxb_host_buffer* src, oxb_buffer* dst) {
    OXB_TRY
    use_device(backend);
    if (!src || !dst) fail(OXB_PLAN, "null buffer");
    size_t n = std::min(src->bytes, dst->a->bytes);
    OXB_CUDA(cudaMemcpyAsync(dst->a->ptr, src->ptr, n, cudaMemcpyHostToDevice, stream_of(stream)->stream));
    OXB_CATCH
}

oxb_status oxb_copy_d2h(oxb_backend* backend, oxb_stream* stream, const oxb_buffer* src, oxb_host_buffer* dst) {
    OXB_TRY
    use_device(backend);
    if (!src || !dst) fail(OXB_PLAN, "null buffer");
    size_t n = std::min(src->a->bytes, dst->bytes);
    OXB_CUDA(cudaMemcpyAsync(dst->ptr, src->a->ptr, n, cudaMemcpyDeviceToHost, stream_of(stream)->stream));
    OXB_CATCH
}

}  // extern "C"

namespace {

void check_column_desc(const oxb_column& c, int64_t rows, int i) {
    if (c.type < OXB_TYPE_INT64 || c.type > OXB_TYPE_VECTOR_F32)
        fail(OXB_UNSUPPORTED, "column " + std::to_string(i) + " has an unsupported type " + std::to_string(c.type));
    if (c.type == OXB_TYPE_VECTOR_F32 && c.dim <= 0) fail(OXB_PLAN, "vector column with dim <= 0");
    if (c.length != rows)
        fail(OXB_PLAN, "column " + std::to_string(i) + " has " + std::to_string(c.length) + " rows, the batch " +
                           std::to_string(rows));
    if (rows > 0 && !c.values) fail(OXB_PLAN, "column " + std::to_string(i) + " has no values");
}

}  // namespace

extern "C" {

}  // extern "C"

namespace oxb {

// The body of oxb_upload (and of the Arrow import): each host column into
// new device memory, queued on the stream.
std::unique_ptr<oxb_batch> upload_columns(oxb_backend* backend, const StreamRef& s, const oxb_column* columns,
                                          int32_t ncols, int64_t rows, oxb_call_stats& st) {
    if ((ncols > 0 && !columns) || ncols < 0 || rows < 0) fail(OXB_PLAN, "bad upload arguments");
    auto b = std::make_unique<oxb_batch>();
    b->rows = rows;
    for (int i = 0; i < ncols; i++) {
        const oxb_column& c = columns[i];
        check_column_desc(c, rows, i);
        Column d;
        d.type = c.type;
        d.dim = c.type == OXB_TYPE_VECTOR_F32 ? c.dim : 1;
        d.length = rows;
        if (rows > 0) {
            size_t bytes = (size_t)rows * d.width();
            d.owner_values = dev_alloc(s, bytes, false);
            d.values = d.owner_values->ptr;
            upload_bytes(backend->b, s, d.values, c.values, bytes);
            if (c.validity) {
                size_t vb = ((size_t)rows + 7) / 8;
                d.owner_validity = dev_alloc(s, vb, false);
                d.validity = (uint8_t*)d.owner_validity->ptr;
                upload_bytes(backend->b, s, d.validity, c.validity, vb);
            }
        }
        st.bytes_h2d += column_bytes(d);
        b->cols.push_back(std::move(d));
    }
    st.rows_in = st.rows_out = (uint64_t)rows;
    return b;
}

}  // namespace oxb

extern "C" {

oxb_status oxb_upload(oxb_backend* backend, oxb_stream* stream, const oxb_column* columns, int32_t ncols, int64_t rows,
                      oxb_batch** out) {
    return counted(backend, OXB_OP_TRANSFER, [&](oxb_call_stats& st) {
        use_device(backend);
        const StreamRef& s = stream_of(stream);
        if (!out) fail(OXB_PLAN, "bad upload arguments");
        *out = upload_columns(backend, s, columns, ncols, rows, st).release();
    });
}

oxb_status oxb_import_arrow(oxb_backend* backend, oxb_stream* stream, struct ArrowArray* array,
                            struct ArrowSchema* schema, oxb_batch** out) {
    return counted(backend, OXB_OP_TRANSFER, [&](oxb_call_stats& st) {
        use_device(backend);
        const StreamRef& s = stream_of(stream);
        if (!out || !array || !schema) fail(OXB_PLAN, "null Arrow import argument");
        ArrowImport imp = arrow_import_columns(array, schema);
        auto b = upload_columns(backend, s, imp.cols.data(), (int32_t)imp.cols.size(), array->length, st);
        OXB_CUDA(cudaStreamSynchronize(s->stream));  // the Arrow buffers are read before they are released
        array->release(array);
        schema->release(schema);
        *out = b.release();
    });
}

oxb_status oxb_export_arrow(oxb_backend* backend, oxb_stream* stream, const oxb_batch* batch,
                            const char* const* names, struct ArrowArray* out_array, struct ArrowSchema* out_schema) {
    return counted(backend, OXB_OP_TRANSFER, [&](oxb_call_stats& st) {
        use_device(backend);
        const StreamRef& s = stream_of(stream);
        if (!batch || !out_array || !out_schema) fail(OXB_PLAN, "null Arrow export argument");
        arrow_export_batch(backend->b, s, *batch, names, out_array, out_schema, st);
    });
}

oxb_status oxb_batch_from_device(oxb_backend* backend, const oxb_column* columns, int32_t ncols, int64_t rows,
                                 oxb_batch** out) {
    OXB_TRY
    use_device(backend);
    if (!out || (ncols > 0 && !columns) || ncols < 0 || rows < 0) fail(OXB_PLAN, "bad batch arguments");
    auto b = std::make_unique<oxb_batch>();
    b->rows = rows;
    for (int i = 0; i < ncols; i++) {
        const oxb_column& c = columns[i];
        check_column_desc(c, rows, i);
        Column d;
        d.type = c.type;
        d.dim = c.type == OXB_TYPE_VECTOR_F32 ? c.dim : 1;
        d.length = rows;
        d.values = const_cast<void*>(c.values);
        d.validity = const_cast<uint8_t*>(c.validity);
        b->cols.push_back(std::move(d));
    }
    *out = b.release();
    OXB_CATCH
}

int64_t oxb_batch_num_rows(const oxb_batch* batch) { return batch ? batch->rows : -1; }
int32_t oxb_batch_num_columns(const oxb_batch* batch) { return batch ? (int32_t)batch->cols.size() : -1; }

oxb_status oxb_batch_column(const oxb_batch* batch, int32_t index, oxb_column* out) {
    OXB_TRY
    if (!batch || !out) fail(OXB_PLAN, "null argument");
    if (index < 0 || index >= (int)batch->cols.size()) fail(OXB_PLAN, "column index out of range");
    const Column& c = batch->cols[index];
    out->type = c.type;
    out->dim = c.dim;
    out->length = c.length;
    out->values = c.values;
    out->validity = c.validity;
    OXB_CATCH
}

oxb_status oxb_download_column(oxb_backend* backend, oxb_stream* stream, const oxb_batch* batch, int32_t index,
                               void* values, uint8_t* validity, int32_t* has_validity) {
    return counted(backend, OXB_OP_TRANSFER, [&](oxb_call_stats& st) {
        use_device(backend);
        const StreamRef& s = stream_of(stream);
        if (!batch) fail(OXB_PLAN, "batch is null");
        if (index < 0 || index >= (int)batch->cols.size()) fail(OXB_PLAN, "column index out of range");
        const Column& c = batch->cols[index];
        if (has_validity) *has_validity = c.validity ? 1 : 0;
        if (c.length > 0) {
            if (!values) fail(OXB_PLAN, "values buffer is null");
            download_bytes(backend->b, s, values, c.values, (size_t)c.length * c.width());
            st.bytes_d2h += (uint64_t)c.length * c.width();
            if (c.validity && validity) {
                OXB_CUDA(cudaMemcpyAsync(validity, c.validity, ((size_t)c.length + 7) / 8, cudaMemcpyDeviceToHost,
                                         s->stream));
                st.bytes_d2h += ((uint64_t)c.length + 7) / 8;
            }
        }
        OXB_CUDA(cudaStreamSynchronize(s->stream));
        st.rows_in = st.rows_out = (uint64_t)c.length;
    });
}

oxb_status oxb_download(oxb_backend* backend, oxb_stream* stream, const oxb_batch* batch, int32_t ncols,
                        void* const* values, uint8_t* const* validity, int32_t* has_validity) {
    return counted(backend, OXB_OP_TRANSFER, [&](oxb_call_stats& st) {
        use_device(backend);
        const StreamRef& s = stream_of(stream);
        if (!batch) fail(OXB_PLAN, "batch is null");
        if (ncols != (int32_t)batch->cols.size())
            fail(OXB_PLAN, "the batch has " + std::to_string(batch->cols.size()) + " columns, not " +
                               std::to_string(ncols));
        if (ncols > 0 && (!values || !has_validity)) fail(OXB_PLAN, "null output arrays");
        std::vector<DownloadPiece> pieces;
        for (int i = 0; i < ncols; i++) {
            const Column& c = batch->cols[i];
            has_validity[i] = c.validity ? 1 : 0;
            if (c.length == 0) continue;
            if (!values[i]) fail(OXB_PLAN, "values buffer of column " + std::to_string(i) + " is null");
            pieces.push_back(DownloadPiece{values[i], c.values, (size_t)c.length * c.width()});
            st.bytes_d2h += (uint64_t)c.length * c.width();
            if (c.validity && validity && validity[i]) {
                pieces.push_back(DownloadPiece{validity[i], c.validity, ((size_t)c.length + 7) / 8});
                st.bytes_d2h += ((uint64_t)c.length + 7) / 8;
            }
        }
        download_pieces(backend->b, s, pieces);
        st.rows_in = st.rows_out = (uint64_t)batch->rows;
    });
}

void oxb_batch_free(oxb_batch* batch) { delete batch; }

oxb_status oxb_filter_project(oxb_backend* backend, oxb_stream* stream, const oxb_filter_project_args* args,
                              oxb_batch** out) {
    return counted(backend, OXB_OP_FILTER, [&](oxb_call_stats& st) {
        use_device(backend);
        if (!args || !out) fail(OXB_PLAN, "null argument");
        st.rows_in = args->input ? (uint64_t)args->input->rows : 0;
        *out = filter_project(stream_of(stream), backend->b, *args);
        st.rows_out = (uint64_t)(*out)->rows;
    });
}

oxb_status oxb_filter_project_noalloc(oxb_backend* backend, oxb_stream* stream, const oxb_filter_project_args* args,
                                      void* const* out_values, uint32_t* const* out_validity, int64_t capacity,
                                      int64_t* out_rows) {
    return counted(backend, OXB_OP_FILTER, [&](oxb_call_stats& st) {
        use_device(backend);
        if (!args) fail(OXB_PLAN, "null argument");
        st.rows_in = args->input ? (uint64_t)args->input->rows : 0;
        long long rows = 0;
        try {
            filter_project_noalloc(stream_of(stream), backend->b, *args, out_values, out_validity, capacity, &rows);
        } catch (...) {
            if (out_rows) *out_rows = rows;
            throw;
        }
        if (out_rows) *out_rows = rows;
        st.rows_out = (uint64_t)rows;
    });
}

oxb_status oxb_prepare_join_build(oxb_backend* backend, oxb_stream* stream, const oxb_join_build_args* args,
                                  oxb_join_table** out) {
    return counted(backend, OXB_OP_JOIN, [&](oxb_call_stats& st) {
        use_device(backend);
        if (!args || !out) fail(OXB_PLAN, "null argument");
        *out = prepare_join_build(stream_of(stream), backend->b, *args);
        st.rows_in = (uint64_t)(*out)->build_rows;
    });
}

int64_t oxb_join_table_distinct_keys(const oxb_join_table* table) { return table ? table->t.ndistinct : -1; }
int64_t oxb_join_table_rows(const oxb_join_table* table) { return table ? table->t.nrows : -1; }
void oxb_join_table_free(oxb_join_table* table) { delete table; }

oxb_status oxb_probe_join(oxb_backend* backend, oxb_stream* stream, const oxb_join_probe_args* args,
                          oxb_join_matches** out) {
    return counted(backend, OXB_OP_JOIN, [&](oxb_call_stats& st) {
        use_device(backend);
        if (!args || !out) fail(OXB_PLAN, "null argument");
        *out = probe_join(stream_of(stream), backend->b, *args);
        st.rows_in = (uint64_t)(*out)->probe_rows;
        st.rows_out = (*out)->total;
    });
}

uint64_t oxb_join_matches_len(const oxb_join_matches* matches) { return matches ? matches->total : 0; }
int64_t oxb_join_matches_probe_rows(const oxb_join_matches* matches) { return matches ? matches->probe_rows : -1; }
void oxb_join_matches_free(oxb_join_matches* matches) { delete matches; }

oxb_status oxb_hash_join(oxb_backend* backend, oxb_stream* stream, const oxb_hash_join_args* args, oxb_batch** out) {
    return counted(backend, OXB_OP_JOIN, [&](oxb_call_stats& st) {
        use_device(backend);
        if (!args || !out) fail(OXB_PLAN, "null argument");
        *out = hash_join(stream_of(stream), backend->b, *args);
        st.rows_in = st.rows_out = (uint64_t)(*out)->rows;
    });
}

oxb_status oxb_aggregate(oxb_backend* backend, oxb_stream* stream, const oxb_aggregate_args* args, oxb_batch** out) {
    return counted(backend, OXB_OP_AGGREGATE, [&](oxb_call_stats& st) {
        use_device(backend);
        if (!args || !out) fail(OXB_PLAN, "null argument");
        st.rows_in = args->input ? (uint64_t)args->input->rows : 0;
        *out = aggregate(stream_of(stream), backend->b, *args);
        st.rows_out = (uint64_t)(*out)->rows;
    });
}

oxb_status oxb_join_aggregate(oxb_backend* backend, oxb_stream* stream, const oxb_join_aggregate_args* args,
                              oxb_batch** out) {
    return counted(backend, OXB_OP_AGGREGATE, [&](oxb_call_stats& st) {
        use_device(backend);
        if (!args || !out) fail(OXB_PLAN, "null argument");
        st.rows_in = args->probe ? (uint64_t)args->probe->rows : 0;
        *out = join_aggregate(stream_of(stream), backend->b, *args);
        st.rows_out = (uint64_t)(*out)->rows;
    });
}

oxb_status oxb_join_aggregate_many(oxb_backend* backend, oxb_stream* stream, const oxb_join_aggregate_args* args,
                                   int32_t n, oxb_batch** out) {
    return counted(backend, OXB_OP_AGGREGATE, [&](oxb_call_stats& st) {
        use_device(backend);
        if (n < 0 || (n > 0 && (!args || !out))) fail(OXB_PLAN, "null argument");
        for (int i = 0; i < n; i++) {
            if (!args[i].probe || !args[i].table || !args[i].build) fail(OXB_PLAN, "request without probe, build or table");
            st.rows_in += (uint64_t)args[i].probe->rows;
        }
        st.batches = (uint64_t)n;
        std::vector<oxb_batch*> res = join_aggregate_many(stream_of(stream), backend->b, args, n);
        for (int i = 0; i < n; i++) {
            out[i] = res[i];
            st.rows_out += (uint64_t)res[i]->rows;
        }
    });
}

oxb_status oxb_vector_distance(oxb_backend* backend, oxb_stream* stream, const oxb_vector_distance_args* args,
                               oxb_batch** out) {
    return counted(backend, OXB_OP_VECTOR, [&](oxb_call_stats& st) {
        use_device(backend);
        if (!args || !out) fail(OXB_PLAN, "null argument");
        st.rows_in = args->input ? (uint64_t)args->input->rows : 0;
        st.bytes_h2d = args->dim > 0 ? (uint64_t)args->dim * 4 : 0;  // the query
        *out = vector_distance(stream_of(stream), backend->b, *args);
        st.rows_out = (uint64_t)(*out)->rows;
    });
}

oxb_status oxb_aggregate_batches(oxb_backend* backend, oxb_stream* stream, const oxb_aggregate_batches_args* args,
                                 oxb_batch** out) {
    return counted(backend, OXB_OP_AGGREGATE, [&](oxb_call_stats& st) {
        use_device(backend);
        if (!args || !out) fail(OXB_PLAN, "null argument");
        if (args->inputs && args->ninputs > 0) {
            st.batches = (uint64_t)args->ninputs;
            for (int i = 0; i < args->ninputs; i++)
                if (args->inputs[i]) st.rows_in += (uint64_t)args->inputs[i]->rows;
        }
        *out = aggregate_batches(stream_of(stream), backend->b, *args);
        st.rows_out = (uint64_t)(*out)->rows;
    });
}

oxb_status oxb_server_create(oxb_backend* backend, const oxb_server_config* config, oxb_server** out) {
    OXB_TRY
    use_device(backend);
    if (!out) fail(OXB_PLAN, "null argument");
    oxb_server_config cfg{};
    if (config) cfg = *config;
    *out = server_create(backend, cfg);
    OXB_CATCH
}

void oxb_server_destroy(oxb_server* server) { server_destroy(server); }

oxb_status oxb_server_submit_topk(oxb_server* server, const oxb_topk_request* request, uint64_t* ticket) {
    OXB_TRY
    if (!server || !request || !ticket) fail(OXB_PLAN, "null argument");
    *ticket = server_submit_topk(server, *request);
    OXB_CATCH
}

oxb_status oxb_server_submit_join_aggregate(oxb_server* server, const oxb_join_aggregate_args* request,
                                            uint64_t* ticket) {
    OXB_TRY
    if (!server || !request || !ticket) fail(OXB_PLAN, "null argument");
    *ticket = server_submit_join_aggregate(server, *request);
    OXB_CATCH
}

oxb_status oxb_server_wait_topk(oxb_server* server, uint64_t ticket, int64_t* ids, float* dist, double* latency_us) {
    OXB_TRY
    if (!server) fail(OXB_PLAN, "null argument");
    const double l = server_wait(server, ticket, ids, dist, nullptr);
    if (latency_us) *latency_us = l;
    OXB_CATCH
}

oxb_status oxb_server_wait_batch(oxb_server* server, uint64_t ticket, oxb_batch** out, double* latency_us) {
    OXB_TRY
    if (!server) fail(OXB_PLAN, "null argument");
    const double l = server_wait(server, ticket, nullptr, nullptr, out);
    if (latency_us) *latency_us = l;
    OXB_CATCH
}

oxb_status oxb_server_stats_get(oxb_server* server, oxb_server_stats* out, int32_t reset) {
    OXB_TRY
    if (!server || !out) fail(OXB_PLAN, "null argument");
    server_stats(server, out, reset != 0);
    OXB_CATCH
}

oxb_status oxb_vector_index_build(oxb_backend* backend, oxb_stream* stream, const oxb_batch* input, int32_t column,
                                  oxb_vector_index** out) {
    OXB_TRY
    use_device(backend);
    if (!input || !out) fail(OXB_PLAN, "null argument");
    *out = vector_index_build(stream_of(stream), backend->b, *input, column);
    OXB_CATCH
}

void oxb_vector_index_free(oxb_vector_index* index) { delete index; }

oxb_status oxb_vector_topk(oxb_backend* backend, oxb_stream* stream, const oxb_vector_topk_args* args,
                           int64_t* out_ids, float* out_dist, oxb_vector_topk_stats* stats) {
    return counted(backend, OXB_OP_VECTOR, [&](oxb_call_stats& st) {
        use_device(backend);
        if (!args) fail(OXB_PLAN, "null argument");
        st.rows_in = args->index ? (uint64_t)args->index->n : 0;
        vector_topk(stream_of(stream), backend->b, *args, out_ids, out_dist, stats);
        const uint64_t nq = (uint64_t)std::max(args->nqueries, 0), k = (uint64_t)std::max(args->k, 0);
        st.rows_out = nq * k;
        st.bytes_h2d = nq * (uint64_t)std::max(args->dim, 0) * 4 + (args->qleaf_column >= 0 ? nq * 8 : 0);
        st.bytes_d2h = nq * k * 12;  // ids and distances
    });
}

oxb_status oxb_last_call_stats(oxb_call_stats* out) {
    if (!out) return OXB_PLAN;
    *out = g_last_call;
    return OXB_OK;
}

oxb_status oxb_operator_stats_get(oxb_backend* backend, int32_t op, oxb_operator_stats* out, int32_t reset) {
    OXB_TRY
    if (!backend || !out) fail(OXB_PLAN, "null argument");
    if (op < 0 || op >= OXB_OP_COUNT) fail(OXB_PLAN, "operator " + std::to_string(op) + " does not exist");
    std::atomic<uint64_t>* t = backend->tel.v[op];
    uint64_t v[Telemetry::kFields];
    for (int i = 0; i < Telemetry::kFields; i++)
        v[i] = reset ? t[i].exchange(0, std::memory_order_relaxed) : t[i].load(std::memory_order_relaxed);
    out->calls = v[0];
    out->batches = v[1];
    out->rows_in = v[2];
    out->rows_out = v[3];
    out->elapsed_ns = v[4];
    out->device_ns = v[5];
    out->bytes_h2d = v[6];
    out->bytes_d2h = v[7];
    out->unsupported = v[8];
    out->failed = v[9];
    out->fallback_batches = v[10];
    OXB_CATCH
}

int32_t oxb_supports_predicate(const oxb_backend* backend, const oxb_leaf* leaves, int32_t nleaves) {
    (void)backend;
    if (nleaves < 0 || nleaves > OXB_MAX_PREDICATE_LEAVES) return 0;
    for (int i = 0; i < nleaves; i++) {
        int t = leaves[i].lit_type;
        if (t != OXB_TYPE_INT64 && t != OXB_TYPE_FLOAT64 && t != OXB_TYPE_INT32) return 0;
        if (leaves[i].op < 0 || leaves[i].op > 4) return 0;
    }
    return 1;
}

oxb_status oxb_set_kernel_timing(oxb_backend* backend, int32_t enabled) {
    OXB_TRY
    if (!backend) fail(OXB_PLAN, "backend is null");
    backend->b.timing = enabled != 0;
    OXB_CATCH
}

oxb_status oxb_last_kernel_time(oxb_backend* backend, char* name, int32_t name_len, float* ms) {
    OXB_TRY
    if (!backend || !ms) fail(OXB_PLAN, "null argument");
    *ms = g_last_kernel_ms;
    if (name && name_len > 0) {
        std::snprintf(name, (size_t)name_len, "%s", g_last_kernel.c_str());
    }
    OXB_CATCH
}

uint64_t oxb_kernel_launches(void) { return g_launches.load(); }

oxb_status oxb_set_agg_variant(oxb_backend* backend, int32_t combine, int32_t rows_per_thread) {
    OXB_TRY
    if (!backend) fail(OXB_PLAN, "backend is null");
    if (combine < -1 || combine > 17) fail(OXB_PLAN, "combine must be -1 or 0..17");
    if (rows_per_thread != 0 && rows_per_thread != 1 && rows_per_thread != 2 && rows_per_thread != 4 &&
        rows_per_thread != 8)
        fail(OXB_UNSUPPORTED, "rows per thread must be 0 (automatic), 1, 2 or 4");
    backend->b.force_combine = combine;
    backend->b.force_rpt = rows_per_thread;
    OXB_CATCH
}

oxb_status oxb_set_upload_staging(oxb_backend* backend, int32_t threads) {
    OXB_TRY
    use_device(backend);
    set_upload_staging(backend->b, threads);
    OXB_CATCH
}

oxb_status oxb_set_autotune(oxb_backend* backend, int32_t enabled) {
    OXB_TRY
    if (!backend) fail(OXB_PLAN, "backend is null");
    backend->b.autotune = enabled != 0;
    OXB_CATCH
}

int32_t oxb_supports_hash_join(const oxb_backend* backend) {
    (void)backend;
    return 1;
}

int32_t oxb_supports_aggregate(const oxb_backend* backend) {
    (void)backend;
    return 1;
}

}  // extern "C"
