// Ingest of host columns into device memory (oxb_upload), and the way back
// into pageable host memory (oxb_download_column).
//
// The reference uploads every batch from pageable memory with one plain copy
// per buffer (crates/oxidelake-device/src/cuda/mod.rs, `upload`; the
// operator's `round_trip`, crates/oxidelake-compute/src/operator.rs:589-600).
// The driver then stages pageable memory through its own page-locked buffer
// with one host thread.  Here a large pageable column goes through a ring of
// page-locked chunks that a few host threads fill: the host→device copy of
// chunk i runs while chunk i+1 is being filled, so the copy engine sees
// page-locked memory all the time.  Page-locked and device sources, and
// small columns, keep the single copy.  A large download into pageable
// memory runs the ring the other way: the device copies into one slot while
// the host threads drain the slot before it.  A batch's small columns into
// pageable memory are gathered in one page-locked buffer (download_pieces).
#include <condition_variable>
#include <cstring>
#include <thread>

#include "internal.h"

namespace oxb {

namespace {

constexpr size_t kStageChunk = size_t(8) << 20;  // bytes per ring slot
constexpr int kStageSlots = 4;
constexpr size_t kStageMin = size_t(4) << 20;  // smaller columns copy directly
constexpr int kMaxStageThreads = 32;

std::mutex g_stager_mu;  // guards Backend::stager and Backend::stage_threads

// True when the driver does not know `p` (plain pageable host memory).
bool is_pageable(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

}  // namespace

class Stager {
  public:
    Stager(int device, int threads) : device_(device) {
        for (int i = 0; i < kStageSlots; i++) {
            void* p = nullptr;
            cudaEvent_t e = nullptr;
            if (cudaMallocHost(&p, kStageChunk) != cudaSuccess || cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                if (p) cudaFreeHost(p);
                release();
                fail(OXB_ALLOCATION, "page-locked staging buffers could not be allocated");
            }
            slot_[i] = p;
            done_[i] = e;
        }
        // A thread that cannot start leaves the ones already running to be
        // stopped and joined here: the destructor does not run for a
        // constructor that throws, and a joinable std::thread must not be
        // destroyed.
        try {
            for (int i = 1; i < threads; i++) workers_.emplace_back([this, i] { work(i); });
        } catch (const std::exception& e) {
            stop_workers();
            release();
            fail(OXB_ALLOCATION, std::string("staging threads could not be started: ") + e.what());
        }
    }

    ~Stager() {
        stop_workers();
        release();
    }

    // Queues the copy of n bytes from pageable `src` to device `dst` on s.
    // On return `src` is no longer read: every byte sits in a page-locked
    // slot or on the device.
    void upload(const StreamRef& s, void* dst, const void* src, size_t n) {
        std::lock_guard<std::mutex> call(call_);
        for (size_t off = 0; off < n; off += kStageChunk) {
            const size_t len = std::min(kStageChunk, n - off);
            const int k = int(next_++ % kStageSlots);
            if (pending_[k]) OXB_CUDA(cudaEventSynchronize(done_[k]));  // the slot's last copy is done
            pending_[k] = false;
            fill((char*)slot_[k], (const char*)src + off, len);
            OXB_CUDA(cudaMemcpyAsync((char*)dst + off, slot_[k], len, cudaMemcpyHostToDevice, s->stream));
            OXB_CUDA(cudaEventRecord(done_[k], s->stream));
            pending_[k] = true;
        }
    }

    // Copies n bytes from device `src` to pageable `dst` through the slots,
    // draining one slot on the host while the copies into the next ones
    // run.  Returns once every byte is in `dst`.
    void download(const StreamRef& s, void* dst, const void* src, size_t n) {
        std::lock_guard<std::mutex> call(call_);
        for (int k = 0; k < kStageSlots; k++) {  // slots an upload may still be reading
            if (pending_[k]) OXB_CUDA(cudaEventSynchronize(done_[k]));
            pending_[k] = false;
        }
        const size_t chunks = (n + kStageChunk - 1) / kStageChunk;
        auto issue = [&](size_t c) {
            const int k = int(c % kStageSlots);
            const size_t off = c * kStageChunk, len = std::min(kStageChunk, n - off);
            OXB_CUDA(cudaMemcpyAsync(slot_[k], (const char*)src + off, len, cudaMemcpyDeviceToHost, s->stream));
            OXB_CUDA(cudaEventRecord(done_[k], s->stream));
            pending_[k] = true;
        };
        size_t issued = 0;
        for (; issued < chunks && issued < size_t(kStageSlots); issued++) issue(issued);
        for (size_t c = 0; c < chunks; c++) {
            const int k = int(c % kStageSlots);
            const size_t off = c * kStageChunk, len = std::min(kStageChunk, n - off);
            OXB_CUDA(cudaEventSynchronize(done_[k]));
            pending_[k] = false;
            fill((char*)dst + off, (const char*)slot_[k], len);
            if (issued < chunks) issue(issued++);  // chunk c + kStageSlots, into the slot just drained
        }
    }

  private:
    void stop_workers() {
        {
            std::lock_guard<std::mutex> l(m_);
            stop_ = true;
        }
        go_.notify_all();
        for (auto& t : workers_) t.join();
        workers_.clear();
    }

    // Frees the slots and events on the stager's device, then makes the
    // calling thread's previous device current again: the last reference
    // may be dropped on any thread, which must not find its device changed.
    void release() {
        int prev = -1;
        if (cudaGetDevice(&prev) != cudaSuccess) {
            cudaGetLastError();
            prev = -1;
        }
        cudaSetDevice(device_);
        for (int i = 0; i < kStageSlots; i++) {
            if (done_[i]) {
                if (pending_[i]) cudaEventSynchronize(done_[i]);
                cudaEventDestroy(done_[i]);
                done_[i] = nullptr;
            }
            if (slot_[i]) cudaFreeHost(slot_[i]);
            slot_[i] = nullptr;
        }
        if (prev >= 0 && prev != device_) cudaSetDevice(prev);
    }

    // Host copy of n bytes split over the workers and the calling thread,
    // in page-aligned parts.
    void fill(char* d, const char* s, size_t n) {
        const size_t parts = workers_.size() + 1;
        const size_t part = ((n + parts - 1) / parts + 4095) & ~size_t(4095);
        if (parts > 1) {
            {
                std::lock_guard<std::mutex> l(m_);
                jd_ = d;
                js_ = s;
                jn_ = n;
                jpart_ = part;
                left_ = int(parts - 1);
                gen_++;
            }
            go_.notify_all();
        }
        std::memcpy(d, s, std::min(n, part));
        if (parts > 1) {
            std::unique_lock<std::mutex> l(m_);
            fin_.wait(l, [&] { return left_ == 0; });
        }
    }

    // Worker i copies part i of each job.  A job is only posted after every
    // worker finished the one before, so no worker can miss one.
    void work(int i) {
        uint64_t seen = 0;
        for (;;) {
            std::unique_lock<std::mutex> l(m_);
            go_.wait(l, [&] { return stop_ || gen_ != seen; });
            if (stop_) return;
            seen = gen_;
            char* d = jd_;
            const char* s = js_;
            const size_t n = jn_, part = jpart_;
            l.unlock();
            const size_t lo = std::min(n, part * size_t(i)), hi = std::min(n, lo + part);
            if (hi > lo) std::memcpy(d + lo, s + lo, hi - lo);
            l.lock();
            if (--left_ == 0) fin_.notify_one();
        }
    }

    int device_;
    void* slot_[kStageSlots] = {};
    cudaEvent_t done_[kStageSlots] = {};
    bool pending_[kStageSlots] = {};
    uint64_t next_ = 0;
    std::mutex call_;  // one staged copy at a time per backend

    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable go_, fin_;
    char* jd_ = nullptr;
    const char* js_ = nullptr;
    size_t jn_ = 0, jpart_ = 0;
    uint64_t gen_ = 0;
    int left_ = 0;
    bool stop_ = false;
};

void set_upload_staging(Backend& b, int threads) {
    if (threads < 0 || threads > kMaxStageThreads)
        fail(OXB_PLAN, "staging threads must be in [0, " + std::to_string(kMaxStageThreads) + "]");
    std::shared_ptr<Stager> old;
    {
        std::lock_guard<std::mutex> l(g_stager_mu);
        old.swap(b.stager);
        b.stage_threads = threads;
    }
    // `old` is released here, after any upload holding it has finished.
}

void upload_bytes(Backend& b, const StreamRef& s, void* dst, const void* src, size_t n) {
    if (n == 0) return;
    std::shared_ptr<Stager> st;
    if (n >= kStageMin && is_pageable(src)) {
        std::lock_guard<std::mutex> l(g_stager_mu);
        if (b.stage_threads > 0) {
            if (!b.stager) b.stager = std::make_shared<Stager>(b.device, b.stage_threads);
            st = b.stager;
        }
    }
    if (st)
        st->upload(s, dst, src, n);
    else
        OXB_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, s->stream));
}

void download_bytes(Backend& b, const StreamRef& s, void* dst, const void* src, size_t n) {
    if (n == 0) return;
    std::shared_ptr<Stager> st;
    if (n >= kStageMin && is_pageable(dst)) {
        std::lock_guard<std::mutex> l(g_stager_mu);
        if (b.stage_threads > 0) {
            if (!b.stager) b.stager = std::make_shared<Stager>(b.device, b.stage_threads);
            st = b.stager;
        }
    }
    if (st)
        st->download(s, dst, src, n);
    else
        OXB_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, s->stream));
}

// A page-locked buffer a backend gathers small downloads in: a copy into
// pageable memory waits for the driver's own staging, about 15 us each, so a
// batch of ten small columns cost 0.15 ms copied one by one.
struct SmallDownloads {
    std::mutex mu;
    void* buf = nullptr;
    size_t cap = 0;
    ~SmallDownloads() {
        if (buf) cudaFreeHost(buf);
    }
};

namespace {
constexpr size_t kGatherMax = size_t(4) << 20;  // pageable downloads up to this total are gathered
std::mutex g_small_mu;                          // guards Backend::small_dl
}  // namespace

void download_pieces(Backend& b, const StreamRef& s, const std::vector<DownloadPiece>& pieces) {
    size_t total = 0;
    std::vector<size_t> at(pieces.size());
    std::vector<char> gather(pieces.size(), 0);
    for (size_t i = 0; i < pieces.size(); i++) {
        const DownloadPiece& p = pieces[i];
        if (p.n == 0 || p.n >= kStageMin || total + p.n > kGatherMax || !is_pageable(p.dst)) continue;
        gather[i] = 1;
        at[i] = total;
        total += (p.n + 15) & ~size_t(15);
    }
    std::shared_ptr<SmallDownloads> sd;
    if (total) {
        std::lock_guard<std::mutex> l(g_small_mu);
        if (!b.small_dl) b.small_dl = std::make_shared<SmallDownloads>();
        sd = b.small_dl;
    }
    std::unique_lock<std::mutex> hold;
    if (sd) {
        hold = std::unique_lock<std::mutex>(sd->mu);
        if (sd->cap < total) {
            if (sd->buf) OXB_CUDA(cudaFreeHost(sd->buf));
            sd->buf = nullptr;
            sd->cap = 0;
            const size_t want = std::max(total, size_t(1) << 20);
            OXB_CUDA(cudaMallocHost(&sd->buf, want));
            sd->cap = want;
        }
    }
    for (size_t i = 0; i < pieces.size(); i++) {
        const DownloadPiece& p = pieces[i];
        if (p.n == 0) continue;
        if (gather[i])
            OXB_CUDA(cudaMemcpyAsync((char*)sd->buf + at[i], p.src, p.n, cudaMemcpyDeviceToHost, s->stream));
        else
            download_bytes(b, s, p.dst, p.src, p.n);
    }
    OXB_CUDA(cudaStreamSynchronize(s->stream));
    for (size_t i = 0; i < pieces.size(); i++)
        if (gather[i]) std::memcpy(pieces[i].dst, (const char*)sd->buf + at[i], pieces[i].n);
}

}  // namespace oxb
