// Fused filter + projection (GpuBackend::filter_project,
// crates/oxidelake-device/src/backend.rs:98; semantics cpu/kernels.rs:99-152).
//
// Two passes over HBM-resident columns, no host scan:
//   1. filter_mask_kernel: every leaf of the predicate at once, one ballot
//      per 32 rows into a bit mask (n/8 bytes) and a count per 1024-row tile;
//   2. scan_u32_to_u64 of the tile counts (device-wide, decoupled from the
//      host), then one read of the total;
//   3. filter_gather_kernel: each warp compacts its 32-row words by popcount
//      ranks (stable) and writes every projected column and validity bitmap.
// The reference needs 3 + 2·columns launches and a host round trip per batch
// (crates/oxidelake-device/src/cuda/ops.rs:204-373); this needs 3 launches
// plus the scan.
#include "internal.h"

namespace oxb {

namespace {

constexpr int kTileRows = 1024;  // 32 mask words
constexpr int kWords = kTileRows / 32;
constexpr int kThreads = 256;    // 8 warps, 4 words each
constexpr int kMaxProj = 64;

struct DevProjCol {
    const void* src;
    const uint8_t* src_valid;
    void* dst;
    unsigned int* dst_valid;  // u32 words, zeroed; null when the column has no bitmap
    int width;
};
struct DevProjection {
    int ncols;
    DevProjCol cols[kMaxProj];
};

__global__ void __launch_bounds__(kThreads) filter_mask_kernel(const __grid_constant__ DevPredicate pred, long long n,
                                                               unsigned int* __restrict__ mask,
                                                               unsigned int* __restrict__ tile_counts,
                                                               long long ntiles) {
    __shared__ unsigned int warp_counts[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        unsigned int cnt = 0;
        // The warp's 4 words: row (word0 + j) * 32 + lane, every leaf's loads
        // for the 4 rows issued together.
        const long long word0 = tile * kWords + warp * 4;
        unsigned live = 0;
#pragma unroll
        for (int j = 0; j < 4; j++)
            if ((word0 + j) * 32 + lane < n) live |= 1u << j;
        const unsigned sel = predicate_mask<4>(pred, word0 * 32 + lane, 32, live);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const long long word = word0 + j;
            unsigned int bits = __ballot_sync(0xffffffffu, (sel >> j) & 1u);
            if (lane == 0 && word * 32 < n) mask[word] = bits;
            cnt += __popc(bits);
        }
        if (lane == 0) warp_counts[warp] = cnt;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned int t = 0;
#pragma unroll
            for (int w = 0; w < kThreads / 32; w++) t += warp_counts[w];
            tile_counts[tile] = t;
        }
        __syncthreads();
    }
}

// ORs `cnt` bits (bit i = output row base + i) into a zeroed u32 bitmap.
__device__ __forceinline__ void or_bits(unsigned int* words, unsigned long long base, unsigned int bits) {
    if (bits == 0) return;
    unsigned long long w = base >> 5;
    unsigned int sh = (unsigned int)(base & 31);
    unsigned int lo = bits << sh;
    if (lo) atomicOr(&words[w], lo);
    if (sh) {
        unsigned int hi = bits >> (32 - sh);
        if (hi) atomicOr(&words[w + 1], hi);
    }
}

__global__ void __launch_bounds__(kThreads, 5) filter_gather_kernel(
    const unsigned int* __restrict__ mask, const unsigned long long* __restrict__ tile_off, long long n,
    long long ntiles, const __grid_constant__ DevProjection proj) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long nwords = (n + 31) / 32;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        // Prefix of the tile's 32 words, then of this warp's 4.
        long long my_word = tile * kWords + lane;
        unsigned int wbits = my_word < nwords ? __ldg(mask + my_word) : 0u;
        unsigned int c = __popc(wbits), x = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        unsigned int excl = x - c;
        const unsigned long long toff = tile_off[tile];
        // The warp's 4 words: each narrow column's kept values are loaded for
        // all 4 words before any is stored, so 4 loads a lane are in flight.
        unsigned int wb[4];
        unsigned long long wbase[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            wb[j] = __shfl_sync(0xffffffffu, wbits, warp * 4 + j);
            wbase[j] = toff + __shfl_sync(0xffffffffu, excl, warp * 4 + j);
        }
        const unsigned int lt = lanemask_lt();
        for (int ci = 0; ci < proj.ncols; ci++) {
            const DevProjCol& col = proj.cols[ci];
            if (col.width == 8 || col.width == 4) {
                unsigned long long v[4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const long long row = (tile * kWords + warp * 4 + j) * 32 + lane;
                    v[j] = 0;
                    if ((wb[j] >> lane) & 1u)
                        v[j] = col.width == 8 ? __ldcs((const unsigned long long*)col.src + row)
                                              : (unsigned long long)__ldcs((const unsigned int*)col.src + row);
                }
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    if (!((wb[j] >> lane) & 1u)) continue;
                    const long long drow = (long long)(wbase[j] + __popc(wb[j] & lt));
                    if (col.width == 8) ((unsigned long long*)col.dst)[drow] = v[j];
                    else ((unsigned int*)col.dst)[drow] = (unsigned int)v[j];
                }
            }
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int wi = warp * 4 + j;
            unsigned int bits = wb[j];
            if (bits == 0) continue;  // uniform across the warp
            const long long row = (tile * kWords + wi) * 32 + lane;
            const bool sel = (bits >> lane) & 1u;
            const unsigned int rank = __popc(bits & lt);
            const unsigned long long base = wbase[j];
            for (int ci = 0; ci < proj.ncols; ci++) {
                const DevProjCol& col = proj.cols[ci];
                if (col.width <= 8) {
                    // narrow values were copied above
                } else {
                    // Wide rows: the warp copies one selected row at a time.
                    unsigned int m = bits;
                    const int words = col.width / 4;
                    while (m) {
                        int b = __ffs(m) - 1;
                        m &= m - 1;
                        long long srow = (tile * kWords + wi) * 32 + b;
                        long long drow = (long long)(base + __popc(bits & ((1u << b) - 1u)));
                        const unsigned int* s = (const unsigned int*)col.src + srow * words;
                        unsigned int* d = (unsigned int*)col.dst + drow * words;
                        for (int k = lane; k < words; k += 32) d[k] = __ldg(s + k);
                    }
                }
                if (col.dst_valid) {
                    bool v = sel && valid_at(col.src_valid, row);
                    unsigned int vb = __reduce_or_sync(0xffffffffu, v ? (1u << rank) : 0u);
                    if (lane == 0) or_bits(col.dst_valid, base, vb);
                }
            }
        }
    }
}

}  // namespace

DevPredicate make_predicate(const oxb_batch& in, const oxb_leaf* leaves, int nleaves) {
    if (nleaves < 0 || nleaves > kMaxLeaves)
        fail(OXB_UNSUPPORTED, "predicate has " + std::to_string(nleaves) + " leaves; at most 64 run on the device");
    if (nleaves > 0 && !leaves) fail(OXB_PLAN, "predicate leaves pointer is null");
    DevPredicate p{};
    p.nleaves = nleaves;
    for (int l = 0; l < nleaves; l++) {
        const oxb_leaf& lf = leaves[l];
        if (lf.column < 0 || lf.column >= (int)in.cols.size())
            fail(OXB_PLAN, "column index " + std::to_string(lf.column) + " out of range for a batch with " +
                               std::to_string(in.cols.size()) + " columns");
        const Column& c = in.cols[lf.column];
        if (c.type != lf.lit_type)
            fail(OXB_UNSUPPORTED, "column " + std::to_string(lf.column) + " has type " +
                                      std::to_string(c.type) + " but the literal is type " +
                                      std::to_string(lf.lit_type));
        if (c.type != kInt64 && c.type != kFloat64 && c.type != kInt32)
            fail(OXB_UNSUPPORTED, "predicate over a column of type " + std::to_string(c.type));
        if (lf.op < 0 || lf.op > 4) fail(OXB_PLAN, "unknown comparison " + std::to_string(lf.op));
        DevLeaf& d = p.leaves[l];
        d.values = c.values;
        d.validity = c.validity;
        d.type = c.type;
        d.op = lf.op;
        if (c.type == kFloat64) {
            long long bits;
            std::memcpy(&bits, &lf.lit.f, 8);
            if (bits == kEmptyKey) bits = 0;
            d.lit = bits ^ (long long)(((unsigned long long)(bits >> 63)) >> 1);
        } else {
            d.lit = lf.lit.i;
        }
    }
    return p;
}

oxb_batch* filter_project(const StreamRef& s, const Backend& b, const oxb_filter_project_args& a) {
    if (!a.input) fail(OXB_PLAN, "filter_project: input batch is null");
    const oxb_batch& in = *a.input;
    DevPredicate pred = make_predicate(in, a.leaves, a.nleaves);
    if (a.nprojection < 0 || a.nprojection > kMaxProj)
        fail(OXB_UNSUPPORTED, "projection of more than 64 columns");
    if (a.nprojection > 0 && !a.projection) fail(OXB_PLAN, "projection pointer is null");
    for (int i = 0; i < a.nprojection; i++)
        if (a.projection[i] < 0 || a.projection[i] >= (int)in.cols.size())
            fail(OXB_PLAN, "projection index " + std::to_string(a.projection[i]) + " out of range");

    const long long n = in.rows;
    const long long ntiles = (n + kTileRows - 1) / kTileRows;
    unsigned long long total = 0;
    Scratch<unsigned int> mask, tile_counts;
    Scratch<unsigned long long> tile_off;
    // Device time of the mask pass, its scan and the gather (the host's
    // read of the row count between them is not counted).
    KernelTimer timer(b, s, "filter_mask_kernel+filter_gather_kernel");
    if (n > 0) {
        mask = Scratch<unsigned int>(s, (n + 31) / 32);
        tile_counts = Scratch<unsigned int>(s, ntiles);
        tile_off = Scratch<unsigned long long>(s, ntiles + 1);
        int grid = grid_for(b, ntiles * kThreads, kThreads, 8);
        timer.begin();
        note_launch(), filter_mask_kernel<<<grid, kThreads, 0, s->stream>>>(pred, n, mask.get(), tile_counts.get(), ntiles);
        OXB_CUDA(cudaGetLastError());
        scan_u32_to_u64(s, b, tile_counts.get(), tile_off.get(), ntiles);
        timer.end();
        OXB_CUDA(cudaMemcpyAsync(&total, tile_off.get() + ntiles, sizeof total, cudaMemcpyDeviceToHost,
                                 s->stream));
        OXB_CUDA(cudaStreamSynchronize(s->stream));
    }

    auto out = std::make_unique<oxb_batch>();
    out->rows = (long long)total;
    DevProjection proj{};
    proj.ncols = a.nprojection;
    for (int i = 0; i < a.nprojection; i++) {
        const Column& src = in.cols[a.projection[i]];
        Column dst;
        dst.type = src.type;
        dst.dim = src.dim;
        dst.length = (long long)total;
        if (total > 0) {
            dst.owner_values = dev_alloc(s, total * (size_t)src.width(), false);
            dst.values = dst.owner_values->ptr;
            if (src.validity) {
                dst.owner_validity = dev_alloc(s, ((total + 31) / 32) * 4, true);
                dst.validity = (uint8_t*)dst.owner_validity->ptr;
            }
        }
        proj.cols[i] = DevProjCol{src.values, src.validity, dst.values, (unsigned int*)dst.validity,
                                  src.width()};
        out->cols.push_back(std::move(dst));
    }
    if (total > 0 && a.nprojection > 0) {
        int grid = grid_for(b, ntiles * kThreads, kThreads, 8);
        timer.begin();
        note_launch(), filter_gather_kernel<<<grid, kThreads, 0, s->stream>>>(mask.get(), tile_off.get(), n, ntiles, proj);
        timer.end();
        OXB_CUDA(cudaGetLastError());
    }
    return out.release();
}

// The rows a predicate keeps as a bitmap of u32 words (bit r of word w: row
// 32w + r), for operators that apply a WHERE inside their own kernels.
AllocRef predicate_bits(const StreamRef& s, const Backend& b, const DevPredicate& pred, long long n) {
    const long long ntiles = (n + kTileRows - 1) / kTileRows;
    AllocRef mask = dev_alloc(s, (size_t)(ntiles * kWords + 1) * 4, true);
    if (n > 0) {
        Scratch<unsigned int> tile_counts(s, ntiles);
        int grid = grid_for(b, ntiles * kThreads, kThreads, 8);
        note_launch(), filter_mask_kernel<<<grid, kThreads, 0, s->stream>>>(pred, n, (unsigned int*)mask->ptr,
                                                                          tile_counts.get(), ntiles);
        OXB_CUDA(cudaGetLastError());
    }
    return mask;
}

// ---- filter + projection into caller buffers, with static scratch ----------
//
// The same three steps as filter_project, but nothing is allocated: the
// mask, the tile counts, the tile offsets and the scan's block partials live
// in one file-scope device array sized for OXB_NOALLOC_MAX_ROWS input rows,
// and the output goes to buffers the caller owns.  Every scratch word that
// is read is written first by this call (the mask and tile counts for every
// tile of the input, the offsets and partials by the scan), so only the
// output validity bitmaps, which the gather ORs into, are cleared.  There is
// one array per device: calls whose work overlaps on one device race on it.

namespace {

constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr long long kNoAllocRows = OXB_NOALLOC_MAX_ROWS;
constexpr long long kNoAllocTiles = kNoAllocRows / kTileRows;
constexpr size_t kNaMaskOff = 0;
constexpr size_t kNaCountsOff = align256(kNaMaskOff + (size_t)kNoAllocRows / 32 * 4);
constexpr size_t kNaOffsOff = align256(kNaCountsOff + (size_t)kNoAllocTiles * 4);
constexpr size_t kNaPartialsOff = align256(kNaOffsOff + (size_t)(kNoAllocTiles + 1) * 8);
constexpr long long kNaPartials = 32;
constexpr size_t kNaScratchBytes = align256(kNaPartialsOff + (size_t)kNaPartials * 8);
static_assert(kNoAllocRows % kTileRows == 0, "the row limit is a whole number of tiles");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaScratchBytes];

constexpr int kMaxDevices = 64;

// The scratch array's address on `device` (the current device), looked up
// once per device.
unsigned char* noalloc_scratch(int device) {
    static std::mutex mu;
    static void* addr[kMaxDevices] = {};
    if (device < 0 || device >= kMaxDevices) fail(OXB_UNSUPPORTED, "device ordinal beyond 63");
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[device]) OXB_CUDA(cudaGetSymbolAddress(&addr[device], g_noalloc_scratch));
    return (unsigned char*)addr[device];
}

}  // namespace

void filter_project_noalloc(const StreamRef& s, const Backend& b, const oxb_filter_project_args& a,
                            void* const* out_values, uint32_t* const* out_validity, long long capacity,
                            long long* out_rows) {
    if (!a.input) fail(OXB_PLAN, "filter_project_noalloc: input batch is null");
    const oxb_batch& in = *a.input;
    DevPredicate pred = make_predicate(in, a.leaves, a.nleaves);
    if (a.nprojection < 0 || a.nprojection > kMaxProj)
        fail(OXB_UNSUPPORTED, "projection of more than 64 columns");
    if (a.nprojection > 0 && !a.projection) fail(OXB_PLAN, "projection pointer is null");
    for (int i = 0; i < a.nprojection; i++)
        if (a.projection[i] < 0 || a.projection[i] >= (int)in.cols.size())
            fail(OXB_PLAN, "projection index " + std::to_string(a.projection[i]) + " out of range");
    const long long n = in.rows;
    if (n > kNoAllocRows)
        fail(OXB_UNSUPPORTED, "filter_project_noalloc takes at most " + std::to_string(kNoAllocRows) +
                                  " input rows; the batch has " + std::to_string(n));
    if (capacity < 0) fail(OXB_PLAN, "negative output capacity");
    if (capacity > 0 && a.nprojection > 0 && !out_values) fail(OXB_PLAN, "output values array is null");
    for (int i = 0; i < a.nprojection && capacity > 0; i++) {
        const Column& src = in.cols[a.projection[i]];
        const size_t align = src.width() >= 8 ? 8 : 4;
        if (!out_values[i] || ((uintptr_t)out_values[i] % align))
            fail(OXB_PLAN, "output values buffer " + std::to_string(i) + " is null or not " +
                               std::to_string(align) + "-byte aligned");
        if (src.validity && (!out_validity || !out_validity[i] || ((uintptr_t)out_validity[i] & 3)))
            fail(OXB_PLAN, "projected column " + std::to_string(i) +
                               " has a validity bitmap: its output bitmap must be a 4-byte aligned buffer");
    }

    const long long ntiles = (n + kTileRows - 1) / kTileRows;
    unsigned long long total = 0;
    unsigned char* scratch = nullptr;
    if (n > 0) {
        scratch = noalloc_scratch(b.device);
        unsigned int* mask = (unsigned int*)(scratch + kNaMaskOff);
        unsigned int* tile_counts = (unsigned int*)(scratch + kNaCountsOff);
        unsigned long long* tile_off = (unsigned long long*)(scratch + kNaOffsOff);
        unsigned long long* partials = (unsigned long long*)(scratch + kNaPartialsOff);
        if (scan_partials_needed(ntiles) > kNaPartials) fail(OXB_EXECUTION, "scan partials exceed the static scratch");
        int grid = grid_for(b, ntiles * kThreads, kThreads, 8);
        note_launch(), filter_mask_kernel<<<grid, kThreads, 0, s->stream>>>(pred, n, mask, tile_counts, ntiles);
        OXB_CUDA(cudaGetLastError());
        scan_u32_to_u64_into(s, tile_counts, tile_off, ntiles, partials);
        OXB_CUDA(cudaMemcpyAsync(&total, tile_off + ntiles, sizeof total, cudaMemcpyDeviceToHost, s->stream));
        OXB_CUDA(cudaStreamSynchronize(s->stream));
    }
    if (out_rows) *out_rows = (long long)total;
    if ((long long)total > capacity)
        fail(OXB_EXECUTION, "the selection has " + std::to_string(total) + " rows but the output buffers hold " +
                                std::to_string(capacity));
    if (total == 0 || a.nprojection == 0) return;

    DevProjection proj{};
    proj.ncols = a.nprojection;
    for (int i = 0; i < a.nprojection; i++) {
        const Column& src = in.cols[a.projection[i]];
        unsigned int* dv = src.validity ? (unsigned int*)out_validity[i] : nullptr;
        if (dv) OXB_CUDA(cudaMemsetAsync(dv, 0, ((total + 31) / 32) * 4, s->stream));
        proj.cols[i] = DevProjCol{src.values, src.validity, out_values[i], dv, src.width()};
    }
    const unsigned int* mask = (const unsigned int*)(scratch + kNaMaskOff);
    const unsigned long long* tile_off = (const unsigned long long*)(scratch + kNaOffsOff);
    int grid = grid_for(b, ntiles * kThreads, kThreads, 8);
    note_launch(), filter_gather_kernel<<<grid, kThreads, 0, s->stream>>>(mask, tile_off, n, ntiles, proj);
    OXB_CUDA(cudaGetLastError());
}

}  // namespace oxb
