// Device-wide building blocks: exclusive scan of counts, a stable LSD radix
// sort of (key, value) pairs, and the range of an integer key column.
#include "internal.h"

namespace oxb {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanChunk = kScanThreads * kScanItems;  // counts per block

// Exclusive block scan of one u64 per thread; returns the block total in *total.
__device__ __forceinline__ unsigned long long block_exclusive_scan(unsigned long long v,
                                                                   unsigned long long* warp_sums,
                                                                   unsigned long long* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    const int nwarps = blockDim.x >> 5;
    if (warp == 0) {
        unsigned long long w = lane < nwarps ? warp_sums[lane] : 0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nwarps) warp_sums[lane] = w;  // inclusive
    }
    __syncthreads();
    unsigned long long before = warp > 0 ? warp_sums[warp - 1] : 0ull;
    *total = warp_sums[nwarps - 1];
    unsigned long long r = before + x - v;
    __syncthreads();
    return r;
}

__global__ void scan_reduce_kernel(const unsigned int* __restrict__ counts, long long n,
                                   unsigned long long* __restrict__ partials) {
    __shared__ unsigned long long warp_sums[32];
    long long base = (long long)blockIdx.x * kScanChunk;
    unsigned long long s = 0;
#pragma unroll 4
    for (int i = 0; i < kScanItems; i++) {
        long long idx = base + (long long)i * kScanThreads + threadIdx.x;
        if (idx < n) s += counts[idx];
    }
    unsigned long long total;
    block_exclusive_scan(s, warp_sums, &total);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

// A short scan (up to kSmallScan counts) in one launch: one block walks the
// counts a chunk at a time, carrying the running total, and stores it at [n].
constexpr long long kSmallScan = 2 * kScanChunk;
__global__ void scan_small_kernel(const unsigned int* __restrict__ counts, long long n,
                                  unsigned long long* __restrict__ offsets) {
    __shared__ unsigned long long warp_sums[32];
    unsigned long long carry = 0;
    for (long long base = 0; base < n; base += kScanChunk) {
        unsigned int c[kScanItems];
        unsigned long long s = 0;
#pragma unroll
        for (int i = 0; i < kScanItems; i++) {
            const long long idx = base + (long long)threadIdx.x * kScanItems + i;
            c[i] = idx < n ? counts[idx] : 0u;
            s += c[i];
        }
        unsigned long long total;
        unsigned long long run = carry + block_exclusive_scan(s, warp_sums, &total);
#pragma unroll
        for (int i = 0; i < kScanItems; i++) {
            const long long idx = base + (long long)threadIdx.x * kScanItems + i;
            if (idx < n) offsets[idx] = run;
            run += c[i];
        }
        carry += total;
    }
    if (threadIdx.x == 0) offsets[n] = carry;
}

// One block scans `m` partials in place (exclusive) and stores the total at [m].
__global__ void scan_partials_kernel(unsigned long long* __restrict__ p, long long m) {
    __shared__ unsigned long long warp_sums[32];
    long long per = (m + blockDim.x - 1) / blockDim.x;
    long long lo = (long long)threadIdx.x * per;
    long long hi = lo + per < m ? lo + per : m;
    unsigned long long s = 0;
    for (long long i = lo; i < hi; i++) s += p[i];
    unsigned long long total;
    unsigned long long run = block_exclusive_scan(s, warp_sums, &total);
    for (long long i = lo; i < hi; i++) {
        unsigned long long v = p[i];
        p[i] = run;
        run += v;
    }
    if (threadIdx.x == 0) p[m] = total;
}

// The offsets of one block's counts.  A thread scans 16 consecutive counts,
// so its 16 offsets are consecutive too; they are staged in shared memory
// (one u64 of padding every 16, so the lanes' rows fall in different banks)
// and stored by consecutive threads to consecutive addresses.  Stored
// straight from registers, each warp store touched 32 lines with 8 bytes
// apiece, and L2 filled the part-written sectors from DRAM.
constexpr int kScanPad = kScanChunk + kScanChunk / kScanItems;
__global__ void scan_apply_kernel(const unsigned int* __restrict__ counts, long long n,
                                  const unsigned long long* __restrict__ partials,
                                  unsigned long long* __restrict__ offsets) {
    __shared__ unsigned long long stage[kScanPad];  // the counts first (as u32), then the offsets
    __shared__ unsigned long long warp_sums[32];
    unsigned int* tile = (unsigned int*)stage;
    const long long base = (long long)blockIdx.x * kScanChunk;
    for (int i = threadIdx.x; i < kScanChunk; i += kScanThreads) {
        const long long idx = base + i;
        tile[i] = idx < n ? counts[idx] : 0u;
    }
    __syncthreads();
    unsigned int c[kScanItems];
    unsigned long long s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        c[i] = tile[threadIdx.x * kScanItems + i];
        s += c[i];
    }
    unsigned long long total;
    unsigned long long run = block_exclusive_scan(s, warp_sums, &total) + partials[blockIdx.x];  // ends synchronised
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        const int j = threadIdx.x * kScanItems + i;
        stage[j + j / kScanItems] = run;
        run += c[i];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        const int j = k * kScanThreads + threadIdx.x;
        const long long idx = base + j;
        if (idx < n) offsets[idx] = stage[j + j / kScanItems];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) offsets[n] = partials[gridDim.x];
}

// ---- radix sort ---------------------------------------------------------

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortRounds = 16;                                // items per lane
constexpr int kSortTile = kSortThreads * kSortRounds;          // 4096 items
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;

__global__ void radix_hist_kernel(const unsigned long long* __restrict__ keys, long long n, int shift,
                                  unsigned int* __restrict__ hist, long long ntiles) {
    __shared__ unsigned int h[kRadix];
    for (int i = threadIdx.x; i < kRadix; i += blockDim.x) h[i] = 0;
    __syncthreads();
    long long base = (long long)blockIdx.x * kSortTile;
    for (int i = threadIdx.x; i < kSortTile; i += blockDim.x) {
        long long idx = base + i;
        if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & (kRadix - 1)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) hist[(long long)d * ntiles + blockIdx.x] = h[d];
}

// Stable scatter: warp w owns items [w*32*R, (w+1)*32*R) of the tile, in
// rounds of 32 consecutive items; ranks follow tile order exactly.
__global__ void radix_scatter_kernel(const unsigned long long* __restrict__ keys_in,
                                     const unsigned int* __restrict__ vals_in, long long n, int shift,
                                     const unsigned long long* __restrict__ offsets, long long ntiles,
                                     unsigned long long* __restrict__ keys_out,
                                     unsigned int* __restrict__ vals_out) {
    __shared__ unsigned int wh[kSortWarps][kRadix];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kSortWarps * kRadix; i += blockDim.x) (&wh[0][0])[i] = 0;
    __syncthreads();
    const long long wbase = (long long)blockIdx.x * kSortTile + (long long)warp * 32 * kSortRounds;
    for (int r = 0; r < kSortRounds; r++) {
        long long idx = wbase + r * 32 + lane;
        unsigned d = idx < n ? (unsigned)((keys_in[idx] >> shift) & (kRadix - 1)) : kRadix;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        if (d < kRadix && lane == __ffs(peers) - 1) wh[warp][d] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) {
        unsigned long long run = offsets[(long long)d * ntiles + blockIdx.x];
        for (int w = 0; w < kSortWarps; w++) {
            unsigned c = wh[w][d];
            wh[w][d] = (unsigned)run;  // n < 2^32 is checked by the host
            run += c;
        }
    }
    __syncthreads();
    for (int r = 0; r < kSortRounds; r++) {
        long long idx = wbase + r * 32 + lane;
        unsigned long long k = idx < n ? keys_in[idx] : 0ull;
        unsigned d = idx < n ? (unsigned)((k >> shift) & (kRadix - 1)) : kRadix;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        if (d < kRadix) {
            unsigned pos = wh[warp][d] + __popc(peers & lanemask_lt());
            keys_out[pos] = k;
            if (vals_in) vals_out[pos] = vals_in[idx];
        }
        __syncwarp();
        if (d < kRadix && lane == __ffs(peers) - 1) wh[warp][d] += __popc(peers);
        __syncwarp();
    }
}

__global__ void key_range_kernel(const void* __restrict__ values, const uint8_t* __restrict__ validity,
                                 int type, long long n, long long* __restrict__ out /* lo, hi, count */) {
    long long lo = LLONG_MAX, hi = LLONG_MIN, cnt = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (!valid_at(validity, i)) continue;
        long long k = load_key(values, type, i);
        lo = k < lo ? k : lo;
        hi = k > hi ? k : hi;
        cnt++;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        long long a = __shfl_down_sync(0xffffffffu, lo, o);
        long long b = __shfl_down_sync(0xffffffffu, hi, o);
        long long c = __shfl_down_sync(0xffffffffu, cnt, o);
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
        cnt += c;
    }
    if ((threadIdx.x & 31) == 0 && cnt > 0) {
        atomicMin(&out[0], lo);
        atomicMax(&out[1], hi);
        atomicAdd((unsigned long long*)&out[2], (unsigned long long)cnt);
    }
}

__global__ void init_range_kernel(long long* out) {
    out[0] = LLONG_MAX;
    out[1] = LLONG_MIN;
    out[2] = 0;
}

}  // namespace

void scan_u32_to_u64(const StreamRef& s, const Backend& b, const unsigned int* counts,
                     unsigned long long* offsets, long long n) {
    (void)b;
    if (n <= 0) {
        OXB_CUDA(cudaMemsetAsync(offsets, 0, sizeof(unsigned long long), s->stream));
        return;
    }
    if (n <= kSmallScan) {
        note_launch(), scan_small_kernel<<<1, kScanThreads, 0, s->stream>>>(counts, n, offsets);
        OXB_CUDA(cudaGetLastError());
        return;
    }
    long long blocks = (n + kScanChunk - 1) / kScanChunk;
    Scratch<unsigned long long> partials(s, blocks + 1);
    note_launch(), scan_reduce_kernel<<<(unsigned)blocks, kScanThreads, 0, s->stream>>>(counts, n, partials.get());
    note_launch(), scan_partials_kernel<<<1, 1024, 0, s->stream>>>(partials.get(), blocks);
    note_launch(), scan_apply_kernel<<<(unsigned)blocks, kScanThreads, 0, s->stream>>>(counts, n, partials.get(),
                                                                        offsets);
    OXB_CUDA(cudaGetLastError());
}

long long scan_partials_needed(long long n) { return n <= 0 ? 1 : (n + kScanChunk - 1) / kScanChunk + 1; }

void scan_u32_to_u64_into(const StreamRef& s, const unsigned int* counts, unsigned long long* offsets, long long n,
                          unsigned long long* partials) {
    if (n <= 0) {
        OXB_CUDA(cudaMemsetAsync(offsets, 0, sizeof(unsigned long long), s->stream));
        return;
    }
    const long long blocks = (n + kScanChunk - 1) / kScanChunk;
    note_launch(), scan_reduce_kernel<<<(unsigned)blocks, kScanThreads, 0, s->stream>>>(counts, n, partials);
    note_launch(), scan_partials_kernel<<<1, 1024, 0, s->stream>>>(partials, blocks);
    note_launch(), scan_apply_kernel<<<(unsigned)blocks, kScanThreads, 0, s->stream>>>(counts, n, partials, offsets);
    OXB_CUDA(cudaGetLastError());
}

long long scan_block_rows() { return kScanChunk; }

void scan_u32_to_u64_from_totals(const StreamRef& s, const unsigned int* counts, unsigned long long* offsets,
                                 long long n, unsigned long long* partials) {
    if (n <= 0) {
        OXB_CUDA(cudaMemsetAsync(offsets, 0, sizeof(unsigned long long), s->stream));
        return;
    }
    const long long blocks = (n + kScanChunk - 1) / kScanChunk;
    note_launch(), scan_partials_kernel<<<1, 1024, 0, s->stream>>>(partials, blocks);
    note_launch(), scan_apply_kernel<<<(unsigned)blocks, kScanThreads, 0, s->stream>>>(counts, n, partials, offsets);
    OXB_CUDA(cudaGetLastError());
}

namespace {

constexpr int kOrderWords = 1024;  // presence bits for keys below 32768

__global__ void __launch_bounds__(1024) order_distinct_small_kernel(const unsigned long long* __restrict__ keys,
                                                                    const unsigned int* __restrict__ values, long long n,
                                                                    unsigned long long* __restrict__ keys_out,
                                                                    unsigned int* __restrict__ values_out) {
    __shared__ unsigned bits[kOrderWords];
    __shared__ unsigned long long before[kOrderWords];
    __shared__ unsigned long long warp_sums[32];
    for (int w = threadIdx.x; w < kOrderWords; w += blockDim.x) bits[w] = 0;
    __syncthreads();
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
        const unsigned d = (unsigned)keys[i];
        atomicOr(&bits[d >> 5], 1u << (d & 31));
    }
    __syncthreads();
    // one word a thread (blockDim.x == kOrderWords): keys present in earlier words
    unsigned long long total;
    before[threadIdx.x] = block_exclusive_scan((unsigned long long)__popc(bits[threadIdx.x]), warp_sums, &total);
    __syncthreads();
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
        const unsigned d = (unsigned)keys[i];
        const unsigned long long p = before[d >> 5] + __popc(bits[d >> 5] & ((1u << (d & 31)) - 1u));
        keys_out[p] = d;
        values_out[p] = values[i];
    }
}

__global__ void order_dense_flags_kernel(const unsigned long long* __restrict__ keys, long long n,
                                         unsigned int* __restrict__ present) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        present[keys[i]] = 1u;
}

__global__ void order_dense_place_kernel(const unsigned long long* __restrict__ keys,
                                         const unsigned int* __restrict__ values, long long n,
                                         const unsigned long long* __restrict__ pos,
                                         unsigned long long* __restrict__ keys_out, unsigned int* __restrict__ values_out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long d = keys[i];
        const unsigned long long p = pos[d];
        keys_out[p] = d;
        values_out[p] = values[i];
    }
}

}  // namespace

bool order_distinct_keys(const StreamRef& s, const Backend& b, const unsigned long long* keys,
                          const unsigned int* values, long long n, unsigned long long span,
                          unsigned long long* keys_out, unsigned int* values_out) {
    if (span < 32ull * kOrderWords) {
        if (n > 0) {
            note_launch(), order_distinct_small_kernel<<<1, kOrderWords, 0, s->stream>>>(keys, values, n, keys_out,
                                                                                         values_out);
            OXB_CUDA(cudaGetLastError());
        }
        return true;
    }
    // Keys that fill at least a quarter of their span (under 2^28): a key's
    // rank is the count of present offsets below it.
    if (span >= (1ull << 28) || (long long)span >= 4 * n + 4096) return false;
    const long long m = (long long)span + 1;
    Scratch<unsigned int> present(s, m, true);
    Scratch<unsigned long long> pos(s, m + 1);
    const int grid = grid_for(b, n, 256, 8);
    note_launch(), order_dense_flags_kernel<<<grid, 256, 0, s->stream>>>(keys, n, present.get());
    scan_u32_to_u64(s, b, present.get(), pos.get(), m);
    note_launch(), order_dense_place_kernel<<<grid, 256, 0, s->stream>>>(keys, values, n, pos.get(), keys_out,
                                                                        values_out);
    OXB_CUDA(cudaGetLastError());
    return true;
}

void radix_sort_pairs(const StreamRef& s, const Backend& b, unsigned long long* keys,
                      unsigned int* values, long long n, int bits) {
    if (n <= 1 || bits <= 0) return;
    if (n >= (1ll << 32)) fail(OXB_UNSUPPORTED, "radix sort of 2^32 or more items");
    long long ntiles = (n + kSortTile - 1) / kSortTile;
    Scratch<unsigned long long> k2(s, n);
    Scratch<unsigned int> v2(s, values ? n : 1);
    Scratch<unsigned int> hist(s, (size_t)kRadix * ntiles);
    Scratch<unsigned long long> offs(s, (size_t)kRadix * ntiles + 1);
    unsigned long long* kin = keys;
    unsigned long long* kout = k2.get();
    unsigned int* vin = values;
    unsigned int* vout = values ? v2.get() : nullptr;
    int passes = (bits + kRadixBits - 1) / kRadixBits;
    for (int p = 0; p < passes; p++) {
        int shift = p * kRadixBits;
        note_launch(), radix_hist_kernel<<<(unsigned)ntiles, kSortThreads, 0, s->stream>>>(kin, n, shift, hist.get(),
                                                                            ntiles);
        scan_u32_to_u64(s, b, hist.get(), offs.get(), (long long)kRadix * ntiles);
        note_launch(), radix_scatter_kernel<<<(unsigned)ntiles, kSortThreads, 0, s->stream>>>(
            kin, vin, n, shift, offs.get(), ntiles, kout, vout);
        OXB_CUDA(cudaGetLastError());
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    if (kin != keys) {
        OXB_CUDA(cudaMemcpyAsync(keys, kin, n * sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                                 s->stream));
        if (values)
            OXB_CUDA(cudaMemcpyAsync(values, vin, n * sizeof(unsigned int), cudaMemcpyDeviceToDevice,
                                     s->stream));
    }
}

bool key_range(const StreamRef& s, const Backend& b, const Column& key, long long n, long long* lo,
               long long* hi, long long* count) {
    Scratch<long long> out(s, 3);
    note_launch(), init_range_kernel<<<1, 1, 0, s->stream>>>(out.get());
    if (n > 0) {
        int grid = grid_for(b, n, 256, 4);
        note_launch(), key_range_kernel<<<grid, 256, 0, s->stream>>>(key.values, key.validity, key.type, n, out.get());
    }
    OXB_CUDA(cudaGetLastError());
    long long h[3];
    OXB_CUDA(cudaMemcpyAsync(h, out.get(), sizeof h, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaStreamSynchronize(s->stream));
    *lo = h[0];
    *hi = h[1];
    if (count) *count = h[2];
    return h[2] > 0;
}

}  // namespace oxb
