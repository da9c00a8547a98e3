// Inner hash join on one integer key: build once, probe per batch, gather
// output in ranges (GpuBackend::prepare_join_build / probe_join / hash_join,
// crates/oxidelake-device/src/backend.rs:114-163; semantics
// cpu/kernels.rs:185-472).
//
// The build side lives in one open-addressing table in HBM (16-byte slots
// {key, start, count}, load <= 1/2, so a 1M-key build is 32 MB and stays in
// the 126 MB L2 while the probe streams).  It is built on the device: from
// the caller's host index (the reference's JoinBuildArgs::index) or, with no
// index, from the key column itself by a stable radix sort, which yields the
// same runs in build order.  Matches are numbered in probe-row order, then
// build order (backend.rs:148-152).
#include "internal.h"

namespace oxb {

namespace {

__device__ __forceinline__ long long join_key_at(const void* v, int type, long long i) {
    return load_key(v, type, i);
}

// Places run r at its key's slot; a key equal to kEmptyKey goes to the side
// slot at index `capacity`.
__global__ void join_insert_kernel(JoinSlot* __restrict__ slots, unsigned int* __restrict__ first_row,
                                   unsigned int capacity, const long long* __restrict__ keys,
                                   const unsigned int* __restrict__ starts, const unsigned int* __restrict__ counts,
                                   long long nruns, const unsigned int* __restrict__ rows,
                                   unsigned int* __restrict__ status, const unsigned int* __restrict__ skip) {
    // A dense build that met a repeated key placed rows that are not runs:
    // nothing to insert (the host builds again by sorting).
    if (skip && *skip) return;
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nruns;
         r += (long long)gridDim.x * blockDim.x) {
        long long key = keys[r];
        if (key == kEmptyKey) {
            slots[capacity].start = starts[r];
            slots[capacity].count = counts[r];
            first_row[capacity] = rows[starts[r]];
            continue;
        }
        unsigned int s = (unsigned int)(fmix64((unsigned long long)key) & (capacity - 1u));
        bool placed = false;
        for (unsigned int p = 0; p < capacity; p++) {
            unsigned long long old = atomicCAS((unsigned long long*)&slots[s].key,
                                               (unsigned long long)kEmptyKey, (unsigned long long)key);
            if (old == (unsigned long long)kEmptyKey || old == (unsigned long long)key) {
                slots[s].start = starts[r];
                slots[s].count = counts[r];
                first_row[s] = rows[starts[r]];
                placed = true;
                break;
            }
            s = (s + 1u) & (capacity - 1u);
        }
        if (!placed) atomicOr(status, kStatusTableFull);
    }
}

__global__ void join_init_slots_kernel(JoinSlot* slots, unsigned int n) {
    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        slots[i].key = kEmptyKey;
        slots[i].start = 0;
        slots[i].count = 0;
    }
}

// Device build step 1: (key - lo, row) pairs; NULL keys sort after all others.
__global__ void join_pairs_kernel(const void* __restrict__ kv, const uint8_t* __restrict__ kvalid, int type,
                                  long long n, long long lo, unsigned long long null_key,
                                  unsigned long long* __restrict__ ukeys, unsigned int* __restrict__ rows) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        ukeys[i] = valid_at(kvalid, i) ? (unsigned long long)(join_key_at(kv, type, i) - lo) : null_key;
        rows[i] = (unsigned int)i;
    }
}

// Dense build, step 1: rows per key offset (key - lo) of the valid keys; a
// key seen twice raises *dup (the sorted build then runs instead).
__global__ void join_dense_count_kernel(const void* __restrict__ kv, const uint8_t* __restrict__ kvalid, int type,
                                        long long n, long long lo, unsigned int* __restrict__ cnt,
                                        unsigned int* __restrict__ dup) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (!valid_at(kvalid, i)) continue;
        const unsigned long long d = (unsigned long long)(join_key_at(kv, type, i) - lo);
        if (atomicAdd(&cnt[d], 1u) != 0u) *dup = 1u;
    }
}

// Dense build, step 2 (every key unique): a valid row's position in key
// order is the count of smaller keys, pos[key - lo]; it is its own run.
__global__ void join_dense_place_kernel(const void* __restrict__ kv, const uint8_t* __restrict__ kvalid, int type,
                                        long long n, long long lo, const unsigned long long* __restrict__ pos,
                                        unsigned int* __restrict__ rows, long long* __restrict__ rkeys,
                                        unsigned int* __restrict__ rstart, unsigned int* __restrict__ rcount) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (!valid_at(kvalid, i)) continue;
        const long long key = join_key_at(kv, type, i);
        const unsigned long long p = pos[(unsigned long long)(key - lo)];
        rows[p] = (unsigned int)i;
        rkeys[p] = key;
        rstart[p] = (unsigned int)p;
        rcount[p] = 1u;
    }
}

// Dense build, step 3: the direct index of the probe, the run start of each
// key offset (its position in key order) or kNoRun where no row has it.
__global__ void join_dense_index_kernel(const unsigned int* __restrict__ cnt, const unsigned long long* __restrict__ pos,
                                        long long m, unsigned int* __restrict__ index) {
    for (long long d = blockIdx.x * (long long)blockDim.x + threadIdx.x; d < m; d += (long long)gridDim.x * blockDim.x)
        index[d] = cnt[d] ? (unsigned int)pos[d] : kNoRun;
}

// Device build step 2: 1 where a run of equal keys starts.
__global__ void join_heads_kernel(const unsigned long long* __restrict__ ukeys, long long nvalid,
                                  unsigned int* __restrict__ heads) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvalid;
         i += (long long)gridDim.x * blockDim.x)
        heads[i] = (i == 0 || ukeys[i] != ukeys[i - 1]) ? 1u : 0u;
}

// Device build step 3: each run's key and start; step 4: its count, from
// the start of the next run.
__global__ void join_runs_kernel(const unsigned long long* __restrict__ ukeys, long long nvalid,
                                 const unsigned int* __restrict__ heads,
                                 const unsigned long long* __restrict__ run_of, long long lo,
                                 long long* __restrict__ rkeys, unsigned int* __restrict__ rstart) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvalid;
         i += (long long)gridDim.x * blockDim.x) {
        if (!heads[i]) continue;
        long long r = (long long)run_of[i];
        rkeys[r] = (long long)(ukeys[i] + (unsigned long long)lo);
        rstart[r] = (unsigned int)i;
    }
}

__global__ void join_counts_kernel(const unsigned int* __restrict__ rstart, long long nruns, long long nvalid,
                                   unsigned int* __restrict__ rcount) {
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nruns;
         r += (long long)gridDim.x * blockDim.x) {
        long long end = r + 1 < nruns ? (long long)rstart[r + 1] : nvalid;
        rcount[r] = (unsigned int)(end - (long long)rstart[r]);
    }
}

__device__ __forceinline__ bool join_lookup(const JoinTableDev& t, long long key, unsigned int* start,
                                            unsigned int* count) {
    if (key == kEmptyKey) {
        *start = t.special_start;
        *count = t.special_count;
        return *count > 0;
    }
    if (t.dense) {  // unique keys filling their range: one 4-byte read
        const unsigned long long d = (unsigned long long)key - (unsigned long long)t.dense_lo;
        if (d >= t.dense_n) return false;
        const unsigned int v = __ldg(t.dense + d);
        if (v == kNoRun) return false;
        *start = v;
        *count = 1u;
        return true;
    }
    unsigned int s = (unsigned int)(fmix64((unsigned long long)key) & (t.capacity - 1u));
    for (unsigned int p = 0; p < t.capacity; p++) {
        const int4 slot = __ldg((const int4*)&t.slots[s]);
        long long k = ((long long)(unsigned int)slot.y << 32) | (unsigned int)slot.x;
        if (k == key) {
            *start = (unsigned int)slot.z;
            *count = (unsigned int)slot.w;
            return true;
        }
        if (k == kEmptyKey) return false;
        s = (s + 1u) & (t.capacity - 1u);
    }
    return false;
}

// The probe writes each row's match count and first build row, and each
// block of scan_block_rows() rows its total, so the offsets' scan needs no
// reduce pass of its own.
constexpr int kProbeThreads = 256;

// Compiled for the key's type (KT: kInt64 or kInt32) and for a table with a
// direct index (DENSE), so a row's lookup carries no switch on either.
template <int KT, bool DENSE>
__device__ __forceinline__ bool probe_lookup(const JoinTableDev& t, long long key, unsigned int* start,
                                             unsigned int* count) {
    if (DENSE && key != kEmptyKey) {
        const unsigned long long d = (unsigned long long)key - (unsigned long long)t.dense_lo;
        const unsigned int v = d < t.dense_n ? __ldg(t.dense + d) : kNoRun;
        *start = v;
        *count = v != kNoRun ? 1u : 0u;
        return v != kNoRun;
    }
    return join_lookup(t, key, start, count);
}

template <int KT, bool DENSE>
__global__ void __launch_bounds__(kProbeThreads) join_probe_kernel(
    const __grid_constant__ JoinTableDev t, const void* __restrict__ kv, const uint8_t* __restrict__ kvalid,
    long long n, long long block_rows, unsigned int* __restrict__ counts, unsigned int* __restrict__ starts,
    unsigned long long* __restrict__ totals) {
    __shared__ unsigned long long warp_sums[kProbeThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long nblocks = (n + block_rows - 1) / block_rows;
    for (long long blk = blockIdx.x; blk < nblocks; blk += gridDim.x) {
        const long long end = (blk + 1) * block_rows < n ? (blk + 1) * block_rows : n;
        unsigned long long sum = 0;
        for (long long i0 = blk * block_rows; i0 < end; i0 += 4 * kProbeThreads) {
            // four rows a thread: their keys, then their lookups, in flight together
            long long key[4];
            bool live[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const long long i = i0 + k * kProbeThreads + threadIdx.x;
                live[k] = i < end && valid_at(kvalid, i);
                key[k] = !live[k] ? 0 : KT == kInt64 ? __ldg((const long long*)kv + i) : (long long)__ldg((const int*)kv + i);
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const long long i = i0 + k * kProbeThreads + threadIdx.x;
                if (i >= end) continue;
                unsigned int st = 0, c = 0;
                if (live[k] && !probe_lookup<KT, DENSE>(t, key[k], &st, &c)) st = c = 0;
                counts[i] = c;
                starts[i] = st;
                sum += c;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (lane == 0) warp_sums[warp] = sum;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long tot = 0;
#pragma unroll
            for (int w = 0; w < kProbeThreads / 32; w++) tot += warp_sums[w];
            totals[blk] = tot;
        }
        __syncthreads();
    }
}

constexpr int kMaxOut = 128;
struct DevGatherCol {
    const void* src;
    const uint8_t* src_valid;
    void* dst;
    unsigned int* dst_valid;
    int width;
    int side;  // 0 = left (probe), 1 = right (build)
};
struct DevGather {
    int ncols;
    DevGatherCol cols[kMaxOut];
};

// The probe row holding match p is the last one whose offset is <= p
// (cpu/kernels.rs:378-384).  Output rows are cut into kGatherTile-row
// tiles; join_tile_rows_kernel finds the probe row of each tile's first
// output by one binary search over the whole offsets array, and the gather
// then searches only its tile's rows: in shared memory when their offsets
// fit (kGatherRegion rows, the case whenever at least one probe row in two
// matches), else in HBM over that range.
constexpr int kGatherTile = 2048;
constexpr int kGatherThreads = 256;
constexpr int kGatherRegion = 4096;

// offsets[lo] <= p < offsets[hi] on entry; the last i in [lo, hi) with
// offsets[i] <= p.
__device__ __forceinline__ long long last_at_or_below(const unsigned long long* offsets, long long lo, long long hi,
                                                     unsigned long long p) {
    while (hi - lo > 1) {
        const long long mid = lo + (hi - lo) / 2;
        if (offsets[mid] <= p) lo = mid;
        else hi = mid;
    }
    return lo;
}

// tile_row[k] = the probe row of output min(k * kGatherTile, rows - 1), for
// k in [0, ntiles]: tile k's outputs come from probe rows tile_row[k] ..
// tile_row[k + 1].
__global__ void join_tile_rows_kernel(const unsigned long long* __restrict__ offsets, long long nprobe,
                                      unsigned long long first, long long rows, long long ntiles,
                                      long long* __restrict__ tile_row) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k <= ntiles;
         k += (long long)gridDim.x * blockDim.x) {
        const long long t = k * kGatherTile < rows ? k * kGatherTile : rows - 1;
        tile_row[k] = last_at_or_below(offsets, 0, nprobe, first + (unsigned long long)t);
    }
}

__global__ void __launch_bounds__(kGatherThreads, 4) join_gather_kernel(
    const unsigned long long* __restrict__ offsets, const unsigned int* __restrict__ starts,
    const long long* __restrict__ tile_row, long long ntiles, const unsigned int* __restrict__ trows,
    long long ntrows, long long right_rows, unsigned long long first, long long rows,
    const __grid_constant__ DevGather g, unsigned int* __restrict__ status) {
    __shared__ unsigned long long offs[kGatherRegion + 1];
    __shared__ unsigned short out_row[kGatherTile];  // each output's probe row, less r0
    const int lane = threadIdx.x & 31;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long r0 = tile_row[tile], r1 = tile_row[tile + 1];
        const long long span = r1 - r0 + 2;  // offsets[r0 .. r1 + 1]
        const bool local = span <= kGatherRegion + 1;
        __syncthreads();  // the previous tile's outputs are done with offs and out_row
        if (local)
            for (long long i = threadIdx.x; i < span; i += blockDim.x) offs[i] = offsets[r0 + i];
        __syncthreads();
        const long long t0 = tile * kGatherTile;
        if (local) {
            // Each probe row of the tile marks its outputs' slots with its
            // index, so an output finds its row with one shared read instead
            // of a binary search.
            const unsigned long long tlo = first + (unsigned long long)t0;
            const unsigned long long thi = tlo + kGatherTile;
            for (long long i = threadIdx.x; i < span - 1; i += blockDim.x) {
                const unsigned long long a = offs[i] > tlo ? offs[i] : tlo;
                const unsigned long long e = offs[i + 1] < thi ? offs[i + 1] : thi;
                for (unsigned long long q = a; q < e; q++) out_row[q - tlo] = (unsigned short)i;
            }
            __syncthreads();
        }
        constexpr int R = kGatherTile / kGatherThreads;
        // Each output's probe and build rows first, all R of a thread's
        // outputs, then every column's R values loaded before any is stored.
        unsigned int lr[R], rr[R];
#pragma unroll
        for (int k = 0; k < R; k++) {
            const long long t = t0 + k * kGatherThreads + threadIdx.x;
            lr[k] = rr[k] = 0;
            if (t >= rows) continue;
            const unsigned long long p = first + (unsigned long long)t;
            long long lrow;
            unsigned long long base;
            if (local) {  // offs[0] <= p < offs[span - 1]
                const int lo = out_row[t - t0];
                lrow = r0 + lo;
                base = offs[lo];
            } else {
                lrow = last_at_or_below(offsets, r0, r1 + 1, p);
                base = offsets[lrow];
            }
            lr[k] = (unsigned int)lrow;
            const unsigned long long at = (unsigned long long)starts[lrow] + (p - base);
            if (at < (unsigned long long)ntrows) {
                const unsigned int rrow = trows[at];
                if (rrow >= right_rows) atomicOr(status, kStatusBounds);
                else rr[k] = rrow;
            } else {
                atomicOr(status, kStatusBounds);
            }
        }
        for (int ci = 0; ci < g.ncols; ci++) {
            const DevGatherCol& c = g.cols[ci];
            const DevGatherCol& c2 = g.cols[ci + 1 < g.ncols ? ci + 1 : ci];
            const bool narrow = c.width == 8 || c.width == 4;
            if (narrow && ci + 1 < g.ncols && (c2.width == 8 || c2.width == 4) && !c.dst_valid && !c2.dst_valid) {
                // Two narrow columns without bitmaps: both columns' values in
                // flight before either is stored.
                unsigned long long v[R], w[R];
#pragma unroll
                for (int k = 0; k < R; k++) {
                    const long long t = t0 + k * kGatherThreads + threadIdx.x;
                    const long long s1 = c.side == 0 ? lr[k] : rr[k], s2 = c2.side == 0 ? lr[k] : rr[k];
                    v[k] = t >= rows ? 0ull
                           : c.width == 8 ? __ldg((const unsigned long long*)c.src + s1)
                                          : (unsigned long long)__ldg((const unsigned int*)c.src + s1);
                    w[k] = t >= rows ? 0ull
                           : c2.width == 8 ? __ldg((const unsigned long long*)c2.src + s2)
                                           : (unsigned long long)__ldg((const unsigned int*)c2.src + s2);
                }
#pragma unroll
                for (int k = 0; k < R; k++) {
                    const long long t = t0 + k * kGatherThreads + threadIdx.x;
                    if (t >= rows) continue;
                    if (c.width == 8) ((unsigned long long*)c.dst)[t] = v[k];
                    else ((unsigned int*)c.dst)[t] = (unsigned int)v[k];
                    if (c2.width == 8) ((unsigned long long*)c2.dst)[t] = w[k];
                    else ((unsigned int*)c2.dst)[t] = (unsigned int)w[k];
                }
                ci++;
                continue;
            }
            if (narrow) {
                unsigned long long v[R];
#pragma unroll
                for (int k = 0; k < R; k++) {
                    const long long t = t0 + k * kGatherThreads + threadIdx.x;
                    const long long srow = c.side == 0 ? lr[k] : rr[k];
                    v[k] = t >= rows ? 0ull
                           : c.width == 8 ? __ldg((const unsigned long long*)c.src + srow)
                                          : (unsigned long long)__ldg((const unsigned int*)c.src + srow);
                }
#pragma unroll
                for (int k = 0; k < R; k++) {
                    const long long t = t0 + k * kGatherThreads + threadIdx.x;
                    if (t >= rows) continue;
                    if (c.width == 8) ((unsigned long long*)c.dst)[t] = v[k];
                    else ((unsigned int*)c.dst)[t] = (unsigned int)v[k];
                }
            } else {
#pragma unroll
                for (int k = 0; k < R; k++) {
                    const long long t = t0 + k * kGatherThreads + threadIdx.x;
                    if (t >= rows) continue;
                    const long long srow = c.side == 0 ? lr[k] : rr[k];
                    const int w = c.width / 4;
                    const unsigned int* src = (const unsigned int*)c.src + srow * w;
                    unsigned int* d = (unsigned int*)c.dst + t * w;
                    for (int q = 0; q < w; q++) d[q] = __ldg(src + q);
                }
            }
            if (c.dst_valid) {
#pragma unroll
                for (int k = 0; k < R; k++) {
                    const long long t = t0 + k * kGatherThreads + threadIdx.x;
                    const long long srow = c.side == 0 ? lr[k] : rr[k];
                    const unsigned int bits = __ballot_sync(0xffffffffu, t < rows && valid_at(c.src_valid, srow));
                    if (lane == 0 && t < rows) c.dst_valid[t >> 5] = bits;
                }
            }
        }
    }
}

unsigned int pow2_capacity(long long distinct) {
    long long c = 16;
    while (c < 2 * distinct) c <<= 1;
    if (c > (1ll << 31)) fail(OXB_UNSUPPORTED, std::to_string(distinct) + " distinct join keys exceed the device index");
    return (unsigned int)c;
}

}  // namespace

namespace {

// try_dense: place dense unique keys by key offset; returns null when a key
// repeats (found at the status read), and the caller builds again sorted.
oxb_join_table* prepare_join_build_impl(const StreamRef& s, const Backend& b, const oxb_join_build_args& a,
                                        bool try_dense) {
    if (!a.build) fail(OXB_PLAN, "prepare_join_build: build batch is null");
    const oxb_batch& build = *a.build;
    if (a.key < 0 || a.key >= (int)build.cols.size())
        fail(OXB_PLAN, "join key column " + std::to_string(a.key) + " out of range");
    const Column& key = build.cols[a.key];
    if (key.type != kInt64 && key.type != kInt32)
        fail(OXB_UNSUPPORTED, "build join key column has type " + std::to_string(key.type) + "; Int64 and Int32 run on the device");
    const long long n = build.rows;
    if (n >= (1ll << 32)) fail(OXB_EXECUTION, "build side exceeds u32::MAX rows");

    auto out = std::make_unique<oxb_join_table>();
    out->build = a.build;
    out->build_rows = n;
    JoinTableDev& t = out->t;
    t.key_type = key.type;
    Scratch<unsigned int> status(s, 1, true);

    Scratch<long long> rkeys;
    Scratch<unsigned int> rstart, rcount;
    Scratch<unsigned int> dup;  // the dense build's repeated-key flag
    long long nruns = 0;

    if (a.index) {
        // The host's index (JoinSlots::build checks, join_slots.rs:64-95).
        const oxb_join_index& ix = *a.index;
        if (ix.ndistinct < 0 || ix.nrows < 0) fail(OXB_EXECUTION, "negative join index sizes");
        for (long long i = 0; i < ix.nrows; i++)
            if (ix.rows[i] >= (unsigned long long)n)
                fail(OXB_EXECUTION, "join table row " + std::to_string(ix.rows[i]) + " is out of range for a " +
                                        std::to_string(n) + "-row build side");
        for (long long r = 0; r < ix.ndistinct; r++) {
            unsigned long long end = (unsigned long long)ix.starts[r] + ix.counts[r];
            if (ix.counts[r] == 0 || end > (unsigned long long)ix.nrows)
                fail(OXB_EXECUTION, "join table run " + std::to_string(ix.starts[r]) + "+" +
                                        std::to_string(ix.counts[r]) + " is outside its " +
                                        std::to_string(ix.nrows) + " rows");
        }
        nruns = ix.ndistinct;
        t.nrows = ix.nrows;
        out->rows_mem = dev_alloc(s, (size_t)(ix.nrows + 1) * 4, false);
        t.rows = (unsigned int*)out->rows_mem->ptr;
        if (ix.nrows > 0)
            OXB_CUDA(cudaMemcpyAsync(t.rows, ix.rows, ix.nrows * 4, cudaMemcpyHostToDevice, s->stream));
        if (nruns > 0) {
            rkeys = Scratch<long long>(s, nruns);
            rstart = Scratch<unsigned int>(s, nruns);
            rcount = Scratch<unsigned int>(s, nruns);
            OXB_CUDA(cudaMemcpyAsync(rkeys.get(), ix.keys, nruns * 8, cudaMemcpyHostToDevice, s->stream));
            OXB_CUDA(cudaMemcpyAsync(rstart.get(), ix.starts, nruns * 4, cudaMemcpyHostToDevice, s->stream));
            OXB_CUDA(cudaMemcpyAsync(rcount.get(), ix.counts, nruns * 4, cudaMemcpyHostToDevice, s->stream));
            // The side slot is filled on the host for the kEmptyKey run.
            for (long long r = 0; r < nruns; r++) {
                if (ix.keys[r] == kEmptyKey) {
                    t.special_start = ix.starts[r];
                    t.special_count = ix.counts[r];
                    continue;
                }
                if (t.key_lo > t.key_hi) t.key_lo = t.key_hi = ix.keys[r];
                t.key_lo = std::min(t.key_lo, (long long)ix.keys[r]);
                t.key_hi = std::max(t.key_hi, (long long)ix.keys[r]);
            }
        }
    } else {
        // Device build: stable sort of (key, row) by key keeps build order.
        long long lo = 0, hi = 0, nvalid = 0;
        bool any = key_range(s, b, key, n, &lo, &hi, &nvalid);
        if (any) {
            // kEmptyKey lives in the side slot: the placed range starts above it.
            t.key_lo = lo == kEmptyKey ? lo + 1 : lo;
            t.key_hi = hi;
        }
        // Keys that fill at least a quarter of their range (and stay under
        // 2^26 offsets): when every key is unique, counting the rows per key
        // offset and scanning the counts places each row at its position in
        // key order, the order the sort below gives, without the sort.
        bool placed = false;
        const unsigned long long dspan = (unsigned long long)hi - (unsigned long long)lo;
        // Placed optimistically: a repeated key, seen by the count, stops the
        // insert and is read with the status at the end.
        if (try_dense && any && lo != kEmptyKey && dspan < (1ull << 26) && (long long)dspan < 4 * nvalid + 4096) {
            const long long m = (long long)dspan + 1;
            Scratch<unsigned int> cnt(s, m, true);
            dup = Scratch<unsigned int>(s, 1, true);
            const int grid = grid_for(b, n, 256, 8);
            note_launch(), join_dense_count_kernel<<<grid, 256, 0, s->stream>>>(key.values, key.validity, key.type, n, lo,
                                                                               cnt.get(), dup.get());
            OXB_CUDA(cudaGetLastError());
            {
                Scratch<unsigned long long> pos(s, m + 1);
                scan_u32_to_u64(s, b, cnt.get(), pos.get(), m);
                nruns = nvalid;
                rkeys = Scratch<long long>(s, nruns);
                rstart = Scratch<unsigned int>(s, nruns);
                rcount = Scratch<unsigned int>(s, nruns);
                t.nrows = nvalid;
                out->rows_mem = dev_alloc(s, (size_t)(nvalid + 1) * 4, false);
                t.rows = (unsigned int*)out->rows_mem->ptr;
                note_launch(), join_dense_place_kernel<<<grid, 256, 0, s->stream>>>(
                    key.values, key.validity, key.type, n, lo, pos.get(), t.rows, rkeys.get(), rstart.get(),
                    rcount.get());
                out->dense_mem = dev_alloc(s, (size_t)m * 4, false);
                note_launch(), join_dense_index_kernel<<<grid_for(b, m, 256, 8), 256, 0, s->stream>>>(
                    cnt.get(), pos.get(), m, (unsigned int*)out->dense_mem->ptr);
                OXB_CUDA(cudaGetLastError());
                t.dense = (const unsigned int*)out->dense_mem->ptr;
                t.dense_lo = lo;
                t.dense_n = (unsigned long long)m;
                placed = true;
            }
        }
        Scratch<unsigned long long> ukeys;
        Scratch<unsigned int> srows;
        if (any && !placed) {
            unsigned long long span = (unsigned long long)hi - (unsigned long long)lo;
            unsigned long long null_key = span + 1;  // wraps to 0 only for the full i64 range
            int bits = 64;
            if (null_key != 0) {
                bits = 0;
                while (bits < 64 && (null_key >> bits) != 0) bits++;
            }
            ukeys = Scratch<unsigned long long>(s, n);
            srows = Scratch<unsigned int>(s, n);
            int grid = grid_for(b, n, 256, 8);
            note_launch(), join_pairs_kernel<<<grid, 256, 0, s->stream>>>(key.values, key.validity, key.type, n, lo,
                                                            null_key == 0 ? ~0ull : null_key, ukeys.get(), srows.get());
            OXB_CUDA(cudaGetLastError());
            radix_sort_pairs(s, b, ukeys.get(), srows.get(), n, bits);
        }
        if (!placed) {
            t.nrows = nvalid;
            out->rows_mem = dev_alloc(s, (size_t)(nvalid + 1) * 4, false);
            t.rows = (unsigned int*)out->rows_mem->ptr;
        }
        if (nvalid > 0 && !placed) {
            OXB_CUDA(cudaMemcpyAsync(t.rows, srows.get(), nvalid * 4, cudaMemcpyDeviceToDevice, s->stream));
            Scratch<unsigned int> heads(s, nvalid);
            Scratch<unsigned long long> run_of(s, nvalid + 1);
            int grid = grid_for(b, nvalid, 256, 8);
            note_launch(), join_heads_kernel<<<grid, 256, 0, s->stream>>>(ukeys.get(), nvalid, heads.get());
            scan_u32_to_u64(s, b, heads.get(), run_of.get(), nvalid);
            unsigned long long nr = 0;
            OXB_CUDA(cudaMemcpyAsync(&nr, run_of.get() + nvalid, 8, cudaMemcpyDeviceToHost, s->stream));
            OXB_CUDA(cudaStreamSynchronize(s->stream));
            nruns = (long long)nr;
            rkeys = Scratch<long long>(s, nruns);
            rstart = Scratch<unsigned int>(s, nruns);
            rcount = Scratch<unsigned int>(s, nruns);
            note_launch(), join_runs_kernel<<<grid, 256, 0, s->stream>>>(ukeys.get(), nvalid, heads.get(), run_of.get(), lo,
                                                           rkeys.get(), rstart.get());
            note_launch(), join_counts_kernel<<<grid_for(b, nruns, 256, 8), 256, 0, s->stream>>>(rstart.get(), nruns, nvalid,
                                                                                  rcount.get());
            OXB_CUDA(cudaGetLastError());
            if (lo == kEmptyKey) {
                // The smallest key sorts first: run 0; the smallest placed key
                // is run 1's.
                unsigned int c = 0;
                long long next = 0;
                OXB_CUDA(cudaMemcpyAsync(&c, rcount.get(), 4, cudaMemcpyDeviceToHost, s->stream));
                if (nruns > 1)
                    OXB_CUDA(cudaMemcpyAsync(&next, rkeys.get() + 1, 8, cudaMemcpyDeviceToHost, s->stream));
                OXB_CUDA(cudaStreamSynchronize(s->stream));
                t.special_start = 0;
                t.special_count = c;
                if (nruns > 1) t.key_lo = next;
            }
        }
    }

    t.ndistinct = nruns;
    t.capacity = pow2_capacity(nruns);
    out->slots_mem = dev_alloc(s, (size_t)(t.capacity + 1) * (sizeof(JoinSlot) + 4), false);
    t.slots = (JoinSlot*)out->slots_mem->ptr;
    t.first_row = (unsigned int*)(t.slots + t.capacity + 1);
    note_launch(), join_init_slots_kernel<<<grid_for(b, t.capacity + 1, 256, 8), 256, 0, s->stream>>>(t.slots, t.capacity + 1);
    if (nruns > 0)
        note_launch(), join_insert_kernel<<<grid_for(b, nruns, 256, 8), 256, 0, s->stream>>>(
            t.slots, t.first_row, t.capacity, rkeys.get(), rstart.get(), rcount.get(), nruns, t.rows, status.get(),
            dup.get());
    OXB_CUDA(cudaGetLastError());
    uint32_t st = 0, hdup = 0;
    OXB_CUDA(cudaMemcpyAsync(&st, status.get(), 4, cudaMemcpyDeviceToHost, s->stream));
    if (dup.get()) OXB_CUDA(cudaMemcpyAsync(&hdup, dup.get(), 4, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaStreamSynchronize(s->stream));
    if (hdup) return nullptr;
    check_status_word(st, "prepare_join_build");
    return out.release();
}

}  // namespace

oxb_join_table* prepare_join_build(const StreamRef& s, const Backend& b, const oxb_join_build_args& a) {
    oxb_join_table* t = prepare_join_build_impl(s, b, a, true);
    return t ? t : prepare_join_build_impl(s, b, a, false);
}

oxb_join_matches* probe_join(const StreamRef& s, const Backend& b, const oxb_join_probe_args& a) {
    if (!a.probe || !a.table) fail(OXB_PLAN, "probe_join: null probe or table");
    const oxb_batch& probe = *a.probe;
    if (a.key < 0 || a.key >= (int)probe.cols.size())
        fail(OXB_PLAN, "probe key column " + std::to_string(a.key) + " out of range");
    const Column& key = probe.cols[a.key];
    if (key.type != kInt64 && key.type != kInt32)
        fail(OXB_UNSUPPORTED, "probe join key column has type " + std::to_string(key.type));
    const long long n = probe.rows;
    if (n >= (1ll << 32)) fail(OXB_EXECUTION, "batch exceeds u32::MAX rows");
    auto m = std::make_unique<oxb_join_matches>();
    m->table = a.table;
    m->probe_rows = n;
    m->offsets_mem = dev_alloc(s, (size_t)(n + 1) * 8, false);
    m->starts_mem = dev_alloc(s, (size_t)(n + 1) * 4, false);
    auto* offsets = (unsigned long long*)m->offsets_mem->ptr;
    auto* starts = (unsigned int*)m->starts_mem->ptr;
    if (n > 0) {
        const long long block_rows = scan_block_rows();
        const long long nblocks = (n + block_rows - 1) / block_rows;
        Scratch<unsigned int> counts(s, n);
        Scratch<unsigned long long> totals(s, nblocks + 1);
        KernelTimer timer(b, s, "join_probe_kernel+scan");  // the probe and its offsets' scan
        timer.begin();
        const bool dense = a.table->t.dense != nullptr;
        auto probe = key.type == kInt64 ? (dense ? join_probe_kernel<kInt64, true> : join_probe_kernel<kInt64, false>)
                                        : (dense ? join_probe_kernel<kInt32, true> : join_probe_kernel<kInt32, false>);
        note_launch(), probe<<<grid_for(b, nblocks * kProbeThreads, kProbeThreads, 8), kProbeThreads, 0, s->stream>>>(
            a.table->t, key.values, key.validity, n, block_rows, counts.get(), starts, totals.get());
        OXB_CUDA(cudaGetLastError());
        scan_u32_to_u64_from_totals(s, counts.get(), offsets, n, totals.get());
        timer.end();
    } else {
        OXB_CUDA(cudaMemsetAsync(offsets, 0, 8, s->stream));
    }
    unsigned long long total = 0;
    OXB_CUDA(cudaMemcpyAsync(&total, offsets + n, 8, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaStreamSynchronize(s->stream));
    m->total = total;
    return m.release();
}

oxb_batch* hash_join(const StreamRef& s, const Backend& b, const oxb_hash_join_args& a) {
    if (!a.left || !a.right || !a.table || !a.matches) fail(OXB_PLAN, "hash_join: null argument");
    const oxb_batch& left = *a.left;
    const oxb_batch& right = *a.right;
    const oxb_join_matches& m = *a.matches;
    if (m.probe_rows != left.rows)
        fail(OXB_EXECUTION, "join matches cover " + std::to_string(m.probe_rows) +
                                " probe rows but the probe batch has " + std::to_string(left.rows));
    if (m.table != a.table) fail(OXB_EXECUTION, "join matches were probed against another table");
    if (a.table->build_rows != right.rows)
        fail(OXB_EXECUTION, "the join table indexes " + std::to_string(a.table->build_rows) +
                                " build rows but the build batch has " + std::to_string(right.rows));
    if (a.first + a.rows < a.first || a.first + a.rows > m.total)
        fail(OXB_EXECUTION, "matches " + std::to_string(a.first) + "..+" + std::to_string(a.rows) +
                                " are outside a probe with " + std::to_string(m.total) + " matches");
    const int width = (int)left.cols.size();
    const int all = width + (int)right.cols.size();
    std::vector<int> sel;
    if (a.projection) {
        for (int i = 0; i < a.nprojection; i++) {
            if (a.projection[i] < 0 || a.projection[i] >= all)
                fail(OXB_PLAN, "join projection index " + std::to_string(a.projection[i]) +
                                   " out of range for " + std::to_string(all) + " columns");
            sel.push_back(a.projection[i]);
        }
    } else {
        for (int i = 0; i < all; i++) sel.push_back(i);
    }
    if ((int)sel.size() > kMaxOut) fail(OXB_UNSUPPORTED, "join output of more than 128 columns");
    const long long rows = (long long)a.rows;
    auto out = std::make_unique<oxb_batch>();
    out->rows = rows;
    DevGather g{};
    g.ncols = (int)sel.size();
    for (size_t i = 0; i < sel.size(); i++) {
        int side = sel[i] < width ? 0 : 1;
        const Column& src = side == 0 ? left.cols[sel[i]] : right.cols[sel[i] - width];
        Column dst;
        dst.type = src.type;
        dst.dim = src.dim;
        dst.length = rows;
        if (rows > 0) {
            dst.owner_values = dev_alloc(s, rows * (size_t)src.width(), false);
            dst.values = dst.owner_values->ptr;
            if (src.validity) {
                dst.owner_validity = dev_alloc(s, ((rows + 31) / 32) * 4, true);
                dst.validity = (uint8_t*)dst.owner_validity->ptr;
            }
        }
        g.cols[i] = DevGatherCol{src.values, src.validity, dst.values, (unsigned int*)dst.validity, src.width(), side};
        out->cols.push_back(std::move(dst));
    }
    if (rows > 0) {
        Scratch<unsigned int> status(s, 1, true);
        const long long ntiles = (rows + kGatherTile - 1) / kGatherTile;
        Scratch<long long> tile_row(s, ntiles + 1);
        const auto* offsets = (const unsigned long long*)m.offsets_mem->ptr;
        KernelTimer timer(b, s, "join_tile_rows_kernel+join_gather_kernel");
        timer.begin();
        note_launch(), join_tile_rows_kernel<<<grid_for(b, ntiles + 1, 256, 8), 256, 0, s->stream>>>(
            offsets, m.probe_rows, a.first, rows, ntiles, tile_row.get());
        note_launch(), join_gather_kernel<<<grid_for(b, ntiles * kGatherThreads, kGatherThreads, 8), kGatherThreads, 0,
                                            s->stream>>>(offsets, (const unsigned int*)m.starts_mem->ptr, tile_row.get(),
                                                         ntiles, a.table->t.rows, a.table->t.nrows, right.rows, a.first,
                                                         rows, g, status.get());
        timer.end();
        OXB_CUDA(cudaGetLastError());
        uint32_t st = 0;
        OXB_CUDA(cudaMemcpyAsync(&st, status.get(), 4, cudaMemcpyDeviceToHost, s->stream));
        OXB_CUDA(cudaStreamSynchronize(s->stream));
        check_status_word(st, "hash_join");
    }
    return out.release();
}

}  // namespace oxb
