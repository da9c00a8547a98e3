// Vector top-k: ORDER BY l2|cosine(vec, q) LIMIT k, for a batch of queries,
// over the rows a WHERE keeps (GpuVectorDistanceExec followed by the CPU
// SortExec(fetch = k) in the reference, compute/src/exec/vector.rs:29-249 and
// cpu/kernels.rs:841-927; rows with a NULL vector are left out, ties broken by
// row id, the FP32 distance as the reference computes it).
//
// The scan is a dense query x row contraction, so it runs on the 5th-generation
// tensor cores:
//   - a resident BF16 copy of the vectors (oxb_vector_index, built once) with
//     each row's FP32 squared norm and inverse norm;
//   - a persistent kernel per 128 queries: one warp issues TMA loads of
//     128 queries x 64 and 256 rows x 64 BF16 (128-byte swizzle) into a
//     4-stage mbarrier ring, one thread issues tcgen05.mma (BF16 x BF16 ->
//     FP32, M = 128 queries, N = 256 rows) into one of two 256-column TMEM
//     accumulators, and four warps read the scores back with tcgen05.ld and
//     keep, per (CTA, query), the L best rows by approximate score in a
//     lazily compacted buffer;
//   - a per-query kernel merges the CTA lists, re-ranks the best 4k (the
//     over-fetch) with the reference's sequential FP32 formula and checks,
//     with a rigorous bound on the BF16 score error, that no row it did not
//     re-rank can enter the top k; it widens the re-ranked set while the check
//     fails, and flags the query for the exact path when the lists run out;
//   - the exact path (every row's FP32 distance, a stable radix sort of
//     (distance, row)) serves flagged queries and the exact mode.
// No TMA load here uses cluster multicast; every wait is bounded.
#include <cuda.h>
#include <cuda_bf16.h>

#include "async_copy.cuh"
#include "internal.h"

namespace oxb {

namespace {

constexpr int kQTile = 128;   // queries per CTA: the TMEM lanes
constexpr int kRTile = 256;   // rows per tile: the MMA's N
constexpr int kKBlock = 64;   // BF16 per k-block: one 128-byte swizzle span
constexpr int kMaxStages = 4;
constexpr int kABytes = kQTile * kKBlock * 2;  // 16 KB
constexpr int kBBytes = kRTile * kKBlock * 2;  // 32 KB
constexpr int kStageBytes = kABytes + kBBytes;
constexpr int kScanThreads = 256;  // warp 0 TMA, warp 1 MMA, warps 4-7 epilogue
constexpr int kTmemCols = 2 * kRTile;
// Shared memory of the scan: the stage ring, the candidate buffers of the
// 128 queries (C keys each, interleaved by query), two tiles' row norms and
// selection words for the epilogue, the barriers, and alignment slack.
// Per tile: row norms, selection words, and the per-query filter column's
// order keys.
constexpr size_t kTileAux = (size_t)kRTile * 4 + (kRTile / 32) * 4 + (size_t)kRTile * 8;
constexpr size_t scan_smem(int stages, int C) {
    return (size_t)stages * kStageBytes + (size_t)C * kQTile * 8 + 2 * kTileAux + 128 + 1024;
}
constexpr int kPoolMax = 16384;  // merged candidates per query
constexpr int kExactMax = 8192;  // re-ranked candidates per query
constexpr int kFinalThreads = 256;
constexpr unsigned long long kNoKey = ~0ull;

// Instruction descriptor of tcgen05.mma kind::f16: FP32 accumulator (bits
// 4-5), BF16 A and B (bits 7-9, 10-12), both K-major, N >> 3 at bit 17,
// M >> 4 at bit 24.
constexpr unsigned kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(kRTile >> 3) << 17) |
                            ((unsigned)(kQTile >> 4) << 24);

// Shared-memory matrix descriptor of a K-major operand in the canonical
// 128-byte-swizzle layout TMA writes: 8-row groups 1024 bytes apart.
__device__ __forceinline__ unsigned long long sw128_desc(unsigned addr) {
    unsigned long long d = (unsigned long long)((addr >> 4) & 0x3FFFu);
    d |= 1ull << 16;         // leading byte offset (unused with 128-byte swizzle)
    d |= 64ull << 32;        // stride byte offset: 1024 B
    d |= 1ull << 46;         // descriptor version
    d |= 2ull << 61;         // 128-byte swizzle
    return d;
}

__device__ __forceinline__ void tmem_alloc(unsigned* slot, unsigned ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void umma_bf16(unsigned d_tmem, unsigned long long a, unsigned long long b,
                                          unsigned accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate)
        : "memory");
}

// Arrives on `bar` once every tcgen05.mma this thread issued has completed.
__device__ __forceinline__ void umma_commit(unsigned long long* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(bar))
                 : "memory");
}

// 32 consecutive accumulator columns of this warp's 32 TMEM lanes.
__device__ __forceinline__ void tmem_ld32(unsigned taddr, unsigned (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// A 2-D tile of a tensor map (x: innermost coordinate, y: row) into shared
// memory, completing on `bar`.  No cluster multicast.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_addr(dst)),
        "l"((unsigned long long)map), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// float <-> an unsigned key ordered like IEEE totalOrder (positive NaN last).
__host__ __device__ __forceinline__ unsigned f32_order(unsigned u) {
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ unsigned f32_unorder(unsigned o) {
    return (o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o;
}

// Rearranges the keys a[0], a[st], ..., a[(m - 1) st] so the first L are the
// L smallest (keys are distinct); returns the largest of them.
__device__ unsigned long long select_smallest(unsigned long long* base, int m, int L, int st) {
    auto a = [&](int i) -> unsigned long long& { return base[(size_t)i * st]; };
    int lo = 0, hi = m - 1;
    const int kth = L - 1;
    while (lo < hi) {
        unsigned long long x = a(lo), y = a((lo + hi) >> 1), z = a(hi);
        unsigned long long pivot = x < y ? (y < z ? y : (x < z ? z : x)) : (x < z ? x : (y < z ? z : y));
        int i = lo, j = hi;
        while (i <= j) {
            while (a(i) < pivot) i++;
            while (a(j) > pivot) j--;
            if (i <= j) {
                unsigned long long t = a(i);
                a(i) = a(j);
                a(j) = t;
                i++;
                j--;
            }
        }
        if (kth <= j) hi = j;
        else if (kth >= i) lo = i;
        else break;
    }
    unsigned long long mx = 0;
    for (int i = 0; i < L; i++) mx = a(i) > mx ? a(i) : mx;
    return mx;
}

struct ScanParams {
    long long n;
    int kblocks;  // dp / 64
    int groups;   // padded queries / 128
    int nq;
    int metric;
    int L;       // candidates kept per (CTA, query)
    int C;       // shared-memory buffer per query, >= L + 32
    int stages;  // stage ring depth
    const unsigned* sel;        // rows the WHERE keeps (bit per row), null = all
    const uint8_t* valid;       // vector validity, null = all
    const float* norm2;         // per row ||x||^2
    const float* inv;           // per row 1 / ||x||
    // A leaf every query has with its own literal: `qcol <qop> qlits[q]`
    // (qcol null: none); its NULLs fail every query.
    const void* qcol;
    const uint8_t* qvalid;
    int qtype;
    int qop;
    const long long* qlits;     // per query, as filter order keys
    unsigned long long* lists;  // [grid * 128][L]
    unsigned* counts;           // [grid * 128]
    unsigned long long* bounds; // [grid * 128]: every row missing from the list has a larger key
    unsigned* status;
};

__global__ void __launch_bounds__(kScanThreads, 1) topk_scan_kernel(const __grid_constant__ CUtensorMap qmap,
                                                                    const __grid_constant__ CUtensorMap xmap,
                                                                    const __grid_constant__ ScanParams p) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((1024u - (smem_addr(smem_raw) & 1023u)) & 1023u);
    const int stages = p.stages;
    unsigned long long* cands = (unsigned long long*)(smem + (size_t)stages * kStageBytes);
    long long* tqkey = (long long*)(cands + (size_t)p.C * kQTile);  // [2][256]
    float* tnorm = (float*)(tqkey + 2 * kRTile);                      // [2][256]
    unsigned* tsel = (unsigned*)(tnorm + 2 * kRTile);                 // [2][8]
    unsigned long long* bars = (unsigned long long*)(tsel + 2 * (kRTile / 32));
    unsigned long long* full = bars;
    unsigned long long* empty = bars + kMaxStages;
    unsigned long long* tfull = bars + 2 * kMaxStages;
    unsigned long long* tempty = bars + 2 * kMaxStages + 2;
    unsigned* tmem_slot = (unsigned*)(bars + 2 * kMaxStages + 4);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = blockIdx.x % p.groups;
    const int cpg = gridDim.x / p.groups;
    const long long ci = blockIdx.x / p.groups;
    const long long ntiles = (p.n + kRTile - 1) / kRTile;

    if (threadIdx.x == 0) {
        for (int s = 0; s < stages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 4 * 32);
        }
        fence_barrier_init();
    }
    if (warp == 1) tmem_alloc(tmem_slot, kTmemCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            int s = 0;
            unsigned ph = 0;
            for (long long t = ci; t < ntiles; t += cpg) {
                for (int kb = 0; kb < p.kblocks; kb++) {
                    if (!mbar_wait(&empty[s], ph ^ 1u)) {
                        atomicOr(p.status, kStatusTimeout);
                        goto producer_done;
                    }
                    unsigned char* st = smem + (size_t)s * kStageBytes;
                    mbar_arrive_expect_tx(&full[s], kStageBytes);
                    tma_load_2d(st, &qmap, kb * kKBlock, g * kQTile, &full[s]);
                    tma_load_2d(st + kABytes, &xmap, kb * kKBlock, (int)(t * kRTile), &full[s]);
                    if (++s == stages) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
            }
        producer_done:;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int s = 0, buf = 0;
            unsigned ph = 0, tph = 0;
            for (long long t = ci; t < ntiles; t += cpg) {
                if (!mbar_wait(&tempty[buf], tph ^ 1u)) {
                    atomicOr(p.status, kStatusTimeout);
                    break;
                }
                tc_fence_after();
                const unsigned d = tmem + (unsigned)(buf * kRTile);
                bool ok = true;
                for (int kb = 0; kb < p.kblocks; kb++) {
                    if (!mbar_wait(&full[s], ph)) {
                        atomicOr(p.status, kStatusTimeout);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const unsigned a0 = smem_addr(smem + (size_t)s * kStageBytes);
                    const unsigned long long ad = sw128_desc(a0), bd = sw128_desc(a0 + kABytes);
#pragma unroll
                    for (int k = 0; k < kKBlock / 16; k++)  // 32 bytes of K per instruction
                        umma_bf16(d, ad + 2ull * k, bd + 2ull * k, (kb | k) != 0);
                    umma_commit(&empty[s]);
                    if (++s == stages) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
                if (!ok) break;
                umma_commit(&tfull[buf]);
                if (++buf == 2) {
                    buf = 0;
                    tph ^= 1u;
                }
            }
        }
    } else if (warp >= 4) {
        const int qw = warp & 3;
        const int ql = qw * 32 + lane;
        const int q = g * kQTile + ql;
        const bool active = q < p.nq;
        // This query's keys: entry i at sb[i * 128] (lanes side by side).
        unsigned long long* sb = cands + ql;
        unsigned long long thr = kNoKey;
        float thr_f = INFINITY;  // the score part of thr (+inf while the list has room)
        int cnt = 0;
        bool dropped = false;
        int buf = 0;
        unsigned tph = 0;
        const float* nsrc = p.metric == 0 ? p.norm2 : p.inv;
        const long long qlit = p.qcol && active ? __ldg(p.qlits + q) : 0;
        int par = 0;
        for (long long t = ci; t < ntiles; t += cpg, par ^= 1) {
            // The four epilogue warps stage this tile's row norms and
            // selection words (WHERE, validity, rows past n) once for all
            // 128 queries; two buffers, so a warp one tile ahead cannot
            // overwrite what a slower one still reads.
            {
                float* tn = tnorm + par * kRTile;
                for (int h = 0; h < kRTile / kQTile; h++) {
                    const long long r = t * kRTile + h * kQTile + ql;
                    tn[h * kQTile + ql] = r < p.n ? __ldg(nsrc + r) : 0.0f;
                    if (p.qcol && r < p.n)
                        tqkey[par * kRTile + h * kQTile + ql] =
                            p.qtype == kFloat64 ? filter_order_key(__ldg((const double*)p.qcol + r))
                            : p.qtype == kInt64 ? __ldg((const long long*)p.qcol + r)
                                                : (long long)__ldg((const int*)p.qcol + r);
                }
                if (ql < kRTile / 32) {
                    const long long row0 = t * kRTile + ql * 32;
                    unsigned sel = 0;
                    if (row0 < p.n) {
                        sel = p.sel ? __ldg(p.sel + (row0 >> 5)) : ~0u;
                        // The bitmaps' bytes for these 32 rows, none past their end.
                        const long long b0 = row0 >> 3, nbytes = (p.n + 7) >> 3;
                        for (int bm = 0; bm < 2; bm++) {
                            const uint8_t* vb = bm == 0 ? p.valid : (p.qcol ? p.qvalid : nullptr);
                            if (!vb) continue;
                            unsigned v = 0;
#pragma unroll
                            for (int bi = 0; bi < 4; bi++)
                                if (b0 + bi < nbytes) v |= (unsigned)__ldg(vb + b0 + bi) << (8 * bi);
                            sel &= v;
                        }
                        if (row0 + 32 > p.n) sel &= (1u << (p.n - row0)) - 1u;
                    }
                    tsel[par * (kRTile / 32) + ql] = sel;
                }
                asm volatile("bar.sync 1, 128;" ::: "memory");
            }
            // Every epilogue thread leaves together if any wait gave up, so
            // none is left at the next named barrier.
            const bool ok = mbar_wait(&tfull[buf], tph);
            unsigned any_fail;
            asm volatile(
                "{\n\t.reg .pred p, q;\n\t"
                "setp.eq.u32 p, %1, 0;\n\t"
                "bar.red.or.pred q, 2, 128, p;\n\t"
                "selp.u32 %0, 1, 0, q;\n\t}"
                : "=r"(any_fail)
                : "r"((unsigned)ok)
                : "memory");
            if (any_fail) {
                if (!ok) atomicOr(p.status, kStatusTimeout);
                break;
            }
            tc_fence_after();
            const float* tn = tnorm + par * kRTile;
            for (int c = 0; c < kRTile / 32; c++) {
                unsigned r[32];
                __syncwarp();
                tmem_ld32(tmem + ((unsigned)(qw * 32) << 16) + (unsigned)(buf * kRTile + c * 32), r);
                // Room for 32 more keys in every buffer: when one is nearly
                // full, the warp's lanes compact theirs together.
                if (__any_sync(0xffffffffu, cnt > p.C - 32) && cnt > p.L) {
                    thr = select_smallest(sb, cnt, p.L, kQTile);
                    thr_f = __uint_as_float(f32_unorder((unsigned)(thr >> 32)));
                    cnt = p.L;
                    dropped = true;
                }
                unsigned sel = tsel[par * (kRTile / 32) + c];
                if (p.qcol && active && sel) {
                    // This query's own leaf over the chunk's rows.
                    const long long* qk = tqkey + par * kRTile + c * 32;
                    unsigned m = 0;
                    switch (p.qop) {
                        case 0:
#pragma unroll
                            for (int j = 0; j < 32; j++) m |= (unsigned)(qk[j] == qlit) << j;
                            break;
                        case 1:
#pragma unroll
                            for (int j = 0; j < 32; j++) m |= (unsigned)(qk[j] < qlit) << j;
                            break;
                        case 2:
#pragma unroll
                            for (int j = 0; j < 32; j++) m |= (unsigned)(qk[j] <= qlit) << j;
                            break;
                        case 3:
#pragma unroll
                            for (int j = 0; j < 32; j++) m |= (unsigned)(qk[j] > qlit) << j;
                            break;
                        default:
#pragma unroll
                            for (int j = 0; j < 32; j++) m |= (unsigned)(qk[j] >= qlit) << j;
                            break;
                    }
                    sel &= m;
                }
                if (!active || !sel) continue;
                const unsigned row0 = (unsigned)(t * kRTile + c * 32);
                // Scores (a NaN counts as +inf, after every finite score) and
                // their minimum over the selected rows; only a chunk whose
                // minimum reaches the threshold is looked at row by row.
                float sc[32];
                float mn = INFINITY;
                const float4* tn4 = (const float4*)(tn + c * 32);
#pragma unroll
                for (int j4 = 0; j4 < 8; j4++) {
                    const float4 nr = tn4[j4];
                    const float nv[4] = {nr.x, nr.y, nr.z, nr.w};
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int j = j4 * 4 + u;
                        const float dot = __uint_as_float(r[j]);
                        float x = p.metric == 0 ? fmaf(-2.0f, dot, nv[u]) : -dot * nv[u];
                        x = x == x ? x : INFINITY;
                        sc[j] = x;
                        mn = fminf(mn, ((sel >> j) & 1u) ? x : INFINITY);
                    }
                }
                if (!(mn <= thr_f)) continue;
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    if (!((sel >> j) & 1u) || !(sc[j] <= thr_f)) continue;
                    const unsigned long long key =
                        ((unsigned long long)f32_order(__float_as_uint(sc[j])) << 32) | (row0 + j);
                    if (key < thr) sb[(size_t)(cnt++) * kQTile] = key;
                }
            }
            tc_fence_before();
            mbar_arrive(&tempty[buf]);
            if (++buf == 2) {
                buf = 0;
                tph ^= 1u;
            }
        }
        if (cnt > p.L) {
            thr = select_smallest(sb, cnt, p.L, kQTile);
            cnt = p.L;
            dropped = true;
        }
        if (!active) cnt = 0;
        unsigned long long* out = p.lists + ((size_t)blockIdx.x * kQTile + ql) * p.L;
        for (int i = 0; i < cnt; i++) out[i] = sb[(size_t)i * kQTile];
        p.counts[(size_t)blockIdx.x * kQTile + ql] = (unsigned)cnt;
        p.bounds[(size_t)blockIdx.x * kQTile + ql] = dropped ? thr : kNoKey;
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem, kTmemCols);
    }
}

// The reference's FP32 distance of row x (l2 = sqrt of the sum of squared
// differences, cosine = 1 - dot / (|x| |q|)), its sums taken in index order
// (cpu/kernels.rs:909-927), by a whole warp: the lanes load the row 32
// values at a time and form each term; the terms are added in index order
// from -0.0, one correctly rounded operation per step (the same additions as
// a serial loop, so the same bits); a zero norm gives the NaN 0x7fc00000.  Also the
// FP64 dot product and squared norm, summed in any order (a report only).
// Every lane returns the distance's bits.
__device__ unsigned exact_distance_warp(const float* x, const float* q, int dim, int metric, float qnorm,
                                        double* dot64, double* xx64) {
    const int lane = threadIdx.x & 31;
    float s0 = -0.0f, s1 = -0.0f;
    double dd = 0.0, xd = 0.0;
    constexpr int kChunks = 8;  // 32-value chunks whose loads are in flight together
    for (int base = 0; base < dim; base += 32 * kChunks) {
        float a[kChunks];
#pragma unroll
        for (int c = 0; c < kChunks; c++) {
            const int i = base + c * 32 + lane;
            a[c] = i < dim ? __ldg(x + i) : 0.0f;
        }
#pragma unroll
        for (int c = 0; c < kChunks; c++) {
            const int b0 = base + c * 32;
            if (b0 >= dim) break;
            const int i = b0 + lane;
            float t0 = 0.0f, t1 = 0.0f;
            if (i < dim) {
                dd += (double)a[c] * (double)q[i];
                xd += (double)a[c] * (double)a[c];
                if (metric == 0) {
                    const float d = __fsub_rn(a[c], q[i]);
                    t0 = __fmul_rn(d, d);
                } else {
                    t0 = __fmul_rn(a[c], q[i]);
                    t1 = __fmul_rn(a[c], a[c]);
                }
            }
            const int cnt = dim - b0 < 32 ? dim - b0 : 32;
            for (int l = 0; l < 32; l++) {
                const float v0 = __shfl_sync(0xffffffffu, t0, l);
                const float v1 = __shfl_sync(0xffffffffu, t1, l);
                if (l < cnt) {
                    s0 = __fadd_rn(s0, v0);
                    s1 = __fadd_rn(s1, v1);
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        dd += __shfl_xor_sync(0xffffffffu, dd, o);
        xd += __shfl_xor_sync(0xffffffffu, xd, o);
    }
    *dot64 = dd;
    *xx64 = xd;
    // every lane added the same values in the same order: s0, s1 agree
    if (metric == 0) return __float_as_uint(__fsqrt_rn(s0));
    const float na = __fsqrt_rn(s1);
    if (na == 0.0f || qnorm == 0.0f) return 0x7fc00000u;
    return __float_as_uint(__fsub_rn(1.0f, __fdiv_rn(s0, __fmul_rn(na, qnorm))));
}

// Ascending bitonic sort of a[0, m), m a power of two, by the whole block.
__device__ void bitonic_sort(unsigned long long* a, int m) {
    for (int size = 2; size <= m; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            __syncthreads();
            for (int i = threadIdx.x; i < m; i += blockDim.x) {
                const int j = i ^ stride;
                if (j > i) {
                    const bool up = (i & size) == 0;
                    const unsigned long long x = a[i], y = a[j];
                    if ((x > y) == up) {
                        a[i] = y;
                        a[j] = x;
                    }
                }
            }
        }
    }
    __syncthreads();
}

struct FinalParams {
    int k, overfetch, groups, cpg, cap, nq, dim, metric;
    int pool_cap;  // merged candidates a query can have: a power of two >= cpg * cap, <= kPoolMax
    int ex_cap;    // re-ranked candidates at most: min(pool_cap, kExactMax)
    const unsigned long long* lists;
    const unsigned* counts;
    const unsigned long long* bounds;
    const float* table;   // FP32 vectors, row-major
    const unsigned* rowmap;  // candidate index -> row (a compacted scan), or null
    const float* queries; // FP32, nq x dim
    const float* qnorm;   // per query ||q|| (FP32, folded in order)
    float xmax;
    long long* ids;
    float* dist;
    int* fallback;                  // per query: 1 = take the exact path
    unsigned long long* err_max;    // bits of the largest |BF16 score - FP64 score|
    double* err_sum;
    unsigned long long* err_count;
};

// The smallest true distance a row outside the re-ranked set can have, from
// the smallest approximate score `sb` among such rows, and the bound on the
// BF16 score error: each product carries at most 2^-8 relative error from
// each operand's rounding to BF16 (2^-7 together, plus FP32 accumulation),
// so |score error| <= 0.008 * ||q|| * ||x|| for the dot product.
__device__ float distance_floor(int metric, float sb, float qn, float xmax) {
    if (metric == 0) {
        const float eps = 2.0f * 0.008f * qn * xmax + 2e-6f * (xmax * xmax + qn * qn);
        const float d2 = sb - eps + qn * qn;
        return d2 > 0.0f ? sqrtf(d2) : 0.0f;
    }
    const float eps = 0.0081f * qn;
    return qn > 0.0f ? 1.0f + (sb - eps) / qn : -INFINITY;
}

__global__ void __launch_bounds__(kFinalThreads) topk_final_kernel(const __grid_constant__ FinalParams p) {
    extern __shared__ __align__(16) unsigned char sm[];
    unsigned long long* pool = (unsigned long long*)sm;         // pool_cap
    unsigned long long* ex = pool + p.pool_cap;                 // ex_cap
    float* qv = (float*)(ex + p.ex_cap);                        // dim
    __shared__ int offs[1024], cnts[1024];
    __shared__ int total_s, R_s, state_s;  // state: 0 go on, 1 done, 2 exact path
    __shared__ unsigned long long bmin_s;
    const int q = blockIdx.x;
    const int g = q / kQTile, lane = q % kQTile;
    for (int i = threadIdx.x; i < p.dim; i += blockDim.x) qv[i] = p.queries[(size_t)q * p.dim + i];
    if (threadIdx.x == 0) {
        int total = 0;
        unsigned long long bmin = kNoKey;
        for (int i = 0; i < p.cpg; i++) {
            const size_t c = (size_t)(g + i * p.groups) * kQTile + lane;
            offs[i] = total;
            cnts[i] = (int)p.counts[c];
            total += cnts[i];
            bmin = p.bounds[c] < bmin ? p.bounds[c] : bmin;
        }
        total_s = total;
        bmin_s = bmin;
        state_s = total > p.pool_cap ? 2 : 0;
    }
    __syncthreads();
    if (state_s == 2) {
        if (threadIdx.x == 0) p.fallback[q] = 1;
        return;
    }
    const int total = total_s;
    for (int i = 0; i < p.cpg; i++) {
        const unsigned long long* src = p.lists + ((size_t)(g + i * p.groups) * kQTile + lane) * p.cap;
        for (int j = threadIdx.x; j < cnts[i]; j += blockDim.x) pool[offs[i] + j] = src[j];
    }
    int m = 1;
    while (m < total) m <<= 1;
    for (int i = total + threadIdx.x; i < m; i += blockDim.x) pool[i] = kNoKey;
    bitonic_sort(pool, m);

    const float qn = p.qnorm[q];
    int R = min(p.overfetch * p.k, total);
    if (R > p.ex_cap) R = p.ex_cap;
    int done = 0;
    double emax = 0.0, esum = 0.0;
    unsigned long long ecount = 0;
    for (int iter = 0; iter < 32; iter++) {
        // One warp per candidate: coalesced row loads, the terms added in
        // index order.
        for (int i = done + (threadIdx.x >> 5); i < R; i += blockDim.x >> 5) {
            const unsigned idx = (unsigned)(pool[i] & 0xFFFFFFFFu);
            // compacted indices keep row order, so (score, index) sorts as (score, row)
            const unsigned row = p.rowmap ? __ldg(p.rowmap + idx) : idx;
            const float* x = p.table + (size_t)row * p.dim;
            double dot, xx;
            const unsigned d = exact_distance_warp(x, qv, p.dim, p.metric, qn, &dot, &xx);
            if ((threadIdx.x & 31) != 0) continue;
            ex[i] = ((unsigned long long)f32_order(d) << 32) | row;
            // The BF16 score against the FP64 one, for the report.
            const double s64 = p.metric == 0 ? xx - 2.0 * dot : (xx > 0.0 ? -dot / sqrt(xx) : 0.0);
            const float sa = __uint_as_float(f32_unorder((unsigned)(pool[i] >> 32)));
            const double e = fabs((double)sa - s64);
            if (isfinite(e)) {
                emax = e > emax ? e : emax;
                esum += e;
                ecount++;
            }
        }
        int m2 = 1;
        while (m2 < R) m2 <<= 1;
        __syncthreads();
        for (int i = R + threadIdx.x; i < m2; i += blockDim.x) ex[i] = kNoKey;
        bitonic_sort(ex, m2);
        if (threadIdx.x == 0) {
            unsigned long long b = bmin_s;
            if (R < total && pool[R] < b) b = pool[R];
            int st = 0;
            if (b == kNoKey) {
                st = 1;  // every row the WHERE keeps was re-ranked
            } else if (R >= p.k) {
                const float dk = __uint_as_float(f32_unorder((unsigned)(ex[p.k - 1] >> 32)));
                const float sb = __uint_as_float(f32_unorder((unsigned)(b >> 32)));
                const float lb = distance_floor(p.metric, sb, qn, p.xmax);
                // The reference's own FP32 rounding, so a row outside may not tie.
                const float delta = (float)p.dim * 2.5e-7f * fmaxf(fabsf(dk), 1.0f) + 1e-6f;
                if (isfinite(dk) && lb - delta > dk) st = 1;
            }
            if (st == 0) {
                if (R < total && R < p.ex_cap) {
                    R_s = min(min(2 * R, total), p.ex_cap);
                } else {
                    st = 2;
                }
            }
            state_s = st;
        }
        __syncthreads();
        if (state_s != 0) break;
        done = R;
        R = R_s;
    }
    if (state_s != 1) {
        if (threadIdx.x == 0) p.fallback[q] = 1;
    } else {
        for (int j = threadIdx.x; j < p.k; j += blockDim.x) {
            const unsigned long long e = j < R ? ex[j] : kNoKey;
            p.ids[(size_t)q * p.k + j] = e == kNoKey ? -1 : (long long)(e & 0xFFFFFFFFu);
            ((unsigned*)p.dist)[(size_t)q * p.k + j] = e == kNoKey ? 0x7fc00000u : f32_unorder((unsigned)(e >> 32));
        }
    }
    if (ecount) {
        atomicMax(p.err_max, (unsigned long long)__double_as_longlong(emax));
        atomicAdd(p.err_sum, esum);
        atomicAdd(p.err_count, ecount);
    }
}

// The exact path's keys: (distance order, row) for rows the WHERE keeps with
// a valid vector, the largest key for the rest.
__global__ void topk_exact_keys_kernel(const float* __restrict__ d, const unsigned* __restrict__ sel,
                                       const uint8_t* __restrict__ valid, long long n, DevLeaf qleaf,
                                       unsigned long long* __restrict__ keys) {
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
        bool ok = (!sel || ((__ldg(sel + (r >> 5)) >> (r & 31)) & 1u)) && valid_at(valid, r);
        if (ok && qleaf.values) {
            if (!valid_at(qleaf.validity, r)) ok = false;
            else {
                const long long a = qleaf.type == kFloat64 ? filter_order_key(__ldg((const double*)qleaf.values + r))
                                    : qleaf.type == kInt64 ? __ldg((const long long*)qleaf.values + r)
                                                           : (long long)__ldg((const int*)qleaf.values + r);
                ok = cmp_holds(qleaf.op, a, qleaf.lit);
            }
        }
        // The distance's bits, loaded as an integer: a NaN keeps its bits.
        const unsigned bits = __ldg((const unsigned*)d + r);
        keys[r] = ok ? ((unsigned long long)f32_order(bits) << 32) | (unsigned long long)r : kNoKey;
    }
}

__global__ void topk_exact_out_kernel(const unsigned long long* __restrict__ keys, long long n, int k,
                                      long long* __restrict__ ids, float* __restrict__ dist) {
    for (int j = threadIdx.x; j < k; j += blockDim.x) {
        const unsigned long long e = j < n ? keys[j] : kNoKey;
        ids[j] = e == kNoKey ? -1 : (long long)(e & 0xFFFFFFFFu);
        ((unsigned*)dist)[j] = e == kNoKey ? 0x7fc00000u : f32_unorder((unsigned)(e >> 32));
    }
}

// One warp per row: the BF16 copy (zero-padded to dp), ||x||^2 and 1/||x||.
__global__ void vector_index_kernel(const float* __restrict__ x, long long n, int dim, int dp,
                                    __nv_bfloat16* __restrict__ out, float* __restrict__ norm2,
                                    float* __restrict__ inv, unsigned* __restrict__ xmax_bits) {
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long r = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); r < n; r += warps) {
        float s = 0.0f;
        for (int i = lane; i < dp; i += 32) {
            const float v = i < dim ? __ldg(x + r * dim + i) : 0.0f;
            out[r * dp + i] = __float2bfloat16_rn(v);
            s = fmaf(v, v, s);
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            norm2[r] = s;
            const float nr = sqrtf(s);
            inv[r] = nr > 0.0f ? 1.0f / nr : __int_as_float(0x7fc00000);
            if (nr == nr) atomicMax(xmax_bits, __float_as_uint(nr));
        }
    }
}

// Queries: the BF16 copy (qp x dp, zero rows and columns past the real ones)
// and ||q|| folded in index order in FP32 (the reference's q norm).
__global__ void query_prep_kernel(const float* __restrict__ q, int nq, int dim, int qp, int dp,
                                  __nv_bfloat16* __restrict__ out, float* __restrict__ qnorm) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)qp * dp;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / dp), c = (int)(i % dp);
        out[i] = __float2bfloat16_rn(r < nq && c < dim ? q[(size_t)r * dim + c] : 0.0f);
    }
    // ||q|| folded in index order from -0.0 (the reference's FP32 norm), one
    // warp a query: coalesced loads, each lane's squares added in order.
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; r < nq; r += warps) {
        const float* row = q + (size_t)r * dim;
        float s = -0.0f;
        for (int base = 0; base < dim; base += 32) {
            const int c = base + lane;
            const float v = c < dim ? row[c] : 0.0f;
            const float t = __fmul_rn(v, v);
            const int cnt = dim - base < 32 ? dim - base : 32;
            for (int l = 0; l < 32; l++) {
                const float u = __shfl_sync(0xffffffffu, t, l);
                if (l < cnt) s = __fadd_rn(s, u);
            }
        }
        if (lane == 0) qnorm[r] = __fsqrt_rn(s);
    }
}

// cuTensorMapEncodeTiled, found through the runtime so the library itself
// does not link the driver library.
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_tiled() {
    static std::mutex mu;
    static EncodeTiled fn = nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        OXB_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p) fail(OXB_DEVICE, "cuTensorMapEncodeTiled is not available");
        fn = (EncodeTiled)p;
    }
    return fn;
}

// Compaction of the rows a query batch can return (a WHERE that keeps few
// rows): per 32-row word, the rows the shared WHERE keeps with a valid
// vector and, when there is a per-query leaf, a valid leaf operand (a NULL
// operand fails every query); and its count.
__global__ void topk_compact_words_kernel(const unsigned* __restrict__ sel, const uint8_t* __restrict__ valid,
                                          const uint8_t* __restrict__ qvalid, long long n, unsigned* __restrict__ words,
                                          unsigned* __restrict__ counts) {
    const long long nwords = (n + 31) >> 5, nbytes = (n + 7) >> 3;
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < nwords;
         w += (long long)gridDim.x * blockDim.x) {
        const long long row0 = w << 5, b0 = row0 >> 3;
        unsigned m = sel ? __ldg(sel + w) : ~0u;
        for (int bm = 0; bm < 2; bm++) {
            const uint8_t* vb = bm == 0 ? valid : qvalid;
            if (!vb) continue;
            unsigned v = 0;
#pragma unroll
            for (int i = 0; i < 4; i++)
                if (b0 + i < nbytes) v |= (unsigned)__ldg(vb + b0 + i) << (8 * i);
            m &= v;
        }
        if (row0 + 32 > n) m &= (1u << (n - row0)) - 1u;
        words[w] = m;
        counts[w] = (unsigned)__popc(m);
    }
}

// Copies the kept rows, in row order, to the compacted table: BF16 row,
// norms, row id and (with a per-query leaf) the operand's order key.  One
// warp per 32-row word.
__global__ void topk_compact_gather_kernel(const unsigned* __restrict__ words, const unsigned long long* __restrict__ offs,
                                           long long nwords, const uint4* __restrict__ bf16, int row_u4,
                                           const float* __restrict__ norm2, const float* __restrict__ inv,
                                           const void* __restrict__ qcol, int qtype, uint4* __restrict__ cb,
                                           float* __restrict__ cn2, float* __restrict__ cinv,
                                           unsigned* __restrict__ rowmap, long long* __restrict__ cqkey) {
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long w = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); w < nwords; w += warps) {
        unsigned m = words[w];
        unsigned long long pos = offs[w];
        while (m) {
            const unsigned r = (unsigned)(w << 5) + (unsigned)(__ffs(m) - 1);
            m &= m - 1u;
            for (int i = lane; i < row_u4; i += 32) cb[pos * row_u4 + i] = __ldg(bf16 + (size_t)r * row_u4 + i);
            if (lane == 0) {
                cn2[pos] = __ldg(norm2 + r);
                cinv[pos] = __ldg(inv + r);
                rowmap[pos] = r;
                if (cqkey)
                    cqkey[pos] = qtype == kFloat64 ? filter_order_key(__ldg((const double*)qcol + r))
                                 : qtype == kInt64 ? __ldg((const long long*)qcol + r)
                                                   : (long long)__ldg((const int*)qcol + r);
            }
            pos++;
        }
    }
}

void encode_bf16_map(CUtensorMap* map, const void* base, long long rows, int dp, int box_rows) {
    cuuint64_t dims[2] = {(cuuint64_t)dp, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)dp * 2};
    cuuint32_t box[2] = {(cuuint32_t)kKBlock, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = encode_tiled()(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims,
                                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(OXB_DEVICE, "cuTensorMapEncodeTiled failed with code " + std::to_string((int)r));
}

}  // namespace

oxb_vector_index* vector_index_build(const StreamRef& s, const Backend& b, const oxb_batch& in, int column) {
    if (column < 0 || column >= (int)in.cols.size()) fail(OXB_PLAN, "vector column index out of range");
    const Column& vec = in.cols[column];
    if (vec.type != kVectorF32) fail(OXB_UNSUPPORTED, "column " + std::to_string(column) + " is not FixedSizeList<Float32>");
    if (vec.dim < 1) fail(OXB_UNSUPPORTED, "vectors of dimension 0");
    if (in.rows >= (1ll << 32)) fail(OXB_UNSUPPORTED, "vector top-k over 2^32 or more rows");
    auto ix = std::make_unique<oxb_vector_index>();
    ix->vec = vec;
    ix->n = in.rows;
    ix->dim = vec.dim;
    ix->dp = (vec.dim + kKBlock - 1) / kKBlock * kKBlock;
    const long long n = in.rows;
    // At least one tile of rows, so the tensor map's box never exceeds it
    // (rows past n are never scored).
    const long long mrows = n > kRTile ? n : kRTile;
    ix->bf16 = dev_alloc(s, (size_t)mrows * ix->dp * 2, true);
    ix->norm2 = dev_alloc(s, (size_t)(n > 0 ? n : 1) * 4, false);
    ix->inv = dev_alloc(s, (size_t)(n > 0 ? n : 1) * 4, false);
    Scratch<unsigned> xmax(s, 1, true);
    if (n > 0) {
        note_launch(), vector_index_kernel<<<grid_for(b, n * 32, 256, 8), 256, 0, s->stream>>>(
            (const float*)vec.values, n, vec.dim, ix->dp, (__nv_bfloat16*)ix->bf16->ptr, (float*)ix->norm2->ptr,
            (float*)ix->inv->ptr, xmax.get());
        OXB_CUDA(cudaGetLastError());
    }
    unsigned bits = 0;
    OXB_CUDA(cudaMemcpyAsync(&bits, xmax.get(), 4, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaStreamSynchronize(s->stream));
    std::memcpy(&ix->xmax, &bits, 4);
    if (n > 0) encode_bf16_map(&ix->xmap, ix->bf16->ptr, mrows, ix->dp, kRTile);
    return ix.release();
}

void vector_topk(const StreamRef& s, const Backend& b, const oxb_vector_topk_args& a, int64_t* out_ids,
                 float* out_dist, oxb_vector_topk_stats* stats) {
    if (!a.index || !a.input) fail(OXB_PLAN, "vector_topk: null index or input");
    const oxb_vector_index& ix = *a.index;
    const oxb_batch& in = *a.input;
    if (in.rows != ix.n) fail(OXB_PLAN, "the index was built over " + std::to_string(ix.n) + " rows, the batch has " +
                                            std::to_string(in.rows));
    if (a.dim != ix.dim) fail(OXB_PLAN, "queries have " + std::to_string(a.dim) + " dimensions, the index " +
                                            std::to_string(ix.dim));
    if (a.metric != OXB_METRIC_L2 && a.metric != OXB_METRIC_COSINE) fail(OXB_PLAN, "unknown metric");
    if (a.k < 1 || a.k > kExactMax / 2) fail(OXB_UNSUPPORTED, "k must be between 1 and 4096");
    if (a.nqueries < 0) fail(OXB_PLAN, "negative query count");
    if (a.nqueries > 0 && (!a.queries || !out_ids || !out_dist)) fail(OXB_PLAN, "null queries or outputs");
    DevPredicate pred = make_predicate(in, a.leaves, a.nleaves);
    // The per-query leaf: checked like a shared one, literals as order keys.
    DevLeaf qleaf{};
    std::vector<long long> qlits_h;
    if (a.qleaf_column >= 0 && a.nqueries > 0) {
        if (!a.qleaf_lits) fail(OXB_PLAN, "per-query literals are null");
        oxb_leaf probe{};
        probe.column = a.qleaf_column;
        probe.op = a.qleaf_op;
        probe.lit_type = a.qleaf_type;
        qlits_h.resize(a.nqueries);
        for (int q = 0; q < a.nqueries; q++) {
            probe.lit.i = a.qleaf_lits[q];
            const DevPredicate one = make_predicate(in, &probe, 1);
            qlits_h[q] = one.leaves[0].lit;
            qleaf = one.leaves[0];
        }
    }
    oxb_vector_topk_stats st{};
    const int nq = a.nqueries, k = a.k, dim = ix.dim, dp = ix.dp;
    const long long n = ix.n;
    if (nq == 0) {
        if (stats) *stats = st;
        return;
    }
    const int qp = (nq + kQTile - 1) / kQTile * kQTile;
    const int groups = qp / kQTile;
    Scratch<float> qf(s, (size_t)nq * dim);
    Scratch<__nv_bfloat16> qb(s, (size_t)qp * dp);
    Scratch<float> qnorm(s, nq);
    OXB_CUDA(cudaMemcpyAsync(qf.get(), a.queries, (size_t)nq * dim * 4, cudaMemcpyHostToDevice, s->stream));
    note_launch(), query_prep_kernel<<<grid_for(b, (long long)qp * dp, 256, 4), 256, 0, s->stream>>>(
        qf.get(), nq, dim, qp, dp, qb.get(), qnorm.get());
    OXB_CUDA(cudaGetLastError());
    AllocRef sel;
    if (pred.nleaves > 0 && n > 0) sel = predicate_bits(s, b, pred, n);
    Scratch<long long> qlits;
    if (qleaf.values || (!qlits_h.empty() && n == 0)) {
        qlits = Scratch<long long>(s, nq);
        OXB_CUDA(cudaMemcpyAsync(qlits.get(), qlits_h.data(), (size_t)nq * 8, cudaMemcpyHostToDevice, s->stream));
    }
    const unsigned* selp = sel ? (const unsigned*)sel->ptr : nullptr;

    Scratch<long long> ids(s, (size_t)nq * k);
    Scratch<float> dist(s, (size_t)nq * k);
    Scratch<int> fallback(s, nq, true);
    Scratch<unsigned long long> err(s, 3, true);  // max bits, sum (double), count
    const int over = a.overfetch > 0 ? a.overfetch : 4;
    int cpg = b.sms / groups;
    if (cpg < 1) cpg = 1;
    const int grid = cpg * groups;
    // Candidates kept per (CTA, query): enough that each CTA's bound sits far
    // below the k-th distance (the over-fetch of 4k is taken from the merged
    // lists), and buffers with room for them plus a 32-key chunk plus slack,
    // so a compaction frees many slots; the deepest stage ring that fits.
    int L = std::max(1, std::min({std::max(2 * k, k + 16), over * k, kPoolMax / cpg}));
    int C = 0, stages = 0;
    for (; L >= 1 && !C; L = L * 3 / 4) {
        for (stages = kMaxStages; stages >= 2; stages--) {
            const size_t fixed = scan_smem(stages, 0);
            if (fixed >= b.smem_optin) continue;
            const int cmax = (int)((b.smem_optin - fixed) / ((size_t)kQTile * 8));
            if (cmax >= L + 32 + std::min(L, 16)) {
                C = std::min(cmax, 2 * L + 32);
                break;
            }
        }
        if (C) break;
    }
    const bool fast = !a.exact && n > 0 && C > 0;
    std::vector<int> host_fb(nq, 1);
    // A WHERE (or NULL vectors) that keeps at most 40 % of the rows: the kept
    // rows are copied, in row order, to a compacted BF16 table and only those
    // are scanned; the re-rank maps each candidate back to its row.
    bool compact = false;
    long long nsel = n;
    AllocRef cb_mem, cn2_mem, cinv_mem, rowmap_mem, cq_mem;
    CUtensorMap cmap;
    // Timed: the compaction and the scan (the host's read of the kept count
    // between them is not).
    KernelTimer timer(b, s, "topk_scan_kernel");
    Scratch<unsigned> words, wcounts;
    Scratch<unsigned long long> woffs;
    if (fast && (selp || ix.vec.validity || qleaf.validity)) {
        const long long nwords = (n + 31) / 32;
        words = Scratch<unsigned>(s, nwords);
        wcounts = Scratch<unsigned>(s, nwords);
        woffs = Scratch<unsigned long long>(s, nwords + 1);
        timer.begin();
        note_launch(), topk_compact_words_kernel<<<grid_for(b, nwords, 256, 8), 256, 0, s->stream>>>(
            selp, ix.vec.validity, qleaf.validity, n, words.get(), wcounts.get());
        OXB_CUDA(cudaGetLastError());
        scan_u32_to_u64(s, b, wcounts.get(), woffs.get(), nwords);
        timer.end();
        unsigned long long hn = 0;
        OXB_CUDA(cudaMemcpyAsync(&hn, woffs.get() + nwords, 8, cudaMemcpyDeviceToHost, s->stream));
        OXB_CUDA(cudaStreamSynchronize(s->stream));
        // Measured on B200: a full scan costs about 0.72 ns a row, a compacted
        // one about 0.57 ns (copy) + 1.14 ns (scan) a kept row: compaction
        // pays below about 42 % kept.
        if ((long long)hn * 5 <= n * 2) {
            compact = true;
            nsel = (long long)hn;
            const long long crows = nsel > kRTile ? nsel : kRTile;  // the tensor map's box fits
            const long long m1 = nsel > 0 ? nsel : 1;
            cb_mem = dev_alloc(s, (size_t)crows * dp * 2, nsel < kRTile);
            cn2_mem = dev_alloc(s, (size_t)m1 * 4, false);
            cinv_mem = dev_alloc(s, (size_t)m1 * 4, false);
            rowmap_mem = dev_alloc(s, (size_t)m1 * 4, false);
            if (qleaf.values) cq_mem = dev_alloc(s, (size_t)m1 * 8, false);
            timer.begin();
            if (nsel > 0) {
                note_launch(), topk_compact_gather_kernel<<<grid_for(b, nwords * 32, 256, 8), 256, 0, s->stream>>>(
                    words.get(), woffs.get(), nwords, (const uint4*)ix.bf16->ptr, dp * 2 / 16,
                    (const float*)ix.norm2->ptr, (const float*)ix.inv->ptr, qleaf.values, qleaf.type,
                    (uint4*)cb_mem->ptr, (float*)cn2_mem->ptr, (float*)cinv_mem->ptr, (unsigned*)rowmap_mem->ptr,
                    qleaf.values ? (long long*)cq_mem->ptr : nullptr);
                OXB_CUDA(cudaGetLastError());
            }
            encode_bf16_map(&cmap, cb_mem->ptr, crows, dp, kRTile);
        }
    }
    if (fast) {
        const int cap = L;
        Scratch<unsigned long long> lists(s, (size_t)grid * kQTile * cap);
        Scratch<unsigned> counts(s, (size_t)grid * kQTile);
        Scratch<unsigned long long> bounds(s, (size_t)grid * kQTile);
        Scratch<unsigned> status(s, 1, true);
        CUtensorMap qmap;
        encode_bf16_map(&qmap, qb.get(), qp, dp, kQTile);
        ScanParams sp{};
        sp.n = nsel;
        sp.kblocks = dp / kKBlock;
        sp.groups = groups;
        sp.nq = nq;
        sp.metric = a.metric;
        sp.L = L;
        sp.C = C;
        sp.stages = stages;
        sp.sel = compact ? nullptr : selp;
        sp.valid = compact ? nullptr : ix.vec.validity;
        sp.norm2 = compact ? (const float*)cn2_mem->ptr : (const float*)ix.norm2->ptr;
        sp.inv = compact ? (const float*)cinv_mem->ptr : (const float*)ix.inv->ptr;
        sp.qcol = compact && qleaf.values ? cq_mem->ptr : qleaf.values;
        sp.qvalid = compact ? nullptr : qleaf.validity;
        sp.qtype = compact && qleaf.values ? kInt64 : qleaf.type;
        sp.qop = qleaf.op;
        sp.qlits = qlits.get();
        sp.lists = lists.get();
        sp.counts = counts.get();
        sp.bounds = bounds.get();
        sp.status = status.get();
        const size_t smem = scan_smem(stages, C);
        allow_smem(topk_scan_kernel, smem);
        if (!compact) timer.begin();  // a compacted scan's segment began with the copy
        note_launch(), topk_scan_kernel<<<grid, kScanThreads, smem, s->stream>>>(qmap, compact ? cmap : ix.xmap, sp);
        timer.end();
        OXB_CUDA(cudaGetLastError());
        FinalParams fp{};
        fp.k = k;
        fp.overfetch = over;
        fp.groups = groups;
        fp.cpg = cpg;
        fp.cap = cap;
        fp.nq = nq;
        fp.dim = dim;
        fp.metric = a.metric;
        fp.lists = lists.get();
        fp.counts = counts.get();
        fp.bounds = bounds.get();
        fp.table = (const float*)ix.vec.values;
        fp.rowmap = compact ? (const unsigned*)rowmap_mem->ptr : nullptr;
        fp.queries = qf.get();
        fp.qnorm = qnorm.get();
        fp.xmax = ix.xmax;
        fp.ids = ids.get();
        fp.dist = dist.get();
        fp.fallback = fallback.get();
        fp.err_max = err.get();
        fp.err_sum = (double*)(err.get() + 1);
        fp.err_count = err.get() + 2;
        // Sized by the lists' capacity (not the largest one allowed), so
        // that several queries share an SM.
        int pool_cap = 2;
        while (pool_cap < cpg * cap) pool_cap <<= 1;
        pool_cap = std::min(pool_cap, kPoolMax);
        fp.pool_cap = pool_cap;
        fp.ex_cap = std::min(pool_cap, kExactMax);
        const size_t fsmem = (size_t)(fp.pool_cap + fp.ex_cap) * 8 + (size_t)dim * 4;
        if (fsmem + 12 * 1024 > b.smem_optin) fail(OXB_UNSUPPORTED, "vector dimension too large for the re-rank kernel");
        allow_smem(topk_final_kernel, fsmem);
        note_launch(), topk_final_kernel<<<nq, kFinalThreads, fsmem, s->stream>>>(fp);
        OXB_CUDA(cudaGetLastError());
        uint32_t hs = 0;
        OXB_CUDA(cudaMemcpyAsync(&hs, status.get(), 4, cudaMemcpyDeviceToHost, s->stream));
        OXB_CUDA(cudaMemcpyAsync(host_fb.data(), fallback.get(), (size_t)nq * 4, cudaMemcpyDeviceToHost, s->stream));
        unsigned long long he[3];
        OXB_CUDA(cudaMemcpyAsync(he, err.get(), sizeof he, cudaMemcpyDeviceToHost, s->stream));
        OXB_CUDA(cudaStreamSynchronize(s->stream));
        check_status_word(hs, "vector_topk scan");
        std::memcpy(&st.max_score_error, &he[0], 8);
        double sum;
        std::memcpy(&sum, &he[1], 8);
        st.reranked = (long long)he[2];
        st.mean_score_error = he[2] ? sum / (double)he[2] : 0.0;
    }
    // The exact path for the queries the fast path could not settle.
    Scratch<float> d;
    Scratch<unsigned long long> keys;
    for (int q = 0; q < nq; q++) {
        if (!host_fb[q]) continue;
        st.exact_queries++;
        if (n == 0) {
            note_launch(), topk_exact_out_kernel<<<1, 256, 0, s->stream>>>(nullptr, 0, k, ids.get() + (size_t)q * k,
                                                                          dist.get() + (size_t)q * k);
            continue;
        }
        if (!d.get()) {
            d = Scratch<float>(s, n);
            keys = Scratch<unsigned long long>(s, n);
        }
        launch_vector_distance(s, b, ix.vec, n, qf.get() + (size_t)q * dim, a.metric, d.get());
        DevLeaf ql = qleaf;
        if (ql.values) ql.lit = qlits_h[q];
        note_launch(), topk_exact_keys_kernel<<<grid_for(b, n, 256, 8), 256, 0, s->stream>>>(d.get(), selp,
                                                                                             ix.vec.validity, n, ql,
                                                                                             keys.get());
        radix_sort_pairs(s, b, keys.get(), nullptr, n, 64);
        note_launch(), topk_exact_out_kernel<<<1, 256, 0, s->stream>>>(keys.get(), n, k, ids.get() + (size_t)q * k,
                                                                       dist.get() + (size_t)q * k);
        OXB_CUDA(cudaGetLastError());
    }
    OXB_CUDA(cudaMemcpyAsync(out_ids, ids.get(), (size_t)nq * k * 8, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaMemcpyAsync(out_dist, dist.get(), (size_t)nq * k * 4, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaStreamSynchronize(s->stream));
    if (stats) *stats = st;
}

}  // namespace oxb
