// Grouped SUM / COUNT / MIN / MAX / AVG / COUNT(*) over one integer key
// (GpuBackend::aggregate, crates/oxidelake-device/src/backend.rs:166;
// semantics cpu/kernels.rs:478-818), and the fused inner-join probe ->
// WHERE -> GROUP BY form that runs a whole join + aggregate query in one
// pass over the probe side.
//
// Groups live in one open-addressing table in HBM: a key array (empty =
// kEmptyKey, claimed by one 64-bit CAS, so no publication wait is needed)
// and structure-of-arrays accumulators beside it.  Each CTA first folds its
// rows into a private table in shared memory — direct-mapped when the keys
// fall in a small range, hashed otherwise — and merges it into HBM when its
// rows are done; rows whose key does not fit go straight to HBM.
//
// Within a warp, lanes whose rows fall in the same group are combined first
// (__match_any_sync on the slot): one leader lane folds its peers' values
// and issues a single set of shared-memory atomics, so a Zipf-hot group
// costs one update per warp instead of one per row.  Aggregates over the
// same column share accumulators (SUM(x) and AVG(x) share one sum).
//
// Float64 sums: the leader's fold is an exact TwoSum chain, and every
// atomicAdd returns the old sum, so the rounding error of that very addition
// is recovered (TwoSum) and accumulated in a compensation array; the result
// is sum + compensation, O(eps) relative whatever order atomics land in.
// Int64 SUM wraps (unsigned add); MIN/MAX over Float64 follow totalOrder via
// integer keys, exactly as the reference.
#include <climits>
#include <map>

#include "async_copy.cuh"
#include "internal.h"

namespace oxb {

namespace {

constexpr int kMaxOuts = OXB_MAX_AGGREGATES;
constexpr int kMaxAccs = OXB_MAX_AGGREGATES;
constexpr int kMaxArrays = 1 + 2 * kMaxAccs;
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kSmemProbes = 16;
constexpr int kSlotNone = -1;    // the lane has no row to fold
constexpr int kSlotGlobal = -2;  // the row folds straight into HBM

enum : int { kAccCount = 1, kAccSumInt = 2, kAccSumF64 = 3, kAccMin = 4, kAccMax = 5 };
enum : unsigned char { kInitZero = 0, kInitMax = 1, kInitMin = 2 };
enum : unsigned char { kMergeAddU64 = 0, kMergeAddF64Comp = 1, kMergeAddF64 = 2, kMergeMin = 3, kMergeMax = 4 };

// One accumulator: what one column (of one side) contributes per row.
struct DevAcc {
    const void* values;
    const uint8_t* validity;
    int kind;
    int in_type;
    int side;  // 0: the input (probe) row, 1: the build row
    int arr;   // its array (a Float64 sum uses arr and arr + 1)
    // A Float64 sum whose CTA-table words hold a fixed-point window (the
    // fused join kernels only): fix = 1 and the window's unit 2^fix_lo.
    int fix;
    int fix_lo;
};

// One output column: the function, and where its value and count live.
struct DevOut {
    int func;
    int in_type;
    int arr;  // value array (COUNT: the count array)
    int nn;   // array counting the rows with a non-NULL input (0 = rows)
};

struct AggProgram {
    int nacc;
    DevAcc acc[kMaxAccs];
    int nout;
    DevOut out[kMaxOuts];
    int narrays;
    unsigned char init[kMaxArrays];
    unsigned char merge[kMaxArrays];
    long long* keys;          // capacity entries
    unsigned long long* arr;  // narrays * stride entries
    long long stride;         // capacity + 2: [capacity] NULL group, [capacity+1] key == kEmptyKey
    unsigned int capacity;
    int smem_slots;    // CTA table slots (power of two), 0 = none
    int scratch_accs;  // accumulators per lane in the warps' combining scratch
    int direct;        // CTA table indexed by key - direct_lo
    long long direct_lo;
    int wslots;        // slots of each warp's private cache (power of two), 0 = none
    int wdirect;       // warp caches indexed by key - wdirect_lo (else tagged by key)
    long long wdirect_lo;
    unsigned int* status;
    unsigned int probe_limit;  // a new key is refused a slot this far past its home
};

// While the host can still retry with a larger table, a new key is refused
// a slot more than kMaxInsertProbes slots past its home: at the planned
// load (at most 1/2) such a run has odds far below 1e-20 a key, and a table
// that the estimate left too small reaches it quickly.  A bound on the run
// instead of a count of placed keys: a shared counter bumped once per group
// serialises every insert of a many-group fold in one L2 slice.  The last
// attempt takes every slot (probe_limit = capacity).
constexpr unsigned kMaxInsertProbes = 256;

struct AggKey {
    const void* values;
    const uint8_t* validity;
    int type;
    int side;
};

__device__ __forceinline__ long long load_int(const void* v, int type, long long row) {
    return type == kInt64 ? __ldg((const long long*)v + row) : (long long)__ldg((const int*)v + row);
}

__device__ __forceinline__ double as_f64(unsigned long long u) { return __longlong_as_double((long long)u); }
__device__ __forceinline__ unsigned long long as_u64(double d) { return (unsigned long long)__double_as_longlong(d); }

// s + x with the rounding error of that addition added to *c (exact TwoSum);
// no error term once the sum is not finite.
__device__ __forceinline__ double two_sum_into(double s, double x, double* c) {
    double t = __dadd_rn(s, x);
    if (isfinite(t)) {
        double bp = __dsub_rn(t, s);
        *c = __dadd_rn(*c, __dadd_rn(__dsub_rn(s, __dsub_rn(t, bp)), __dsub_rn(x, bp)));
    }
    return t;
}

__device__ __forceinline__ void add_f64_comp(double* sum, double* comp, double x) {
    double old = atomicAdd(sum, x);
    double c = 0.0;
    two_sum_into(old, x, &c);
    if (c != 0.0) atomicAdd(comp, c);
}

// What accumulator `a` takes from one row (its identity when the value is NULL).
__device__ __forceinline__ unsigned long long contribution(const DevAcc& a, long long row_p, long long row_b) {
    const long long row = a.side ? row_b : row_p;
    const bool v = valid_at(a.validity, row);
    switch (a.kind) {
        case kAccCount:
            return v ? 1ull : 0ull;
        case kAccSumInt:
            return v ? (unsigned long long)load_int(a.values, a.in_type, row) : 0ull;
        case kAccSumF64: {
            double x = 0.0;
            if (v) x = a.in_type == kFloat64 ? __ldg((const double*)a.values + row) : (double)load_int(a.values, a.in_type, row);
            return as_u64(x);
        }
        case kAccMin:
            if (!v) return 0x7fffffffffffffffull;
            return (unsigned long long)(a.in_type == kFloat64 ? total_order_key(__ldg((const double*)a.values + row))
                                                              : load_int(a.values, a.in_type, row));
        default:
            if (!v) return 0x8000000000000000ull;
            return (unsigned long long)(a.in_type == kFloat64 ? total_order_key(__ldg((const double*)a.values + row))
                                                              : load_int(a.values, a.in_type, row));
    }
}

// The HBM slot of a key: [capacity] for NULL, [capacity + 1] for kEmptyKey.
__device__ __forceinline__ long long global_slot(const AggProgram& P, bool kvalid, long long key) {
    if (!kvalid) return P.capacity;
    if (key == kEmptyKey) return (long long)P.capacity + 1;
    unsigned int h = (unsigned int)(fmix64((unsigned long long)key) & (P.capacity - 1u));
    for (unsigned int p = 0; p < P.capacity; p++) {
        long long k = __ldcg(&P.keys[h]);
        if (k == key) return h;
        if (k == kEmptyKey) {
            if (p >= P.probe_limit) break;
            unsigned long long old = atomicCAS((unsigned long long*)&P.keys[h], (unsigned long long)kEmptyKey,
                                               (unsigned long long)key);
            if (old == (unsigned long long)kEmptyKey || old == (unsigned long long)key) return h;
        }
        h = (h + 1u) & (P.capacity - 1u);
    }
    atomicOr(P.status, kStatusTableFull);
    return -1;
}

// The private slot of a valid key (kSlotGlobal when it has none).
__device__ __forceinline__ int smem_slot(const AggProgram& P, long long key, long long* s_keys, int* s_fill) {
    const int S = P.smem_slots;
    if (S == 0 || key == kEmptyKey) return kSlotGlobal;
    if (P.direct) {
        unsigned long long d = (unsigned long long)(key - P.direct_lo);
        return d < (unsigned long long)S ? (int)d : kSlotGlobal;
    }
    unsigned int h = (unsigned int)(fmix64((unsigned long long)key) & (unsigned)(S - 1));
    for (int p = 0; p < kSmemProbes; p++) {
        long long k = ((volatile long long*)s_keys)[h];
        if (k == key) return (int)h;
        if (k == kEmptyKey) {
            if (*(volatile int*)s_fill >= S / 2) return kSlotGlobal;
            unsigned long long old =
                atomicCAS((unsigned long long*)&s_keys[h], (unsigned long long)kEmptyKey, (unsigned long long)key);
            if (old == (unsigned long long)kEmptyKey) {
                atomicAdd(s_fill, 1);
                return (int)h;
            }
            if ((long long)old == key) return (int)h;
        }
        h = (h + 1u) & (unsigned)(S - 1);
    }
    return kSlotGlobal;
}

// Shared memory of one CTA: its table (keys + arrays), each warp's private
// cache (tags + arrays), the warps' combining scratch, the table's fill.
struct SmemView {
    long long* keys;              // S (hash mode)
    unsigned long long* arr;      // narrays * S
    long long* wtags;             // kWarps * Sw (tagged mode)
    unsigned long long* warr;     // kWarps * narrays * Sw
    unsigned long long* scratch;  // kWarps * scratch_accs * 32
    int* fill;
};

__device__ __forceinline__ SmemView smem_view(const AggProgram& P, unsigned char* smem) {
    SmemView v;
    v.keys = (long long*)smem;
    v.arr = (unsigned long long*)(v.keys + P.smem_slots);
    v.wtags = (long long*)(v.arr + (long long)P.smem_slots * P.narrays);
    v.warr = (unsigned long long*)(v.wtags + kWarps * P.wslots);
    v.scratch = v.warr + (long long)kWarps * P.narrays * P.wslots;
    v.fill = (int*)(v.scratch + kWarps * P.scratch_accs * 32);
    return v;
}

size_t smem_bytes(int S, int Sw, int narrays, int scratch_accs) {
    return 8ull * ((size_t)S * (1 + narrays) + (size_t)kWarps * Sw * (1 + narrays) + (size_t)kWarps * scratch_accs * 32) +
           16;
}

__device__ __forceinline__ unsigned long long init_value(unsigned char tag) {
    return tag == kInitMax ? 0x7fffffffffffffffull : (tag == kInitMin ? 0x8000000000000000ull : 0ull);
}

__device__ void smem_init(const AggProgram& P, const SmemView& v) {
    const int S = P.smem_slots, W = kWarps * P.wslots;
    for (int i = threadIdx.x; i < S; i += blockDim.x) v.keys[i] = kEmptyKey;
    for (int i = threadIdx.x; i < S * P.narrays; i += blockDim.x) v.arr[i] = init_value(P.init[i / S]);
    for (int i = threadIdx.x; i < W; i += blockDim.x) v.wtags[i] = kEmptyKey;
    // warp w's cache: array a at warr[(w * narrays + a) * Sw]
    for (int i = threadIdx.x; i < W * P.narrays; i += blockDim.x) v.warr[i] = init_value(P.init[(i / P.wslots) % P.narrays]);
    if (threadIdx.x == 0) *v.fill = 0;
    __syncthreads();
}

// Folds combined values into the arrays at `slot`: `rows` rows, per
// accumulator its folded value and (Float64 sums) the folding error.
template <int MAXACC>
__device__ __forceinline__ void apply_vals(const AggProgram& P, unsigned long long* arr, long long stride,
                                           long long slot, unsigned long long rows, const unsigned long long* val,
                                           const double* comp) {
    atomicAdd(&arr[slot], rows);  // array 0: rows of the group
#pragma unroll
    for (int j = 0; j < MAXACC; j++) {
        if (j >= P.nacc) break;
        const DevAcc& a = P.acc[j];
        unsigned long long* p = arr + a.arr * stride + slot;
        switch (a.kind) {
            case kAccCount:
            case kAccSumInt:
                if (val[j]) atomicAdd(p, val[j]);
                break;
            case kAccSumF64: {
                double* c = (double*)(p + stride);
                add_f64_comp((double*)p, c, as_f64(val[j]));
                if (comp[j] != 0.0) atomicAdd(c, comp[j]);
                break;
            }
            case kAccMin:
                if (val[j] != 0x7fffffffffffffffull) atomicMin((long long*)p, (long long)val[j]);
                break;
            default:
                if (val[j] != 0x8000000000000000ull) atomicMax((long long*)p, (long long)val[j]);
                break;
        }
    }
}

// Folds `val` into accumulator value `x` the way kind `kind` combines.
__device__ __forceinline__ unsigned long long combine(int kind, unsigned long long acc, unsigned long long x,
                                                      double* comp) {
    switch (kind) {
        case kAccCount:
        case kAccSumInt: return acc + x;
        case kAccSumF64: return as_u64(two_sum_into(as_f64(acc), as_f64(x), comp));
        case kAccMin: return (long long)x < (long long)acc ? x : acc;
        default: return (long long)x > (long long)acc ? x : acc;
    }
}

// The slot of `key` in this warp's private cache, claiming a free one; -1
// when the key has none.  Only this warp touches its cache, and lanes with
// different keys that meet on one empty slot settle it with a CAS.
__device__ __forceinline__ int warp_cache_slot(const AggProgram& P, const SmemView& v, int warp, long long key) {
    const int Sw = P.wslots;
    if (Sw == 0) return -1;
    if (P.wdirect) {
        const unsigned long long d = (unsigned long long)(key - P.wdirect_lo);
        return d < (unsigned long long)Sw ? (int)d : -1;
    }
    long long* tags = v.wtags + warp * Sw;
    const int h = (int)(fmix64((unsigned long long)key) & (unsigned)(Sw - 1));
    const long long t = ((volatile long long*)tags)[h];
    if (t == key) return h;
    if (t != kEmptyKey) return -1;
    const unsigned long long old =
        atomicCAS((unsigned long long*)&tags[h], (unsigned long long)kEmptyKey, (unsigned long long)key);
    return (old == (unsigned long long)kEmptyKey || (long long)old == key) ? h : -1;
}

// One group's folded update (rows, values, folding errors) into the warp's
// cache (plain loads and stores: with lanes combined, one leader per key and
// warp writes a slot, and no other warp does), else the CTA table
// (atomics), else HBM.  Without combining the warp cache is skipped.
template <int MAXACC, bool WARP_CACHE>
__device__ __forceinline__ void update_group(const AggProgram& P, const SmemView& v, int warp, long long key,
                                             unsigned long long rows, const unsigned long long* val,
                                             const double* comp) {
    const int ws = WARP_CACHE ? warp_cache_slot(P, v, warp, key) : -1;
    if (ws >= 0) {
        const int Sw = P.wslots;
        unsigned long long* w = v.warr + (long long)warp * P.narrays * Sw + ws;
        w[0] += rows;
#pragma unroll
        for (int j = 0; j < MAXACC; j++) {
            if (j >= P.nacc) break;
            const DevAcc& a = P.acc[j];
            unsigned long long* p = w + a.arr * Sw;
            if (a.kind == kAccSumF64) {
                double c = as_f64(p[Sw]) + comp[j];
                *p = as_u64(two_sum_into(as_f64(*p), as_f64(val[j]), &c));
                p[Sw] = as_u64(c);
            } else {
                double unused = 0.0;
                *p = combine(a.kind, *p, val[j], &unused);
            }
        }
        return;
    }
    const int cs = smem_slot(P, key, v.keys, v.fill);
    if (cs >= 0) {
        apply_vals<MAXACC>(P, v.arr, P.smem_slots, cs, rows, val, comp);
        return;
    }
    const long long g = global_slot(P, true, key);
    if (g >= 0) apply_vals<MAXACC>(P, P.arr, P.stride, g, rows, val, comp);
}

// Folds one row (or nothing, when !live) of every lane of the warp; all 32
// lanes call it together.  MAXACC bounds P.nacc at compile time, so the
// per-accumulator values stay in registers.  With COMBINE, lanes of the same
// group are merged first (exact TwoSum for Float64) and one leader updates.
// NULL keys, and the key equal to kEmptyKey, fold straight into HBM.
template <int MAXACC, bool COMBINE>
__device__ __forceinline__ void fold(const AggProgram& P, const SmemView& v, bool live, bool kvalid, long long key,
                                     long long row_p, long long row_b) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long val[MAXACC];
    double comp[MAXACC];
#pragma unroll
    for (int j = 0; j < MAXACC; j++) {
        comp[j] = 0.0;
        val[j] = (j < P.nacc && live) ? contribution(P.acc[j], row_p, row_b) : 0ull;
    }
    const bool local = live && kvalid && key != kEmptyKey;
    if (COMBINE) {
        const unsigned locals = __ballot_sync(0xffffffffu, local);
        const unsigned peers = __match_any_sync(0xffffffffu, (unsigned long long)key) & locals;
        unsigned long long* mine = v.scratch + warp * MAXACC * 32;
        if (local) {
#pragma unroll
            for (int j = 0; j < MAXACC; j++)
                if (j < P.nacc) mine[j * 32 + lane] = val[j];
        }
        __syncwarp();
        if (local && lane == __ffs(peers) - 1) {
            for (unsigned m = peers & (peers - 1); m; m &= m - 1) {
                const int l = __ffs(m) - 1;
#pragma unroll
                for (int j = 0; j < MAXACC; j++) {
                    if (j >= P.nacc) break;
                    val[j] = combine(P.acc[j].kind, val[j], mine[j * 32 + l], &comp[j]);
                }
            }
            update_group<MAXACC, true>(P, v, warp, key, __popc(peers), val, comp);
        }
        __syncwarp();
    } else if (local) {
        update_group<MAXACC, false>(P, v, warp, key, 1, val, comp);
    }
    if (live && !local) {
        const long long g = global_slot(P, kvalid, key);
        if (g >= 0) apply_vals<MAXACC>(P, P.arr, P.stride, g, 1, val, comp);
    }
}

// Merges one slot's arrays (src, arrays `sstride` apart) into another slot
// (dst, arrays `dstride` apart) with atomics.
__device__ __forceinline__ void merge_slot(const AggProgram& P, const unsigned long long* src, long long sstride,
                                           unsigned long long* dst, long long dstride) {
    for (int a = 0; a < P.narrays; a++) {
        const unsigned long long x = src[a * sstride];
        unsigned long long* d = dst + a * dstride;
        switch (P.merge[a]) {
            case kMergeAddU64:
                if (x) atomicAdd(d, x);
                break;
            case kMergeAddF64Comp:
                add_f64_comp((double*)d, (double*)(d + dstride), as_f64(x));
                break;
            case kMergeAddF64:
                if (as_f64(x) != 0.0) atomicAdd((double*)d, as_f64(x));
                break;
            case kMergeMin:
                if ((long long)x != 0x7fffffffffffffffll) atomicMin((long long*)d, (long long)x);
                break;
            default:
                if ((long long)x != (long long)0x8000000000000000ull) atomicMax((long long*)d, (long long)x);
                break;
        }
    }
}

// Merges the warps' caches into the CTA table (or HBM), then the CTA table
// into HBM.
__device__ void smem_flush(const AggProgram& P, const SmemView& v) {
    __syncthreads();
    const int Sw = P.wslots;
    for (int i = threadIdx.x; i < kWarps * Sw; i += blockDim.x) {
        const int w = i / Sw, ws = i - w * Sw;
        const unsigned long long* src = v.warr + (long long)w * P.narrays * Sw + ws;
        if (src[0] == 0) continue;  // no rows in this slot
        const long long key = P.wdirect ? P.wdirect_lo + ws : v.wtags[i];
        const int cs = smem_slot(P, key, v.keys, v.fill);
        if (cs >= 0) {
            merge_slot(P, src, Sw, v.arr + cs, P.smem_slots);
        } else {
            const long long g = global_slot(P, true, key);
            if (g >= 0) merge_slot(P, src, Sw, P.arr + g, P.stride);
        }
    }
    __syncthreads();
    const int S = P.smem_slots;
    for (int i = threadIdx.x; i < S; i += blockDim.x) {
        if (v.arr[i] == 0) continue;  // no rows in this slot
        const long long key = P.direct ? P.direct_lo + i : v.keys[i];
        const long long g = global_slot(P, true, key);
        if (g < 0) continue;
        for (int a = 0; a < P.narrays; a++) {
            const unsigned long long x = v.arr[a * S + i];
            unsigned long long* dst = P.arr + a * P.stride + g;
            switch (P.merge[a]) {
                case kMergeAddU64:
                    if (x) atomicAdd(dst, x);
                    break;
                case kMergeAddF64Comp:
                    add_f64_comp((double*)dst, (double*)(dst + P.stride), as_f64(x));
                    break;
                case kMergeAddF64:
                    if (as_f64(x) != 0.0) atomicAdd((double*)dst, as_f64(x));
                    break;
                case kMergeMin:
                    if ((long long)x != 0x7fffffffffffffffll) atomicMin((long long*)dst, (long long)x);
                    break;
                default:
                    if ((long long)x != (long long)0x8000000000000000ull) atomicMax((long long*)dst, (long long)x);
                    break;
            }
        }
    }
}

// GROUP BY over the rows of one batch, with an optional fused WHERE; each
// thread takes RPT rows per step (their loads in flight together).
template <int MAXACC, bool COMBINE, int RPT>
__global__ void __launch_bounds__(kThreads) agg_rows_kernel(const __grid_constant__ AggProgram P,
                                                            const __grid_constant__ DevPredicate pred,
                                                            const __grid_constant__ AggKey key, long long n) {
    extern __shared__ __align__(128) unsigned char smem[];
    const SmemView v = smem_view(P, smem);
    if (P.smem_slots || P.wslots) smem_init(P, v);
    const long long step = (long long)gridDim.x * blockDim.x * RPT;
    for (long long base = blockIdx.x * (long long)blockDim.x * RPT; base < n; base += step) {
        bool live[RPT], kv[RPT];
        long long k[RPT];
#pragma unroll
        for (int r = 0; r < RPT; r++) {
            const long long i = base + r * (long long)blockDim.x + threadIdx.x;
            live[r] = i < n && (pred.nleaves == 0 || predicate_holds(pred, i));
            kv[r] = live[r] && valid_at(key.validity, i);
            k[r] = kv[r] ? load_int(key.values, key.type, i) : 0;
        }
#pragma unroll
        for (int r = 0; r < RPT; r++)
            fold<MAXACC, COMBINE>(P, v, live[r], kv[r], k[r], base + r * (long long)blockDim.x + threadIdx.x, 0);
    }
    if (P.smem_slots || P.wslots) smem_flush(P, v);
}

// A probe key's run: (start, count) and the run's first build row, which
// lives beside the slot and is loaded in parallel with it.
__device__ __forceinline__ bool jt_lookup(const JoinTableDev& t, long long key, unsigned int* start,
                                          unsigned int* count, unsigned int* first) {
    if (key == kEmptyKey) {
        *start = t.special_start;
        *count = t.special_count;
        *first = *count ? t.first_row[t.capacity] : 0u;
        return *count > 0;
    }
    unsigned int s = (unsigned int)(fmix64((unsigned long long)key) & (t.capacity - 1u));
    for (unsigned int p = 0; p < t.capacity; p++) {
        const int4 slot = __ldg((const int4*)&t.slots[s]);
        const unsigned int fr = __ldg(&t.first_row[s]);
        long long k = ((long long)(unsigned int)slot.y << 32) | (unsigned int)slot.x;
        if (k == key) {
            *start = (unsigned int)slot.z;
            *count = (unsigned int)slot.w;
            *first = fr;
            return true;
        }
        if (k == kEmptyKey) return false;
        s = (s + 1u) & (t.capacity - 1u);
    }
    return false;
}

// probe JOIN build ON key WHERE <probe leaves> GROUP BY <key of either side>:
// each lane looks up RPT probe rows at once (independent L2 chains), then
// walks each row's matches in build order; the warp steps through match
// m = 0, 1, ... together so its lanes can combine.
template <int MAXACC, bool COMBINE, int RPT>
__global__ void __launch_bounds__(kThreads) agg_join_kernel(const __grid_constant__ AggProgram P,
                                                            const __grid_constant__ DevPredicate pred,
                                                            const __grid_constant__ AggKey gkey,
                                                            const void* __restrict__ pk, const uint8_t* __restrict__ pkv,
                                                            int pk_type, const __grid_constant__ JoinTableDev jt,
                                                            long long n) {
    extern __shared__ __align__(128) unsigned char smem[];
    const SmemView v = smem_view(P, smem);
    if (P.smem_slots || P.wslots) smem_init(P, v);
    const long long step = (long long)gridDim.x * blockDim.x * RPT;
    for (long long base = blockIdx.x * (long long)blockDim.x * RPT; base < n; base += step) {
        unsigned int start[RPT], count[RPT], first[RPT];
#pragma unroll
        for (int r = 0; r < RPT; r++) {
            const long long i = base + r * (long long)blockDim.x + threadIdx.x;
            count[r] = 0;
            start[r] = first[r] = 0;
            if (i < n && (pred.nleaves == 0 || predicate_holds(pred, i)) && valid_at(pkv, i)) {
                if (!jt_lookup(jt, load_int(pk, pk_type, i), &start[r], &count[r], &first[r])) count[r] = 0;
            }
        }
#pragma unroll
        for (int r = 0; r < RPT; r++) {
            const long long i = base + r * (long long)blockDim.x + threadIdx.x;
            for (unsigned int m = 0; __any_sync(0xffffffffu, m < count[r]); m++) {
                const bool live = m < count[r];
                bool kv = false;
                long long k = 0, b = 0;
                if (live) {
                    b = m == 0 ? first[r] : jt.rows[start[r] + m];
                    const long long grow = gkey.side ? b : i;
                    kv = valid_at(gkey.validity, grow);
                    k = kv ? load_int(gkey.values, gkey.type, grow) : 0;
                }
                fold<MAXACC, COMBINE>(P, v, live, kv, k, i, b);
            }
        }
    }
    if (P.smem_slots || P.wslots) smem_flush(P, v);
}

// ---- tile sort-reduce ----------------------------------------------------
//
// A CTA folds its rows tile by tile (kTileRows rows).  Each row's slot in
// the CTA table is found, its rank within the slot taken with a native u32
// shared atomic, and its values scattered so that every slot's rows are
// contiguous (a counting sort in shared memory).  Each slot's run is then
// reduced by one thread — or, for runs of kBigRun rows or more (Zipf-hot
// groups), by a whole warp — with an exact TwoSum chain, and added to the
// slot's accumulators with plain loads and stores: one writer per slot per
// tile, no contention and no floating-point atomics.  Per row this costs a
// handful of instructions whatever the skew.

constexpr int kTileV = 4;                      // rows per thread per tile
constexpr int kTileRows = kThreads * kTileV;   // 1024
constexpr int kBigRun = 64;

struct TileView {
    long long* keys;          // S (hash mode)
    unsigned long long* arr;  // narrays * S
    unsigned int* cnt;        // S
    unsigned int* off;        // S
    unsigned long long* tval; // MAXACC * kTileRows
    unsigned int* big;        // kTileRows / kBigRun
    int* misc;                // [0] big runs, [1] table fill, [2..9] warp sums of the scan
};

size_t tile_smem_bytes(int S, int narrays, int maxacc) {
    return 8ull * S * (1 + narrays) + 8ull * S + 8ull * maxacc * kTileRows + 4ull * (kTileRows / kBigRun) + 64;
}

__device__ __forceinline__ TileView tile_view(const AggProgram& P, unsigned char* smem, int maxacc) {
    TileView t;
    const int S = P.smem_slots;
    t.keys = (long long*)smem;
    t.arr = (unsigned long long*)(t.keys + S);
    t.tval = t.arr + (long long)S * P.narrays;
    t.cnt = (unsigned int*)(t.tval + (long long)maxacc * kTileRows);
    t.off = t.cnt + S;
    t.big = t.off + S;
    t.misc = (int*)(t.big + kTileRows / kBigRun);
    return t;
}

// Adds a folded run (rows, values, folding errors) to CTA slot `b` (plain
// read-modify-write: the caller is the slot's only writer in this tile).
template <int MAXACC>
__device__ __forceinline__ void add_run(const AggProgram& P, const TileView& t, int b, unsigned long long rows,
                                        const unsigned long long* val, const double* comp) {
    const int S = P.smem_slots;
    t.arr[b] += rows;
#pragma unroll
    for (int j = 0; j < MAXACC; j++) {
        if (j >= P.nacc) break;
        const DevAcc& a = P.acc[j];
        unsigned long long* p = t.arr + a.arr * S + b;
        if (a.kind == kAccSumF64) {
            double c = as_f64(p[S]) + comp[j];
            *p = as_u64(two_sum_into(as_f64(*p), as_f64(val[j]), &c));
            p[S] = as_u64(c);
        } else {
            double unused = 0.0;
            *p = combine(a.kind, *p, val[j], &unused);
        }
    }
}

// Block-wide exclusive scan of the S slot counts into t.off.
__device__ __forceinline__ void scan_counts(const TileView& t, int S) {
    const int per = (S + kThreads - 1) / kThreads;
    const int lo = threadIdx.x * per, hi = min(lo + per, S);
    unsigned int s = 0;
    for (int b = lo; b < hi; b++) s += t.cnt[b];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned int x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    int* ws = t.misc + 2;
    if (lane == 31) ws[warp] = (int)x;
    __syncthreads();
    unsigned int before = 0;
    for (int w = 0; w < warp; w++) before += (unsigned int)ws[w];
    unsigned int run = before + x - s;
    for (int b = lo; b < hi; b++) {
        t.off[b] = run;
        run += t.cnt[b];
    }
}

// Reduces every slot's run of this tile into the CTA table and clears the
// counts for the next tile.
template <int MAXACC>
__device__ __forceinline__ void reduce_runs(const AggProgram& P, const TileView& t) {
    const int S = P.smem_slots;
    for (int b = threadIdx.x; b < S; b += blockDim.x) {
        const unsigned int c = t.cnt[b];
        if (c == 0) continue;
        if (c >= kBigRun) {
            t.big[atomicAdd(&t.misc[0], 1)] = b;
            continue;
        }
        const unsigned int o = t.off[b];
        unsigned long long val[MAXACC];
        double comp[MAXACC];
#pragma unroll
        for (int j = 0; j < MAXACC; j++) {
            comp[j] = 0.0;
            val[j] = j < P.nacc ? t.tval[j * kTileRows + o] : 0ull;
        }
        for (unsigned int e = 1; e < c; e++) {
#pragma unroll
            for (int j = 0; j < MAXACC; j++) {
                if (j >= P.nacc) break;
                val[j] = combine(P.acc[j].kind, val[j], t.tval[j * kTileRows + o + e], &comp[j]);
            }
        }
        add_run<MAXACC>(P, t, b, c, val, comp);
        t.cnt[b] = 0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nbig = t.misc[0];
    for (int r = warp; r < nbig; r += kWarps) {
        const int b = (int)t.big[r];
        const unsigned int c = t.cnt[b], o = t.off[b];
        unsigned long long val[MAXACC];
        double comp[MAXACC];
        bool any = false;
#pragma unroll
        for (int j = 0; j < MAXACC; j++) comp[j] = 0.0;
        for (unsigned int e = lane; e < c; e += 32) {
#pragma unroll
            for (int j = 0; j < MAXACC; j++) {
                if (j >= P.nacc) break;
                const unsigned long long x = t.tval[j * kTileRows + o + e];
                val[j] = any ? combine(P.acc[j].kind, val[j], x, &comp[j]) : x;
            }
            any = true;
        }
        // every lane holds at least one element (c >= kBigRun >= 32)
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
#pragma unroll
            for (int j = 0; j < MAXACC; j++) {
                if (j >= P.nacc) break;
                const unsigned long long x = __shfl_xor_sync(0xffffffffu, val[j], d);
                const double xc = __shfl_xor_sync(0xffffffffu, comp[j], d);
                if (P.acc[j].kind == kAccSumF64) comp[j] += xc;
                val[j] = combine(P.acc[j].kind, val[j], x, &comp[j]);
            }
        }
        if (lane == 0) {
            add_run<MAXACC>(P, t, b, c, val, comp);
            t.cnt[b] = 0;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) t.misc[0] = 0;
    __syncthreads();
}

// One round of a tile: the rows (`live`, key, contributing rows) each lane
// holds for its kTileV positions.
template <int MAXACC>
__device__ __forceinline__ void tile_round(const AggProgram& P, const TileView& t, const bool* live, const bool* kv,
                                           const long long* key, const long long* row_p, const long long* row_b) {
    int slot[kTileV];
    unsigned int rank[kTileV];
    unsigned long long val[kTileV][MAXACC];
#pragma unroll
    for (int v = 0; v < kTileV; v++) {
        slot[v] = kSlotNone;
        if (!live[v]) continue;
#pragma unroll
        for (int j = 0; j < MAXACC; j++) val[v][j] = j < P.nacc ? contribution(P.acc[j], row_p[v], row_b[v]) : 0ull;
        slot[v] = (kv[v] && key[v] != kEmptyKey) ? smem_slot(P, key[v], t.keys, t.misc + 1) : kSlotGlobal;
        if (slot[v] >= 0) {
            rank[v] = atomicAdd(&t.cnt[slot[v]], 1u);
        } else {
            double comp[MAXACC];
#pragma unroll
            for (int j = 0; j < MAXACC; j++) comp[j] = 0.0;
            const long long g = global_slot(P, kv[v], key[v]);
            if (g >= 0) apply_vals<MAXACC>(P, P.arr, P.stride, g, 1, val[v], comp);
        }
    }
    __syncthreads();
    scan_counts(t, P.smem_slots);
    __syncthreads();
#pragma unroll
    for (int v = 0; v < kTileV; v++) {
        if (slot[v] < 0) continue;
        const unsigned int pos = t.off[slot[v]] + rank[v];
#pragma unroll
        for (int j = 0; j < MAXACC; j++)
            if (j < P.nacc) t.tval[j * kTileRows + pos] = val[v][j];
    }
    __syncthreads();
    reduce_runs<MAXACC>(P, t);
}

template <int MAXACC>
__device__ void tile_init(const AggProgram& P, const TileView& t) {
    const int S = P.smem_slots;
    for (int i = threadIdx.x; i < S; i += blockDim.x) {
        t.keys[i] = kEmptyKey;
        t.cnt[i] = 0;
    }
    for (int i = threadIdx.x; i < S * P.narrays; i += blockDim.x) t.arr[i] = init_value(P.init[i / S]);
    if (threadIdx.x < 16) t.misc[threadIdx.x] = 0;
    __syncthreads();
}

template <int MAXACC>
__device__ void tile_flush(const AggProgram& P, const TileView& t) {
    __syncthreads();
    const int S = P.smem_slots;
    for (int i = threadIdx.x; i < S; i += blockDim.x) {
        if (t.arr[i] == 0) continue;  // no rows in this slot
        const long long key = P.direct ? P.direct_lo + i : t.keys[i];
        const long long g = global_slot(P, true, key);
        if (g >= 0) merge_slot(P, t.arr + i, S, P.arr + g, P.stride);
    }
}

template <int MAXACC>
__global__ void __launch_bounds__(kThreads) agg_tile_rows_kernel(const __grid_constant__ AggProgram P,
                                                                 const __grid_constant__ DevPredicate pred,
                                                                 const __grid_constant__ AggKey key, long long n) {
    extern __shared__ __align__(128) unsigned char smem[];
    const TileView t = tile_view(P, smem, MAXACC);
    tile_init<MAXACC>(P, t);
    for (long long base = blockIdx.x * (long long)kTileRows; base < n; base += (long long)gridDim.x * kTileRows) {
        bool live[kTileV], kv[kTileV];
        long long k[kTileV], rp[kTileV], rb[kTileV];
#pragma unroll
        for (int v = 0; v < kTileV; v++) {
            const long long i = base + v * (long long)kThreads + threadIdx.x;
            rp[v] = i;
            rb[v] = 0;
            live[v] = i < n && (pred.nleaves == 0 || predicate_holds(pred, i));
            kv[v] = live[v] && valid_at(key.validity, i);
            k[v] = kv[v] ? load_int(key.values, key.type, i) : 0;
        }
        tile_round<MAXACC>(P, t, live, kv, k, rp, rb);
    }
    tile_flush<MAXACC>(P, t);
}

template <int MAXACC>
__global__ void __launch_bounds__(kThreads) agg_tile_join_kernel(const __grid_constant__ AggProgram P,
                                                                 const __grid_constant__ DevPredicate pred,
                                                                 const __grid_constant__ AggKey gkey,
                                                                 const void* __restrict__ pk,
                                                                 const uint8_t* __restrict__ pkv, int pk_type,
                                                                 const __grid_constant__ JoinTableDev jt, long long n) {
    extern __shared__ __align__(128) unsigned char smem[];
    const TileView t = tile_view(P, smem, MAXACC);
    tile_init<MAXACC>(P, t);
    for (long long base = blockIdx.x * (long long)kTileRows; base < n; base += (long long)gridDim.x * kTileRows) {
        unsigned int start[kTileV], count[kTileV], first[kTileV];
        unsigned int most = 0;
#pragma unroll
        for (int v = 0; v < kTileV; v++) {
            const long long i = base + v * (long long)kThreads + threadIdx.x;
            count[v] = 0;
            start[v] = first[v] = 0;
            if (i < n && (pred.nleaves == 0 || predicate_holds(pred, i)) && valid_at(pkv, i)) {
                if (!jt_lookup(jt, load_int(pk, pk_type, i), &start[v], &count[v], &first[v])) count[v] = 0;
            }
            most = max(most, count[v]);
        }
        // Round m folds every row's m-th match (rows matching one build row: one round).
        for (unsigned int m = 0; __syncthreads_or(m < most); m++) {
            bool live[kTileV], kv[kTileV];
            long long k[kTileV], rp[kTileV], rb[kTileV];
#pragma unroll
            for (int v = 0; v < kTileV; v++) {
                rp[v] = base + v * (long long)kThreads + threadIdx.x;
                live[v] = m < count[v];
                rb[v] = live[v] ? (m == 0 ? first[v] : jt.rows[start[v] + m]) : 0;
                const long long grow = gkey.side ? rb[v] : rp[v];
                kv[v] = live[v] && valid_at(gkey.validity, grow);
                k[v] = kv[v] ? load_int(gkey.values, gkey.type, grow) : 0;
            }
            tile_round<MAXACC>(P, t, live, kv, k, rp, rb);
        }
    }
    tile_flush<MAXACC>(P, t);
}

// ---- streamed row loop ----------------------------------------------------
//
// One producer warp streams every input column the query reads from the
// probe side (predicate, keys, aggregate inputs, validity bitmaps) into a
// ring of kStages shared-memory stages with 1-D bulk copies (TMA), kStreamT
// rows per stage, completing on an mbarrier; kConsumerWarps warps fold the
// rows from shared memory.  One thread keeps ~kStages x 20 KB per CTA in
// flight, which is what saturates HBM; the consumers see shared-memory
// latency for the columns and spend their instructions on the fold.  A tile
// whose columns are not whole 16-byte pieces (the last, partial one) is read
// straight from global memory instead.  All waits are bounded.
//
// The CTA table is slot-major ("aos" arrays per slot) so a Float64 sum and
// its compensation sit in one aligned 16-byte pair, updated together by a
// 128-bit compare-and-swap with an exact TwoSum: compensated partials for
// the price of one atomic.

constexpr int kStreamT = 1024;  // rows per stage
constexpr int kConsumerWarps = 8;
constexpr int kStreamThreads = 32 * (1 + kConsumerWarps);
constexpr int kStages = 3;
constexpr int kMaxStreamCols = 8;

struct StreamCol {
    const void* values;
    const uint8_t* validity;
    int width;  // bytes per row: 4 or 8
    int type;
    int voff;   // offset of the values within a stage
    int boff;   // offset of the validity bits within a stage (-1: none)
};

struct StreamPlan {
    int ncols;
    StreamCol cols[kMaxStreamCols];
    int stage_bytes;
    int tx_bytes;  // bytes the bulk copies of one full stage deliver
    long long n, ntiles;
    int leaf_col[kMaxLeaves];  // stream column of each predicate leaf
    int acc_col[kMaxAccs];     // stream column of each probe-side accumulator, -1 otherwise
    int key_col;               // group key (plain aggregate) or probe key (join)
    int aos;                   // 8-byte words per CTA-table slot (even)
    int aos_idx[kMaxArrays];   // word of each accumulator array within a slot
};

struct StreamView {
    unsigned char* stages;
    unsigned long long* full;
    unsigned long long* empty;
    int* direct;
    long long* keys;          // S (hash mode)
    unsigned long long* tab;  // S * aos
    int* fill;
    int* abort;
};

size_t stream_smem_bytes(int S, int stage_bytes, int aos) {
    return (size_t)kStages * stage_bytes + 16 * kStages + 16 * kStages + 16 + 8ull * S * (1 + aos) + 64;
}

__device__ __forceinline__ StreamView stream_view(const AggProgram& P, const StreamPlan& SP, unsigned char* smem) {
    StreamView v;
    v.stages = smem;
    unsigned char* p = smem + (size_t)kStages * SP.stage_bytes;
    v.full = (unsigned long long*)p;
    v.empty = v.full + kStages;
    v.direct = (int*)(v.empty + kStages);
    p = (unsigned char*)(v.direct + 4 * kStages);
    p = (unsigned char*)(((uintptr_t)p + 15) & ~(uintptr_t)15);
    v.keys = (long long*)p;
    v.tab = (unsigned long long*)(v.keys + P.smem_slots);
    v.fill = (int*)(v.tab + (long long)P.smem_slots * SP.aos);
    v.abort = v.fill + 1;
    return v;
}

// Column c of tile row r: from the stage, or (direct tiles) from global row g.
__device__ __forceinline__ long long stream_raw(const StreamPlan& SP, int c, const unsigned char* stage, bool direct,
                                                long long g, int r) {
    const StreamCol& col = SP.cols[c];
    if (!direct) {
        const unsigned char* q = stage + col.voff + (size_t)r * col.width;
        return col.width == 8 ? *(const long long*)q : (long long)*(const int*)q;
    }
    return col.width == 8 ? __ldcs((const long long*)col.values + g) : (long long)__ldcs((const int*)col.values + g);
}

__device__ __forceinline__ bool stream_valid(const StreamPlan& SP, int c, const unsigned char* stage, bool direct,
                                             long long g, int r) {
    const StreamCol& col = SP.cols[c];
    if (!col.validity) return true;
    if (!direct) return (stage[col.boff + (r >> 3)] >> (r & 7)) & 1;
    return valid_at(col.validity, g);
}

__device__ __forceinline__ bool stream_predicate(const DevPredicate& pred, const StreamPlan& SP,
                                                 const unsigned char* stage, bool direct, long long g, int r) {
    for (int l = 0; l < pred.nleaves; l++) {
        const int c = SP.leaf_col[l];
        if (!stream_valid(SP, c, stage, direct, g, r)) return false;
        const long long raw = stream_raw(SP, c, stage, direct, g, r);
        const long long a = pred.leaves[l].type == kFloat64 ? filter_order_key(__longlong_as_double(raw)) : raw;
        if (!cmp_holds(pred.leaves[l].op, a, pred.leaves[l].lit)) return false;
    }
    return true;
}

// What an accumulator takes from a value (its identity when NULL).
__device__ __forceinline__ unsigned long long contribution_raw(int kind, int in_type, bool valid, long long raw) {
    switch (kind) {
        case kAccCount: return valid ? 1ull : 0ull;
        case kAccSumInt: return valid ? (unsigned long long)raw : 0ull;
        case kAccSumF64:
            if (!valid) return 0ull;
            return in_type == kFloat64 ? (unsigned long long)raw : as_u64((double)raw);
        case kAccMin:
            if (!valid) return 0x7fffffffffffffffull;
            return (unsigned long long)(in_type == kFloat64 ? total_order_key(__longlong_as_double(raw)) : raw);
        default:
            if (!valid) return 0x8000000000000000ull;
            return (unsigned long long)(in_type == kFloat64 ? total_order_key(__longlong_as_double(raw)) : raw);
    }
}

// Folds one row's values into CTA slot `slot` (slot-major table).
template <int MAXACC>
__device__ __forceinline__ void stream_apply(const AggProgram& P, const StreamPlan& SP, const StreamView& v,
                                             int slot, const unsigned long long* val) {
    unsigned long long* t = v.tab + (long long)slot * SP.aos;
    atomicAdd(&t[SP.aos_idx[0]], 1ull);
#pragma unroll
    for (int j = 0; j < MAXACC; j++) {
        if (j >= P.nacc) break;
        const DevAcc& a = P.acc[j];
        unsigned long long* p = t + SP.aos_idx[a.arr];
        switch (a.kind) {
            case kAccCount:
            case kAccSumInt:
                if (val[j]) atomicAdd(p, val[j]);
                break;
            case kAccSumF64: {
                const double x = as_f64(val[j]);
                unsigned long long s = p[0], c = p[1];
                int tries = 0;
                for (; tries < (1 << 20); tries++) {
                    double cs = as_f64(c);
                    const double ns = two_sum_into(as_f64(s), x, &cs);
                    unsigned long long os, oc;
                    cas128_shared(smem_addr(p), s, c, as_u64(ns), as_u64(cs), &os, &oc);
                    if (os == s && oc == c) break;
                    s = os;
                    c = oc;
                }
                if (tries == (1 << 20)) atomicOr(P.status, kStatusTimeout);
                break;
            }
            case kAccMin:
                if (val[j] != 0x7fffffffffffffffull) atomicMin((long long*)p, (long long)val[j]);
                break;
            default:
                if (val[j] != 0x8000000000000000ull) atomicMax((long long*)p, (long long)val[j]);
                break;
        }
    }
}

// One row: its group key (valid or not) and values, folded into the CTA
// table, or straight into HBM when the key has no slot there.
template <int MAXACC>
__device__ __forceinline__ void stream_fold(const AggProgram& P, const StreamPlan& SP, const StreamView& v,
                                            bool kvalid, long long key, const unsigned long long* val) {
    const int slot = (kvalid && key != kEmptyKey) ? smem_slot(P, key, v.keys, v.fill) : kSlotGlobal;
    if (slot >= 0) {
        stream_apply<MAXACC>(P, SP, v, slot, val);
    } else {
        double comp[MAXACC];
#pragma unroll
        for (int j = 0; j < MAXACC; j++) comp[j] = 0.0;
        const long long g = global_slot(P, kvalid, key);
        if (g >= 0) apply_vals<MAXACC>(P, P.arr, P.stride, g, 1, val, comp);
    }
}

__device__ void stream_init(const AggProgram& P, const StreamPlan& SP, const StreamView& v) {
    const int S = P.smem_slots;
    for (int i = threadIdx.x; i < S; i += blockDim.x) v.keys[i] = kEmptyKey;
    for (int i = threadIdx.x; i < S * SP.aos; i += blockDim.x) {
        const int w = i % SP.aos;
        unsigned long long x = 0;
        for (int a = 0; a < P.narrays; a++)
            if (SP.aos_idx[a] == w) x = init_value(P.init[a]);
        v.tab[i] = x;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) {
            mbar_init(&v.full[s], 1);
            mbar_init(&v.empty[s], kConsumerWarps);
        }
        *v.fill = 0;
        *v.abort = 0;
        fence_barrier_init();
    }
    __syncthreads();
}

// Merges the CTA table into HBM.
__device__ void stream_flush(const AggProgram& P, const StreamPlan& SP, const StreamView& v) {
    __syncthreads();
    const int S = P.smem_slots;
    for (int i = threadIdx.x; i < S; i += blockDim.x) {
        const unsigned long long* t = v.tab + (long long)i * SP.aos;
        if (t[SP.aos_idx[0]] == 0) continue;  // no rows in this slot
        const long long key = P.direct ? P.direct_lo + i : v.keys[i];
        const long long g = global_slot(P, true, key);
        if (g < 0) continue;
        for (int a = 0; a < P.narrays; a++) {
            const unsigned long long x = t[SP.aos_idx[a]];
            unsigned long long* d = P.arr + a * P.stride + g;
            switch (P.merge[a]) {
                case kMergeAddU64:
                    if (x) atomicAdd(d, x);
                    break;
                case kMergeAddF64Comp:
                    add_f64_comp((double*)d, (double*)(d + P.stride), as_f64(x));
                    break;
                case kMergeAddF64:
                    if (as_f64(x) != 0.0) atomicAdd((double*)d, as_f64(x));
                    break;
                case kMergeMin:
                    if ((long long)x != 0x7fffffffffffffffll) atomicMin((long long*)d, (long long)x);
                    break;
                default:
                    if ((long long)x != (long long)0x8000000000000000ull) atomicMax((long long*)d, (long long)x);
                    break;
            }
        }
    }
}

// The producer: one lane streams this CTA's tiles into the stage ring.
__device__ void stream_produce(const AggProgram& P, const StreamPlan& SP, const StreamView& v) {
    const unsigned long long pol = policy_evict_first();
    int it = 0;
    for (long long tile = blockIdx.x; tile < SP.ntiles; tile += gridDim.x, it++) {
        const int st = it % kStages;
        if (it >= kStages && !mbar_wait(&v.empty[st], ((it / kStages) - 1) & 1)) {
            atomicOr(P.status, kStatusTimeout);
            *(volatile int*)v.abort = 1;
            break;
        }
        if (*(volatile int*)v.abort) break;
        const long long base = tile * kStreamT;
        const bool direct = SP.n - base < kStreamT;
        v.direct[st] = direct;
        if (direct) {
            mbar_arrive(&v.full[st]);
            continue;
        }
        unsigned char* stage = v.stages + (size_t)st * SP.stage_bytes;
        mbar_arrive_expect_tx(&v.full[st], (unsigned)SP.tx_bytes);
        for (int c = 0; c < SP.ncols; c++) {
            const StreamCol& col = SP.cols[c];
            bulk_copy_g2s(stage + col.voff, (const unsigned char*)col.values + base * col.width,
                          (unsigned)(kStreamT * col.width), &v.full[st], pol);
            if (col.validity)
                bulk_copy_g2s(stage + col.boff, col.validity + base / 8, kStreamT / 8, &v.full[st], pol);
        }
    }
    // Before leaving, wait for the copies still landing in this CTA's stages.
    for (int k = 1; k <= kStages && k <= it; k++) {
        const int use = it - k;
        mbar_wait(&v.full[use % kStages], (use / kStages) & 1);
    }
}

template <int MAXACC>
__global__ void __launch_bounds__(kStreamThreads) agg_stream_rows_kernel(const __grid_constant__ AggProgram P,
                                                                         const __grid_constant__ DevPredicate pred,
                                                                         const __grid_constant__ StreamPlan SP) {
    extern __shared__ __align__(128) unsigned char smem[];
    const StreamView v = stream_view(P, SP, smem);
    stream_init(P, SP, v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        if (lane == 0) stream_produce(P, SP, v);
        __syncwarp();
    } else {
        const int ct = threadIdx.x - 32;
        int it = 0;
        for (long long tile = blockIdx.x; tile < SP.ntiles; tile += gridDim.x, it++) {
            const int st = it % kStages;
            if (!mbar_wait(&v.full[st], (it / kStages) & 1) || *(volatile int*)v.abort) {
                atomicOr(P.status, kStatusTimeout);
                *(volatile int*)v.abort = 1;
                break;
            }
            const bool direct = v.direct[st];
            const unsigned char* stage = v.stages + (size_t)st * SP.stage_bytes;
#pragma unroll
            for (int k = 0; k < kStreamT / (32 * kConsumerWarps); k++) {
                const int r = ct + k * 32 * kConsumerWarps;
                const long long g = tile * kStreamT + r;
                if (g >= SP.n) continue;
                if (pred.nleaves && !stream_predicate(pred, SP, stage, direct, g, r)) continue;
                const bool kv = stream_valid(SP, SP.key_col, stage, direct, g, r);
                const long long key = kv ? stream_raw(SP, SP.key_col, stage, direct, g, r) : 0;
                unsigned long long val[MAXACC];
#pragma unroll
                for (int j = 0; j < MAXACC; j++) {
                    if (j >= P.nacc) break;
                    const int c = SP.acc_col[j];
                    val[j] = contribution_raw(P.acc[j].kind, P.acc[j].in_type, stream_valid(SP, c, stage, direct, g, r),
                                              stream_raw(SP, c, stage, direct, g, r));
                }
                stream_fold<MAXACC>(P, SP, v, kv, key, val);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&v.empty[st]);
        }
    }
    stream_flush(P, SP, v);
}

template <int MAXACC>
__global__ void __launch_bounds__(kStreamThreads) agg_stream_join_kernel(const __grid_constant__ AggProgram P,
                                                                         const __grid_constant__ DevPredicate pred,
                                                                         const __grid_constant__ StreamPlan SP,
                                                                         const __grid_constant__ AggKey gkey,
                                                                         const __grid_constant__ JoinTableDev jt) {
    extern __shared__ __align__(128) unsigned char smem[];
    const StreamView v = stream_view(P, SP, smem);
    stream_init(P, SP, v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        if (lane == 0) stream_produce(P, SP, v);
        __syncwarp();
    } else {
        const unsigned long long keep = policy_evict_last();
        const int ct = threadIdx.x - 32;
        constexpr int kRows = kStreamT / (32 * kConsumerWarps);
        int it = 0;
        for (long long tile = blockIdx.x; tile < SP.ntiles; tile += gridDim.x, it++) {
            const int st = it % kStages;
            if (!mbar_wait(&v.full[st], (it / kStages) & 1) || *(volatile int*)v.abort) {
                atomicOr(P.status, kStatusTimeout);
                *(volatile int*)v.abort = 1;
                break;
            }
            const bool direct = v.direct[st];
            const unsigned char* stage = v.stages + (size_t)st * SP.stage_bytes;
            // Look every row's key up first: kRows independent L2 chains.
            unsigned int start[kRows], count[kRows], first[kRows];
#pragma unroll
            for (int k = 0; k < kRows; k++) {
                const int r = ct + k * 32 * kConsumerWarps;
                const long long g = tile * kStreamT + r;
                count[k] = 0;
                start[k] = first[k] = 0;
                if (g >= SP.n) continue;
                if (pred.nleaves && !stream_predicate(pred, SP, stage, direct, g, r)) continue;
                if (!stream_valid(SP, SP.key_col, stage, direct, g, r)) continue;
                const long long pkey = stream_raw(SP, SP.key_col, stage, direct, g, r);
                if (pkey == kEmptyKey) {
                    start[k] = jt.special_start;
                    count[k] = jt.special_count;
                    first[k] = count[k] ? jt.first_row[jt.capacity] : 0u;
                    continue;
                }
                unsigned int s = (unsigned int)(fmix64((unsigned long long)pkey) & (jt.capacity - 1u));
                for (unsigned int p = 0; p < jt.capacity; p++) {
                    const int4 slot = ld_keep_v4(&jt.slots[s], keep);
                    const unsigned int fr = ld_keep_u32(&jt.first_row[s], keep);
                    const long long sk = ((long long)(unsigned int)slot.y << 32) | (unsigned int)slot.x;
                    if (sk == pkey) {
                        start[k] = (unsigned int)slot.z;
                        count[k] = (unsigned int)slot.w;
                        first[k] = fr;
                        break;
                    }
                    if (sk == kEmptyKey) break;
                    s = (s + 1u) & (jt.capacity - 1u);
                }
            }
#pragma unroll
            for (int k = 0; k < kRows; k++) {
                const int r = ct + k * 32 * kConsumerWarps;
                const long long g = tile * kStreamT + r;
                for (unsigned int m = 0; m < count[k]; m++) {
                    const long long b = m == 0 ? first[k] : jt.rows[start[k] + m];
                    const long long grow = gkey.side ? b : g;
                    bool kv;
                    long long key;
                    if (gkey.side) {
                        kv = valid_at(gkey.validity, grow);
                        key = kv ? (gkey.type == kInt64 ? ld_keep_s64((const long long*)gkey.values + grow, keep)
                                                        : (long long)(int)ld_keep_u32((const int*)gkey.values + grow, keep))
                                 : 0;
                    } else {
                        kv = valid_at(gkey.validity, grow);
                        key = kv ? load_int(gkey.values, gkey.type, grow) : 0;
                    }
                    unsigned long long val[MAXACC];
#pragma unroll
                    for (int j = 0; j < MAXACC; j++) {
                        if (j >= P.nacc) break;
                        const DevAcc& a = P.acc[j];
                        const int c = SP.acc_col[j];
                        if (c >= 0) {
                            val[j] = contribution_raw(a.kind, a.in_type, stream_valid(SP, c, stage, direct, g, r),
                                                      stream_raw(SP, c, stage, direct, g, r));
                        } else {
                            val[j] = contribution(a, g, b);
                        }
                    }
                    stream_fold<MAXACC>(P, SP, v, kv, key, val);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&v.empty[st]);
        }
    }
    stream_flush(P, SP, v);
}

// ---- streamed tile sort-reduce ----------------------------------------------
//
// The producer warp streams the columns as above; the consumer warps take
// a stage's rows into registers and release the stage at once (so the next
// copies overlap the rest of the tile), then counting-sort the rows by CTA
// slot in shared memory and reduce each slot's run with one writer per slot
// (a thread, or a warp for runs of kBigRun rows or more): no atomics on the
// accumulators, no contention whatever the skew, compensated Float64 sums.
// Only the consumer warps meet at their barriers (named barrier 1).

constexpr int kSTRows = kStreamT / (32 * kConsumerWarps);  // rows per consumer thread per stage

__device__ __forceinline__ void consumer_sync() {
    asm volatile("bar.sync 1, %0;" ::"n"(32 * kConsumerWarps) : "memory");
}

// A consumer-warps barrier that also ORs a flag across them.
__device__ __forceinline__ bool consumer_sync_or(bool x) {
    unsigned r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, 1, %2, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((unsigned)x), "n"(32 * kConsumerWarps)
        : "memory");
    return r != 0;
}

struct STView {
    unsigned char* stages;
    unsigned long long* full;
    unsigned long long* empty;
    int* direct;
    long long* keys;           // S (hash mode)
    unsigned long long* arr;   // narrays * S
    unsigned long long* tval;  // maxacc * kStreamT
    unsigned int* cnt;         // S
    unsigned int* off;         // S
    unsigned int* big;         // kStreamT / kBigRun
    int* misc;                 // [0] big runs, [1] table fill, [2..9] scan warp sums, [10] abort
};

size_t stile_smem_bytes(int S, int stage_bytes, int narrays, int maxacc) {
    return (size_t)kStages * stage_bytes + 16 * kStages + 16 * kStages + 16 + 8ull * S * (1 + narrays) +
           8ull * maxacc * kStreamT + 8ull * S + 4ull * (kStreamT / kBigRun) + 64;
}

__device__ __forceinline__ STView stile_view(const AggProgram& P, const StreamPlan& SP, unsigned char* smem,
                                             int maxacc) {
    STView v;
    const int S = P.smem_slots;
    v.stages = smem;
    unsigned char* p = smem + (size_t)kStages * SP.stage_bytes;
    v.full = (unsigned long long*)p;
    v.empty = v.full + kStages;
    v.direct = (int*)(v.empty + kStages);
    p = (unsigned char*)(v.direct + 4 * kStages);
    p = (unsigned char*)(((uintptr_t)p + 15) & ~(uintptr_t)15);
    v.keys = (long long*)p;
    v.arr = (unsigned long long*)(v.keys + S);
    v.tval = v.arr + (long long)S * P.narrays;
    v.cnt = (unsigned int*)(v.tval + (long long)maxacc * kStreamT);
    v.off = v.cnt + S;
    v.big = v.off + S;
    v.misc = (int*)(v.big + kStreamT / kBigRun);
    return v;
}

// add_run over the stream-tile layout.
template <int MAXACC>
__device__ __forceinline__ void st_add_run(const AggProgram& P, const STView& v, int b, unsigned long long rows,
                                           const unsigned long long* val, const double* comp) {
    const int S = P.smem_slots;
    v.arr[b] += rows;
#pragma unroll
    for (int j = 0; j < MAXACC; j++) {
        if (j >= P.nacc) break;
        const DevAcc& a = P.acc[j];
        unsigned long long* p = v.arr + a.arr * S + b;
        if (a.kind == kAccSumF64) {
            double c = as_f64(p[S]) + comp[j];
            *p = as_u64(two_sum_into(as_f64(*p), as_f64(val[j]), &c));
            p[S] = as_u64(c);
        } else {
            double unused = 0.0;
            *p = combine(a.kind, *p, val[j], &unused);
        }
    }
}

// One tile round among the consumer threads (ct in 0..255): rank every row
// in its slot, scan the counts, scatter, reduce the runs.
template <int MAXACC>
__device__ __forceinline__ void st_round(const AggProgram& P, const STView& v, int ct, const int* slot,
                                         unsigned long long (*val)[MAXACC]) {
    const int S = P.smem_slots;
    unsigned int rank[kSTRows];
#pragma unroll
    for (int k = 0; k < kSTRows; k++)
        if (slot[k] >= 0) rank[k] = atomicAdd(&v.cnt[slot[k]], 1u);
    consumer_sync();
    {  // exclusive scan of the counts
        const int nt = 32 * kConsumerWarps;
        const int per = (S + nt - 1) / nt;
        const int lo = ct * per, hi = min(lo + per, S);
        unsigned int sum = 0;
        for (int b = lo; b < hi; b++) sum += v.cnt[b];
        const int lane = ct & 31, w = ct >> 5;
        unsigned int x = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) v.misc[2 + w] = (int)x;
        consumer_sync();
        unsigned int run = x - sum;
        for (int q = 0; q < w; q++) run += (unsigned int)v.misc[2 + q];
        for (int b = lo; b < hi; b++) {
            v.off[b] = run;
            run += v.cnt[b];
        }
    }
    consumer_sync();
#pragma unroll
    for (int k = 0; k < kSTRows; k++) {
        if (slot[k] < 0) continue;
        const unsigned int pos = v.off[slot[k]] + rank[k];
#pragma unroll
        for (int j = 0; j < MAXACC; j++)
            if (j < P.nacc) v.tval[j * kStreamT + pos] = val[k][j];
    }
    consumer_sync();
    // small runs: one thread per slot
    for (int b = ct; b < S; b += 32 * kConsumerWarps) {
        const unsigned int c = v.cnt[b];
        if (c == 0) continue;
        if (c >= kBigRun) {
            v.big[atomicAdd(&v.misc[0], 1)] = b;
            continue;
        }
        const unsigned int o = v.off[b];
        unsigned long long acc[MAXACC];
        double comp[MAXACC];
#pragma unroll
        for (int j = 0; j < MAXACC; j++) {
            comp[j] = 0.0;
            acc[j] = j < P.nacc ? v.tval[j * kStreamT + o] : 0ull;
        }
        for (unsigned int e = 1; e < c; e++) {
#pragma unroll
            for (int j = 0; j < MAXACC; j++) {
                if (j >= P.nacc) break;
                acc[j] = combine(P.acc[j].kind, acc[j], v.tval[j * kStreamT + o + e], &comp[j]);
            }
        }
        st_add_run<MAXACC>(P, v, b, c, acc, comp);
        v.cnt[b] = 0;
    }
    consumer_sync();
    // big runs: one warp per slot
    const int lane = ct & 31, w = ct >> 5;
    const int nbig = v.misc[0];
    for (int r = w; r < nbig; r += kConsumerWarps) {
        const int b = (int)v.big[r];
        const unsigned int c = v.cnt[b], o = v.off[b];
        unsigned long long acc[MAXACC];
        double comp[MAXACC];
#pragma unroll
        for (int j = 0; j < MAXACC; j++) {
            comp[j] = 0.0;
            acc[j] = j < P.nacc ? v.tval[j * kStreamT + o + lane] : 0ull;
        }
        for (unsigned int e = lane + 32; e < c; e += 32) {
#pragma unroll
            for (int j = 0; j < MAXACC; j++) {
                if (j >= P.nacc) break;
                acc[j] = combine(P.acc[j].kind, acc[j], v.tval[j * kStreamT + o + e], &comp[j]);
            }
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
#pragma unroll
            for (int j = 0; j < MAXACC; j++) {
                if (j >= P.nacc) break;
                const unsigned long long x = __shfl_xor_sync(0xffffffffu, acc[j], d);
                const double xc = __shfl_xor_sync(0xffffffffu, comp[j], d);
                if (P.acc[j].kind == kAccSumF64) comp[j] += xc;
                acc[j] = combine(P.acc[j].kind, acc[j], x, &comp[j]);
            }
        }
        if (lane == 0) {
            st_add_run<MAXACC>(P, v, b, c, acc, comp);
            v.cnt[b] = 0;
        }
    }
    consumer_sync();
    if (ct == 0) v.misc[0] = 0;
}

template <int MAXACC, bool JOIN>
__global__ void __launch_bounds__(kStreamThreads) agg_stile_kernel(const __grid_constant__ AggProgram P,
                                                                   const __grid_constant__ DevPredicate pred,
                                                                   const __grid_constant__ StreamPlan SP,
                                                                   const __grid_constant__ AggKey gkey,
                                                                   const __grid_constant__ JoinTableDev jt) {
    extern __shared__ __align__(128) unsigned char smem[];
    const STView v = stile_view(P, SP, smem, MAXACC);
    {  // init
        const int S = P.smem_slots;
        for (int i = threadIdx.x; i < S; i += blockDim.x) {
            v.keys[i] = kEmptyKey;
            v.cnt[i] = 0;
        }
        for (int i = threadIdx.x; i < S * P.narrays; i += blockDim.x) v.arr[i] = init_value(P.init[i / S]);
        if (threadIdx.x < 16) v.misc[threadIdx.x] = 0;
        if (threadIdx.x == 0) {
            for (int s = 0; s < kStages; s++) {
                mbar_init(&v.full[s], 1);
                mbar_init(&v.empty[s], kConsumerWarps);
            }
            fence_barrier_init();
        }
        __syncthreads();
    }
    StreamView sv;  // the producer's view of the same ring
    sv.stages = v.stages;
    sv.full = v.full;
    sv.empty = v.empty;
    sv.direct = v.direct;
    sv.abort = v.misc + 10;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        if (lane == 0) stream_produce(P, SP, sv);
        __syncwarp();
    } else {
        const unsigned long long keep = policy_evict_last();
        const int ct = threadIdx.x - 32;
        int it = 0;
        for (long long tile = blockIdx.x; tile < SP.ntiles; tile += gridDim.x, it++) {
            const int st = it % kStages;
            // Every consumer waits, so they all agree on whether to go on.
            const bool ok = mbar_wait(&v.full[st], (it / kStages) & 1) && !*(volatile int*)sv.abort;
            if (consumer_sync_or(!ok)) {
                if (ct == 0) {
                    atomicOr(P.status, kStatusTimeout);
                    *(volatile int*)sv.abort = 1;
                }
                break;
            }
            const bool direct = v.direct[st];
            const unsigned char* stage = v.stages + (size_t)st * SP.stage_bytes;
            int slot[kSTRows];
            unsigned long long val[kSTRows][MAXACC];
            unsigned int start[kSTRows], count[kSTRows];
            long long brow[kSTRows];
#pragma unroll
            for (int k = 0; k < kSTRows; k++) {
                const int r = ct + k * 32 * kConsumerWarps;
                const long long g = tile * kStreamT + r;
                slot[k] = kSlotNone;
                count[k] = 0;
                start[k] = 0;
                brow[k] = 0;
                if (g >= SP.n) continue;
                if (pred.nleaves && !stream_predicate(pred, SP, stage, direct, g, r)) continue;
                bool kv;
                long long key;
                if (JOIN) {
                    if (!stream_valid(SP, SP.key_col, stage, direct, g, r)) continue;
                    const long long pkey = stream_raw(SP, SP.key_col, stage, direct, g, r);
                    unsigned int first = 0;
                    if (pkey == kEmptyKey) {
                        start[k] = jt.special_start;
                        count[k] = jt.special_count;
                        first = count[k] ? jt.first_row[jt.capacity] : 0u;
                    } else {
                        unsigned int s = (unsigned int)(fmix64((unsigned long long)pkey) & (jt.capacity - 1u));
                        for (unsigned int p = 0; p < jt.capacity; p++) {
                            const int4 sl = ld_keep_v4(&jt.slots[s], keep);
                            const unsigned int fr = ld_keep_u32(&jt.first_row[s], keep);
                            const long long sk = ((long long)(unsigned int)sl.y << 32) | (unsigned int)sl.x;
                            if (sk == pkey) {
                                start[k] = (unsigned int)sl.z;
                                count[k] = (unsigned int)sl.w;
                                first = fr;
                                break;
                            }
                            if (sk == kEmptyKey) break;
                            s = (s + 1u) & (jt.capacity - 1u);
                        }
                    }
                    if (count[k] == 0) continue;
                    brow[k] = first;
                    const long long grow = gkey.side ? brow[k] : g;
                    kv = valid_at(gkey.validity, grow);
                    key = 0;
                    if (kv)
                        key = gkey.side ? (gkey.type == kInt64 ? ld_keep_s64((const long long*)gkey.values + grow, keep)
                                                               : (long long)(int)ld_keep_u32((const int*)gkey.values + grow, keep))
                                        : load_int(gkey.values, gkey.type, grow);
                } else {
                    kv = stream_valid(SP, SP.key_col, stage, direct, g, r);
                    key = kv ? stream_raw(SP, SP.key_col, stage, direct, g, r) : 0;
                }
#pragma unroll
                for (int j = 0; j < MAXACC; j++) {
                    if (j >= P.nacc) break;
                    const int c = SP.acc_col[j];
                    val[k][j] = c >= 0 ? contribution_raw(P.acc[j].kind, P.acc[j].in_type,
                                                          stream_valid(SP, c, stage, direct, g, r),
                                                          stream_raw(SP, c, stage, direct, g, r))
                                       : contribution(P.acc[j], g, brow[k]);
                }
                slot[k] = (kv && key != kEmptyKey) ? smem_slot(P, key, v.keys, v.misc + 1) : kSlotGlobal;
                if (slot[k] == kSlotGlobal) {
                    double comp[MAXACC];
#pragma unroll
                    for (int j = 0; j < MAXACC; j++) comp[j] = 0.0;
                    const long long gs = global_slot(P, kv, key);
                    if (gs >= 0) apply_vals<MAXACC>(P, P.arr, P.stride, gs, 1, val[k], comp);
                }
            }
            // A join row's further matches (a key repeated on the build side)
            // read the stage too, so they fold into HBM before it is released.
            if (JOIN) {
#pragma unroll
                for (int k = 0; k < kSTRows; k++) {
                    const int r = ct + k * 32 * kConsumerWarps;
                    const long long g = tile * kStreamT + r;
                    for (unsigned int m = 1; m < count[k]; m++) {
                        const long long b = jt.rows[start[k] + m];
                        const long long grow = gkey.side ? b : g;
                        const bool kv = valid_at(gkey.validity, grow);
                        const long long key = kv ? load_int(gkey.values, gkey.type, grow) : 0;
                        unsigned long long x[MAXACC];
                        double comp[MAXACC];
#pragma unroll
                        for (int j = 0; j < MAXACC; j++) {
                            comp[j] = 0.0;
                            if (j >= P.nacc) break;
                            const int c = SP.acc_col[j];
                            x[j] = c >= 0 ? contribution_raw(P.acc[j].kind, P.acc[j].in_type,
                                                             stream_valid(SP, c, stage, direct, g, r),
                                                             stream_raw(SP, c, stage, direct, g, r))
                                          : contribution(P.acc[j], g, b);
                        }
                        const long long gs = global_slot(P, kv, key);
                        if (gs >= 0) apply_vals<MAXACC>(P, P.arr, P.stride, gs, 1, x, comp);
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&v.empty[st]);  // the stage may be refilled now
            st_round<MAXACC>(P, v, ct, slot, val);
        }
    }
    __syncthreads();
    // flush the CTA table into HBM
    const int S = P.smem_slots;
    for (int i = threadIdx.x; i < S; i += blockDim.x) {
        if (v.arr[i] == 0) continue;
        const long long key = P.direct ? P.direct_lo + i : v.keys[i];
        const long long g = global_slot(P, true, key);
        if (g >= 0) merge_slot(P, v.arr + i, S, P.arr + g, P.stride);
    }
}

// ---- fused probe table: the join + aggregate hot path -----------------------
//
// For `probe JOIN build GROUP BY <build column>` with every aggregate input
// on the probe side, the group a probe row lands in depends only on the join
// slot it matches.  A pre-pass writes, per join slot, {key, CTA slot of that
// key's group, count} into a 16-byte entry, so a probe row needs one L2 load
// to know both whether it matches and where it folds.  The row loop then
// runs at full occupancy (small shared footprint) with plain coalesced loads,
// and folds with per-lane shared atomics: native 64-bit adds, and for Float64
// sums one 128-bit CAS of the (sum, compensation) pair.  Keys repeated on the
// build side, NULL group keys and groups outside the CTA table's range take a
// slow path that is correct for any shape.

struct FusedSlot {
    long long key;
    int cslot;           // the group's CTA slot, -1: none (slow path)
    unsigned int count;  // matches (0: empty slot)
};

constexpr int kFusedThreads = 256;

__global__ void fuse_table_kernel(const __grid_constant__ JoinTableDev jt, const __grid_constant__ AggKey gkey,
                                  long long lo, int S, FusedSlot* __restrict__ out) {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < jt.capacity;
         s += (long long)gridDim.x * blockDim.x) {
        const JoinSlot js = jt.slots[s];
        FusedSlot f;
        f.key = js.key;
        f.count = js.count;
        f.cslot = -1;
        if (js.count == 1) {
            const unsigned int b = jt.first_row[s];
            if (valid_at(gkey.validity, b)) {
                const unsigned long long d = (unsigned long long)(load_int(gkey.values, gkey.type, b) - lo);
                if (d < (unsigned long long)S) f.cslot = (int)d;
            }
        }
        out[s] = f;
    }
}

struct FusedTab {
    const FusedSlot* slots;   // hashed form: one entry per join slot
    const int* dense;         // dense form: one entry per key in [dense_lo, dense_lo + dense_n)
    long long dense_lo;
    unsigned long long dense_n;
};

// The fused kernel's CTA table, one array after another (no bank falls to a
// fixed stride): the rows of each slot as u32 (a CTA folds fewer than 2^32
// rows, which the host checks), then arrays 1.. as S u64 words each.
__host__ __device__ inline size_t fused_counts_bytes(int S) { return ((size_t)S * 4 + 15) & ~(size_t)15; }
size_t fused_smem_bytes(int S, int narrays) { return fused_counts_bytes(S) + (size_t)S * 8 * (narrays - 1); }

// Dense form, for build keys that fill most of their range: entry
// key - dense_lo holds the CTA slot of the key's group (>= 0), -1 when no
// build row has the key, -2 when the key takes the slow path (repeated key,
// NULL group, group outside the CTA table).  A 4-byte load from a table of
// range x 4 bytes replaces the hashed probe.
constexpr int kDenseNone = -1;
constexpr int kDenseSlow = -2;

__global__ void fuse_dense_kernel(const __grid_constant__ JoinTableDev jt, const __grid_constant__ AggKey gkey,
                                  long long lo, int S, int* __restrict__ dense, long long dense_lo) {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < jt.capacity;
         s += (long long)gridDim.x * blockDim.x) {
        const JoinSlot js = jt.slots[s];
        if (js.key == kEmptyKey) continue;
        int e = kDenseSlow;
        if (js.count == 1) {
            const unsigned int b = jt.first_row[s];
            if (valid_at(gkey.validity, b)) {
                const unsigned long long d = (unsigned long long)(load_int(gkey.values, gkey.type, b) - lo);
                if (d < (unsigned long long)S) e = (int)d;
            }
        }
        dense[(unsigned long long)js.key - (unsigned long long)dense_lo] = e;
    }
}

// The join slot of a key placed in the table, -2 when it has none.
__device__ __forceinline__ long long jt_find_slot(const JoinTableDev& t, long long key) {
    unsigned int s = (unsigned int)(fmix64((unsigned long long)key) & (t.capacity - 1u));
    for (unsigned int p = 0; p < t.capacity; p++) {
        const long long k = t.slots[s].key;
        if (k == key) return s;
        if (k == kEmptyKey) return -2;
        s = (s + 1u) & (t.capacity - 1u);
    }
    return -2;
}

// The slow path of one probe row: every match, folded into HBM.
template <int MAXACC>
__device__ void fused_slow_row(const AggProgram& P, const AggKey& gkey, const JoinTableDev& jt, long long s_or_special,
                               long long i, const unsigned long long* val) {
    unsigned int start, count, first;
    if (s_or_special < 0) {
        start = jt.special_start;
        count = jt.special_count;
        first = count ? jt.first_row[jt.capacity] : 0u;
    } else {
        start = jt.slots[s_or_special].start;
        count = jt.slots[s_or_special].count;
        first = jt.first_row[s_or_special];
    }
    double comp[MAXACC];
#pragma unroll
    for (int j = 0; j < MAXACC; j++) comp[j] = 0.0;
    for (unsigned int m = 0; m < count; m++) {
        const long long b = m == 0 ? first : jt.rows[start + m];
        const bool kv = valid_at(gkey.validity, b);
        const long long key = kv ? load_int(gkey.values, gkey.type, b) : 0;
        const long long g = global_slot(P, kv, key);
        if (g >= 0) apply_vals<MAXACC>(P, P.arr, P.stride, g, 1, val, comp);
    }
    (void)i;
}

// ---- Float64 sums as fixed-point integers in a CTA table ------------------
// A 32-bit shared atomic add is a single instruction that settles lanes of a
// warp on one address in hardware; a 64-bit or Float64 one is a retried
// compare-and-swap, several times slower and far slower when lanes of a warp
// meet on a hot group.  So a fused join kernel folds a Float64 SUM as an
// exact integer: x = X * 2^lo with X an integer, |X| < 2^63, added into a
// 128-bit two's-complement accumulator of four 32-bit words (limb k of slot
// i at limbs[k * S + i]) by 32-bit atomics with their carries.  Integer
// addition is exact and order-free, so the CTA's partial is the exact sum of
// the values it folded.  A value that is no such integer (outside the
// window, or with bits below 2^lo, NaN, infinity) folds into the HBM
// accumulator with the compensated Float64 add instead.

// X for x when x is an integer multiple of 2^lo with |X| < 2^63, read off
// x's bits with integer operations alone (no conversion instructions): x is
// m * 2^(e - 1075) with m its 53-bit significand, so X = m * 2^(e - 1075 - lo)
// when that shift keeps X under 2^63 and drops no set bit of m.  Zero folds
// as X = 0; subnormals, infinities and NaN are left to the Float64 path.
__device__ __forceinline__ bool fixed_of(double x, int lo, long long* X) {
    const long long bits = __double_as_longlong(x);
    if (((unsigned long long)bits << 1) == 0ull) {  // +0 or -0
        *X = 0;
        return true;
    }
    // lo is in [-900, 800] (the host places no window outside it), so a
    // subnormal (e = 0) and an infinity or NaN (e = 2047) land outside
    // sh in [-52, 10] and take the Float64 path with the values that do not fit.
    const int e = (int)((unsigned)((unsigned long long)bits >> 52) & 0x7ffu);
    const int sh = e - 1075 - lo;
    if (sh < -52 || sh > 10) return false;
    const unsigned long long m = ((unsigned long long)bits & ((1ull << 52) - 1ull)) | (1ull << 52);
    unsigned long long mag;
    if (sh >= 0) {
        mag = m << sh;  // below 2^63
    } else {
        if (m << (64 + sh)) return false;  // a set bit below 2^lo
        mag = m >> -sh;
    }
    *X = bits < 0 ? -(long long)mag : (long long)mag;
    return true;
}

// Adds X (sign-extended to 128 bits) into the four limbs: each limb's add,
// then the carry it produced into the next; what carries out of the top limb
// is dropped (arithmetic modulo 2^128).
__device__ __forceinline__ void shared_add_i128(unsigned* limbs, int S, int slot, long long X) {
    const unsigned long long u = (unsigned long long)X;
    const unsigned long long ext = X < 0 ? 0xffffffffull : 0ull;
    unsigned long long carry = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        // at most 2^32: a limb's word plus the carry from below
        const unsigned long long add = (k == 0 ? (u & 0xffffffffull) : k == 1 ? (u >> 32) : ext) + carry;
        carry = add >> 32;
        const unsigned a = (unsigned)add;
        if (a) {
            const unsigned old = atomicAdd(limbs + k * S + slot, a);
            carry += old + a < old ? 1u : 0u;
        }
    }
}

// The exact 128-bit value of a slot's limbs, as up to three doubles whose sum
// is value * 2^lo, each exact (52-bit chunks of the magnitude, scaled by
// powers of two the host keeps in range); returns how many.
__device__ __forceinline__ int fixed_chunks(const unsigned* limbs, int S, int slot, int lo, double* out) {
    unsigned long long l = ((unsigned long long)limbs[S + slot] << 32) | limbs[slot];
    unsigned long long h = ((unsigned long long)limbs[3 * S + slot] << 32) | limbs[2 * S + slot];
    const bool neg = (long long)h < 0;
    if (neg) {  // magnitude: two's complement negation of (h, l)
        l = ~l + 1ull;
        h = ~h + (l == 0 ? 1ull : 0ull);
    }
    const unsigned long long m52 = (1ull << 52) - 1ull;
    const unsigned long long c0 = l & m52;
    const unsigned long long c1 = ((l >> 52) | (h << 12)) & m52;
    const unsigned long long c2 = h >> 40;
    int n = 0;
    const double sg = neg ? -1.0 : 1.0;
    if (c2) out[n++] = sg * scalbn((double)c2, lo + 104);
    if (c1) out[n++] = sg * scalbn((double)c1, lo + 52);
    if (c0) out[n++] = sg * scalbn((double)c0, lo);
    return n;
}

// A Float64 value outside its sum's fixed-point window: straight into the
// group's HBM accumulator, with its rounding error into the compensation.
__device__ __noinline__ void fused_f64_to_hbm(const AggProgram& P, const DevAcc& a, int cslot, double x) {
    const long long g = global_slot(P, true, P.direct_lo + cslot);
    if (g < 0) return;
    double* d = (double*)(P.arr + a.arr * P.stride + g);
    add_f64_comp(d, d + P.stride, x);
}

// Adds a fused kernel's CTA table into the HBM table: each occupied slot's
// rows and arrays, Float64 sums with their compensation.
// `keys` (shared memory) names each slot's key; null: slot i holds key
// direct_lo + i.
// `narrow`: bit a set when array a holds a 32-bit MIN/MAX in its low word.
// A Float64 sum in fixed point (DevAcc::fix) holds its four limbs in arrays
// arr and arr + 1; it reaches HBM as its exact chunks, each added with its
// rounding error into the compensation.
__device__ void fused_flush(const AggProgram& P, const unsigned int* rows, const unsigned long long* tab, int S,
                            const long long* keys = nullptr, unsigned narrow = 0) {
    unsigned long long fixed = 0;  // bit a: arrays a, a + 1 hold limbs
    for (int j = 0; j < P.nacc; j++)
        if (P.acc[j].fix) fixed |= 1ull << P.acc[j].arr;
    for (int i = threadIdx.x; i < S; i += blockDim.x) {
        if (rows[i] == 0) continue;
        const long long g = global_slot(P, true, keys ? keys[i] : P.direct_lo + i);
        if (g < 0) continue;
        atomicAdd(&P.arr[g], (unsigned long long)rows[i]);
        for (int a = 1; a < P.narrays; a++) {
            if ((fixed >> a) & 1ull) {
                int lo = 0;
                for (int j = 0; j < P.nacc; j++)
                    if (P.acc[j].arr == a) lo = P.acc[j].fix_lo;
                double part[3];
                const int np = fixed_chunks((const unsigned*)(tab + a * S), S, i, lo, part);
                double* d = (double*)(P.arr + a * P.stride + g);
                for (int q = 0; q < np; q++) add_f64_comp(d, d + P.stride, part[q]);
                a++;  // array a + 1 held the upper limbs
                continue;
            }
            unsigned long long x = tab[a * S + i];
            if ((narrow >> a) & 1u) x = (unsigned long long)(long long)(int)(unsigned)x;
            unsigned long long* d = P.arr + a * P.stride + g;
            switch (P.merge[a]) {
                case kMergeAddU64:
                    if (x) atomicAdd(d, x);
                    break;
                case kMergeAddF64Comp:
                    add_f64_comp((double*)d, (double*)(d + P.stride), as_f64(x));
                    break;
                case kMergeAddF64:
                    if (as_f64(x) != 0.0) atomicAdd((double*)d, as_f64(x));
                    break;
                case kMergeMin:
                    if ((long long)x != 0x7fffffffffffffffll) atomicMin((long long*)d, (long long)x);
                    break;
                default:
                    if ((long long)x != (long long)0x8000000000000000ull) atomicMax((long long*)d, (long long)x);
                    break;
            }
        }
    }
}

// The slow path of one probe row, out of line: its contributions, then
// every match folded into HBM.
__device__ __noinline__ void fused_slow(const AggProgram& P, const AggKey& gkey, const JoinTableDev& jt,
                                        long long s_or_special, long long i) {
    unsigned long long val[4];
#pragma unroll
    for (int j = 0; j < 4; j++)
        if (j < P.nacc) val[j] = contribution(P.acc[j], i, 0);
    fused_slow_row<4>(P, gkey, jt, s_or_special, i, val);
}

// A 64-bit wrapping add into shared memory as 32-bit atomics (the 64-bit
// shared add is not a single instruction): the low word's add, then its
// carry with the high word.
__device__ __forceinline__ void shared_add_u64(unsigned long long* p, unsigned long long v) {
    unsigned* w = (unsigned*)p;  // little-endian: w[0] the low word
    const unsigned lo = (unsigned)v, hi = (unsigned)(v >> 32);
    const unsigned old = lo ? atomicAdd(w, lo) : 0u;
    const unsigned up = hi + (old + lo < old ? 1u : 0u);
    if (up) atomicAdd(w + 1, up);
}


template <int MAXACC, int RPT, bool DENSE>
__global__ void __launch_bounds__(kFusedThreads, 8) agg_fused_join_kernel(
    const __grid_constant__ AggProgram P, const __grid_constant__ DevPredicate pred, const __grid_constant__ AggKey gkey,
    const void* __restrict__ pk, const uint8_t* __restrict__ pkv, int pk_type, const __grid_constant__ JoinTableDev jt,
    const __grid_constant__ FusedTab ft, long long n) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int S = P.smem_slots;
    unsigned int* rows = (unsigned int*)smem;
    unsigned long long* tab = (unsigned long long*)(smem + fused_counts_bytes(S)) - S;  // array a at tab + a * S
    for (int i = threadIdx.x; i < S; i += blockDim.x) rows[i] = 0;
    for (int i = threadIdx.x; i < S * (P.narrays - 1); i += blockDim.x) tab[S + i] = init_value(P.init[1 + i / S]);
    __syncthreads();
    const unsigned long long keep = policy_evict_last();
    const unsigned int cap_mask = jt.capacity - 1u;
    const long long step = (long long)gridDim.x * blockDim.x * RPT;
    for (long long base = blockIdx.x * (long long)blockDim.x * RPT; base < n; base += step) {
        long long sidx[RPT];  // matched join slot, -1 special key, -2 no match
        int cslot[RPT];
#pragma unroll
        for (int r = 0; r < RPT; r++) {
            const long long i = base + r * (long long)blockDim.x + threadIdx.x;
            sidx[r] = -2;
            cslot[r] = -1;
            if (i >= n) continue;
            if (pred.nleaves && !predicate_holds(pred, i)) continue;
            if (!valid_at(pkv, i)) continue;
            const long long key = pk_type == kInt64 ? __ldcs((const long long*)pk + i) : (long long)__ldcs((const int*)pk + i);
            if (key == kEmptyKey) {
                if (jt.special_count) sidx[r] = -1;
                continue;
            }
            if (DENSE) {
                const unsigned long long d = (unsigned long long)key - (unsigned long long)ft.dense_lo;
                if (d >= ft.dense_n) continue;
                const int e = (int)ld_keep_u32(ft.dense + d, keep);
                if (e >= 0) {
                    sidx[r] = 0;
                    cslot[r] = e;
                } else if (e == kDenseSlow) {
                    sidx[r] = jt_find_slot(jt, key);
                }
                continue;
            }
            unsigned int s = (unsigned int)(fmix64((unsigned long long)key) & cap_mask);
            for (unsigned int p = 0; p <= cap_mask; p++) {
                const int4 e = ld_keep_v4(&ft.slots[s], keep);
                const long long k = ((long long)(unsigned int)e.y << 32) | (unsigned int)e.x;
                if (k == key) {
                    sidx[r] = s;
                    cslot[r] = (unsigned int)e.w == 1u ? e.z : -1;
                    break;
                }
                if (k == kEmptyKey) break;
                s = (s + 1u) & cap_mask;
            }
        }
#pragma unroll
        for (int r = 0; r < RPT; r++) {
            const long long i = base + r * (long long)blockDim.x + threadIdx.x;
            unsigned long long val[MAXACC];
#pragma unroll
            for (int j = 0; j < MAXACC; j++) {
                val[j] = 0;
                if (j >= P.nacc || sidx[r] == -2) continue;
                const DevAcc& a = P.acc[j];
                const bool v = valid_at(a.validity, i);
                long long raw = 0;
                if (v) raw = a.in_type == kInt32 ? (long long)__ldcs((const int*)a.values + i)
                                                 : __ldcs((const long long*)a.values + i);
                val[j] = contribution_raw(a.kind, a.in_type, v, raw);
            }
            if (sidx[r] == -2) continue;
            if (cslot[r] < 0) {
                fused_slow_row<MAXACC>(P, gkey, jt, sidx[r], i, val);
                continue;
            }
            const int cs = cslot[r];
            atomicAdd(&rows[cs], 1u);
#pragma unroll
            for (int j = 0; j < MAXACC; j++) {
                if (j >= P.nacc) break;
                const DevAcc& a = P.acc[j];
                unsigned long long* p = tab + a.arr * S + cs;
                switch (a.kind) {
                    case kAccCount:
                    case kAccSumInt:
                        if (val[j]) shared_add_u64(p, val[j]);
                        break;
                    case kAccSumF64: {
                        const double x = as_f64(val[j]);
                        if (a.fix) {
                            long long X;
                            if (fixed_of(x, a.fix_lo, &X)) {
                                if (X) shared_add_i128((unsigned*)(tab + a.arr * S), S, cs, X);
                            } else {
                                fused_f64_to_hbm(P, a, cs, x);
                            }
                            break;
                        }
                        // The atomic rounds old + x once; TwoSum recovers that
                        // rounding error exactly, and it joins the compensation.
                        const double old = atomicAdd((double*)p, x);
                        double c = 0.0;
                        two_sum_into(old, x, &c);
                        if (c != 0.0) atomicAdd((double*)(p + S), c);
                        break;
                    }
                    case kAccMin:
                        if (val[j] != 0x7fffffffffffffffull) atomicMin((long long*)p, (long long)val[j]);
                        break;
                    default:
                        if (val[j] != 0x8000000000000000ull) atomicMax((long long*)p, (long long)val[j]);
                        break;
                }
            }
        }
    }
    __syncthreads();
    fused_flush(P, rows, tab, S);
}

// The fused join-aggregate, interpreted a vector of rows at a time: each
// thread takes RPT rows; the predicate's leaves, the key, the lookups and
// then each accumulator are handled for all RPT rows together, so a type or
// kind is dispatched once per RPT rows and each column's loads go out
// together.  The CTA table and its flush are agg_fused_join_kernel's.
template <int RPT, bool DENSE>
__global__ void __launch_bounds__(kFusedThreads) agg_fusedv_join_kernel(
    const __grid_constant__ AggProgram P, const __grid_constant__ DevPredicate pred, const __grid_constant__ AggKey gkey,
    const void* __restrict__ pk, const uint8_t* __restrict__ pkv, int pk_type, const __grid_constant__ JoinTableDev jt,
    const __grid_constant__ FusedTab ft, long long n) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int S = P.smem_slots;
    unsigned int* rows = (unsigned int*)smem;
    unsigned long long* tab = (unsigned long long*)(smem + fused_counts_bytes(S)) - S;  // array a at tab + a * S
    for (int i = threadIdx.x; i < S; i += blockDim.x) rows[i] = 0;
    for (int i = threadIdx.x; i < S * (P.narrays - 1); i += blockDim.x) tab[S + i] = init_value(P.init[1 + i / S]);
    __syncthreads();
    const unsigned long long keep = policy_evict_last();
    const long long stride = blockDim.x;
    const long long step = (long long)gridDim.x * blockDim.x * RPT;
    for (long long tile = blockIdx.x * (long long)blockDim.x * RPT; tile < n; tile += step) {
        const long long base = tile + threadIdx.x;  // row r: base + r * stride
        unsigned live = 0;
#pragma unroll
        for (int r = 0; r < RPT; r++)
            if (base + r * stride < n) live |= 1u << r;
        live = predicate_mask<RPT>(pred, base, stride, live);
        if (pkv) {
#pragma unroll
            for (int r = 0; r < RPT; r++)
                if (((live >> r) & 1u) && !valid_at(pkv, base + r * stride)) live &= ~(1u << r);
        }
        long long key[RPT];
        if (pk_type == kInt64) {
#pragma unroll
            for (int r = 0; r < RPT; r++) key[r] = (live >> r) & 1u ? __ldcs((const long long*)pk + base + r * stride) : 0;
        } else {
#pragma unroll
            for (int r = 0; r < RPT; r++)
                key[r] = (live >> r) & 1u ? (long long)__ldcs((const int*)pk + base + r * stride) : 0;
        }
        // Lookups: cs[r] is the CTA slot of a fast row; slow rows fold now.
        int cs[RPT];
        unsigned fast = 0;
        if (DENSE) {
#pragma unroll
            for (int r = 0; r < RPT; r++) {
                cs[r] = kDenseNone;
                const unsigned long long d = (unsigned long long)key[r] - (unsigned long long)ft.dense_lo;
                if (((live >> r) & 1u) && d < ft.dense_n) cs[r] = (int)ld_keep_u32(ft.dense + d, keep);
            }
#pragma unroll
            for (int r = 0; r < RPT; r++) {
                if (!((live >> r) & 1u)) continue;
                if (cs[r] >= 0) {
                    fast |= 1u << r;
                } else if (key[r] == kEmptyKey) {
                    if (jt.special_count) fused_slow(P, gkey, jt, -1, base + r * stride);
                } else if (cs[r] == kDenseSlow) {
                    fused_slow(P, gkey, jt, jt_find_slot(jt, key[r]), base + r * stride);
                }
            }
        } else {
            const unsigned int cap_mask = jt.capacity - 1u;
#pragma unroll
            for (int r = 0; r < RPT; r++) {
                cs[r] = -1;
                if (!((live >> r) & 1u)) continue;
                if (key[r] == kEmptyKey) {
                    if (jt.special_count) fused_slow(P, gkey, jt, -1, base + r * stride);
                    continue;
                }
                unsigned int sl = (unsigned int)(fmix64((unsigned long long)key[r]) & cap_mask);
                for (unsigned int q = 0; q <= cap_mask; q++) {
                    const int4 e = ld_keep_v4(&ft.slots[sl], keep);
                    const long long k = ((long long)(unsigned int)e.y << 32) | (unsigned int)e.x;
                    if (k == key[r]) {
                        if ((unsigned int)e.w == 1u && e.z >= 0) {
                            cs[r] = e.z;
                            fast |= 1u << r;
                        } else {
                            fused_slow(P, gkey, jt, sl, base + r * stride);
                        }
                        break;
                    }
                    if (k == kEmptyKey) break;
                    sl = (sl + 1u) & cap_mask;
                }
            }
        }
        if (!fast) continue;
#pragma unroll
        for (int r = 0; r < RPT; r++)
            if ((fast >> r) & 1u) atomicAdd(&rows[cs[r]], 1u);
        for (int j = 0; j < P.nacc; j++) {
            const DevAcc& a = P.acc[j];
            unsigned long long* col = tab + a.arr * S;
            unsigned vm = fast;
            if (a.validity) {
#pragma unroll
                for (int r = 0; r < RPT; r++)
                    if (((vm >> r) & 1u) && !valid_at(a.validity, base + r * stride)) vm &= ~(1u << r);
            }
            if (a.kind == kAccCount) {
#pragma unroll
                for (int r = 0; r < RPT; r++)
                    if ((vm >> r) & 1u) shared_add_u64(&col[cs[r]], 1ull);
                continue;
            }
            long long raw[RPT];
            if (a.in_type == kInt32) {
#pragma unroll
                for (int r = 0; r < RPT; r++)
                    raw[r] = (vm >> r) & 1u ? (long long)__ldcs((const int*)a.values + base + r * stride) : 0;
            } else {
#pragma unroll
                for (int r = 0; r < RPT; r++)
                    raw[r] = (vm >> r) & 1u ? __ldcs((const long long*)a.values + base + r * stride) : 0;
            }
            switch (a.kind) {
                case kAccSumInt:
#pragma unroll
                    for (int r = 0; r < RPT; r++)
                        if (((vm >> r) & 1u) && raw[r]) shared_add_u64(&col[cs[r]], (unsigned long long)raw[r]);
                    break;
                case kAccSumF64:
#pragma unroll
                    for (int r = 0; r < RPT; r++) {
                        if (!((vm >> r) & 1u)) continue;
                        // The atomic rounds old + x once; TwoSum recovers that
                        // rounding error exactly, and it joins the compensation.
                        const double x = a.in_type == kFloat64 ? __longlong_as_double(raw[r]) : (double)raw[r];
                        if (a.fix) {
                            long long X;
                            if (fixed_of(x, a.fix_lo, &X)) {
                                if (X) shared_add_i128((unsigned*)col, S, cs[r], X);
                            } else {
                                fused_f64_to_hbm(P, a, cs[r], x);
                            }
                            continue;
                        }
                        const double old = atomicAdd((double*)&col[cs[r]], x);
                        double c = 0.0;
                        two_sum_into(old, x, &c);
                        if (c != 0.0) atomicAdd((double*)&col[S + cs[r]], c);
                    }
                    break;
                case kAccMin:
#pragma unroll
                    for (int r = 0; r < RPT; r++) {
                        if (!((vm >> r) & 1u)) continue;
                        const long long v = a.in_type == kFloat64 ? total_order_key(__longlong_as_double(raw[r])) : raw[r];
                        atomicMin((long long*)&col[cs[r]], v);
                    }
                    break;
                default:
#pragma unroll
                    for (int r = 0; r < RPT; r++) {
                        if (!((vm >> r) & 1u)) continue;
                        const long long v = a.in_type == kFloat64 ? total_order_key(__longlong_as_double(raw[r])) : raw[r];
                        atomicMax((long long*)&col[cs[r]], v);
                    }
                    break;
            }
        }
    }
    __syncthreads();
    fused_flush(P, rows, tab, S);
}

// ---- the fused probe table over streamed columns -------------------------
//
// agg_fused_join_kernel's fold (the per-join-slot probe table, a CTA table of
// u32 row counts and fixed-point Float64 sums) fed by the streamed kernels'
// producer: one warp copies each 1024-row tile of the probe columns into a
// ring of shared-memory stages with bulk copies, so the consumer warps read
// every column from shared memory and wait on HBM only through the ring,
// not once per row and column.  Their only global loads are the probe-table
// lookups, all of a thread's rows issued together.

struct FStreamView {
    StreamView sv;          // stages, barriers and abort flag (stream_produce's view)
    unsigned int* rows;     // S
    unsigned long long* tab;  // array a at tab + a * S (a >= 1)
};

size_t fstream_smem_bytes(int S, int stage_bytes, int narrays) {
    return (size_t)kStages * stage_bytes + 16 * kStages + 16 * kStages + 16 + 128 + fused_smem_bytes(S, narrays);
}

__device__ __forceinline__ FStreamView fstream_view(const AggProgram& P, const StreamPlan& SP, unsigned char* smem) {
    FStreamView v;
    v.sv.stages = smem;
    unsigned char* p = smem + (size_t)kStages * SP.stage_bytes;
    v.sv.full = (unsigned long long*)p;
    v.sv.empty = v.sv.full + kStages;
    v.sv.direct = (int*)(v.sv.empty + kStages);
    v.sv.abort = v.sv.direct + 4 * kStages;
    v.sv.fill = v.sv.abort + 1;
    v.sv.keys = nullptr;
    p = (unsigned char*)(((uintptr_t)(v.sv.abort + 2) + 127) & ~(uintptr_t)127);
    v.rows = (unsigned int*)p;
    v.tab = (unsigned long long*)(p + fused_counts_bytes(P.smem_slots)) - P.smem_slots;
    v.sv.tab = v.tab;
    return v;
}

// One fast row's fold into CTA slot cs: its row count, then each
// accumulator from the stage (or, for a direct tile, global row g).
template <int MAXACC>
__device__ __forceinline__ void fstream_fold(const AggProgram& P, const StreamPlan& SP, const FStreamView& v,
                                             const unsigned char* stage, bool direct, long long g, int r, int cs) {
    const int S = P.smem_slots;
    atomicAdd(&v.rows[cs], 1u);
#pragma unroll
    for (int j = 0; j < MAXACC; j++) {
        if (j >= P.nacc) break;
        const DevAcc& a = P.acc[j];
        const int c = SP.acc_col[j];
        const bool valid = stream_valid(SP, c, stage, direct, g, r);
        const long long raw = valid ? stream_raw(SP, c, stage, direct, g, r) : 0;
        const unsigned long long val = contribution_raw(a.kind, a.in_type, valid, raw);
        unsigned long long* p = v.tab + a.arr * S + cs;
        switch (a.kind) {
            case kAccCount:
            case kAccSumInt:
                if (val) shared_add_u64(p, val);
                break;
            case kAccSumF64: {
                const double x = as_f64(val);
                if (a.fix) {
                    long long X;
                    if (fixed_of(x, a.fix_lo, &X)) {
                        if (X) shared_add_i128((unsigned*)(v.tab + a.arr * S), S, cs, X);
                    } else {
                        fused_f64_to_hbm(P, a, cs, x);
                    }
                    break;
                }
                const double old = atomicAdd((double*)p, x);
                double comp = 0.0;
                two_sum_into(old, x, &comp);
                if (comp != 0.0) atomicAdd((double*)(p + S), comp);
                break;
            }
            case kAccMin:
                if (val != 0x7fffffffffffffffull) atomicMin((long long*)p, (long long)val);
                break;
            default:
                if (val != 0x8000000000000000ull) atomicMax((long long*)p, (long long)val);
                break;
        }
    }
}

template <int MAXACC, bool DENSE>
__global__ void __launch_bounds__(kStreamThreads) agg_fstream_join_kernel(
    const __grid_constant__ AggProgram P, const __grid_constant__ DevPredicate pred, const __grid_constant__ StreamPlan SP,
    const __grid_constant__ AggKey gkey, const __grid_constant__ JoinTableDev jt, const __grid_constant__ FusedTab ft) {
    extern __shared__ __align__(128) unsigned char smem[];
    const FStreamView v = fstream_view(P, SP, smem);
    const int S = P.smem_slots;
    for (int i = threadIdx.x; i < S; i += blockDim.x) v.rows[i] = 0;
    for (int i = threadIdx.x; i < S * (P.narrays - 1); i += blockDim.x) v.tab[S + i] = init_value(P.init[1 + i / S]);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) {
            mbar_init(&v.sv.full[s], 1);
            mbar_init(&v.sv.empty[s], kConsumerWarps);
        }
        *v.sv.abort = 0;
        fence_barrier_init();
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        if (lane == 0) stream_produce(P, SP, v.sv);
        __syncwarp();
    } else {
        const unsigned long long keep = policy_evict_last();
        const int ct = threadIdx.x - 32;
        constexpr int kRows = kStreamT / (32 * kConsumerWarps);
        const unsigned int cap_mask = jt.capacity - 1u;
        int it = 0;
        for (long long tile = blockIdx.x; tile < SP.ntiles; tile += gridDim.x, it++) {
            const int st = it % kStages;
            if (!mbar_wait(&v.sv.full[st], (it / kStages) & 1) || *(volatile int*)v.sv.abort) {
                atomicOr(P.status, kStatusTimeout);
                *(volatile int*)v.sv.abort = 1;
                break;
            }
            const bool direct = v.sv.direct[st];
            const unsigned char* stage = v.sv.stages + (size_t)st * SP.stage_bytes;
            // Every row's WHERE and key from the stage, then all its lookups
            // at once: kRows independent L2 loads a thread.
            long long key[kRows];
            unsigned live = 0;
#pragma unroll
            for (int k = 0; k < kRows; k++) {
                const int r = ct + k * 32 * kConsumerWarps;
                const long long g = tile * kStreamT + r;
                key[k] = 0;
                if (g >= SP.n) continue;
                if (pred.nleaves && !stream_predicate(pred, SP, stage, direct, g, r)) continue;
                if (!stream_valid(SP, SP.key_col, stage, direct, g, r)) continue;
                key[k] = stream_raw(SP, SP.key_col, stage, direct, g, r);
                live |= 1u << k;
            }
            int cs[kRows];  // the CTA slot; kDenseSlow / kDenseNone as in the dense table
            long long js[kRows];  // the join slot of a slow row (-1: the kEmptyKey run)
#pragma unroll
            for (int k = 0; k < kRows; k++) {
                cs[k] = kDenseNone;
                js[k] = -2;
                if (!((live >> k) & 1u)) continue;
                if (key[k] == kEmptyKey) {
                    if (jt.special_count) {
                        cs[k] = kDenseSlow;
                        js[k] = -1;
                    }
                    continue;
                }
                if (DENSE) {
                    const unsigned long long d = (unsigned long long)key[k] - (unsigned long long)ft.dense_lo;
                    if (d < ft.dense_n) cs[k] = (int)ld_keep_u32(ft.dense + d, keep);
                } else {
                    unsigned int sl = (unsigned int)(fmix64((unsigned long long)key[k]) & cap_mask);
                    for (unsigned int q = 0; q <= cap_mask; q++) {
                        const int4 e = ld_keep_v4(&ft.slots[sl], keep);
                        const long long kk = ((long long)(unsigned int)e.y << 32) | (unsigned int)e.x;
                        if (kk == key[k]) {
                            if ((unsigned int)e.w == 1u && e.z >= 0) {
                                cs[k] = e.z;
                            } else {
                                cs[k] = kDenseSlow;
                                js[k] = sl;
                            }
                            break;
                        }
                        if (kk == kEmptyKey) break;
                        sl = (sl + 1u) & cap_mask;
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < kRows; k++) {
                const int r = ct + k * 32 * kConsumerWarps;
                const long long g = tile * kStreamT + r;
                if (cs[k] >= 0) {
                    fstream_fold<MAXACC>(P, SP, v, stage, direct, g, r, cs[k]);
                } else if (cs[k] == kDenseSlow) {
                    fused_slow(P, gkey, jt, js[k] == -2 ? jt_find_slot(jt, key[k]) : js[k], g);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&v.sv.empty[st]);
        }
    }
    __syncthreads();
    fused_flush(P, v.rows, v.tab, S);
}

// ---- the fused probe table, compiled per accumulator shape ----------------
//
// agg_fused_join_kernel interprets the accumulator program per row (a loop
// over accumulators, a switch on kind and type each): about 340 instructions
// a row, which bounds it by instruction issue, not by HBM.  This form fixes
// the accumulators at compile time (up to two probe-side sums, COUNT(*)
// being the row count) and takes rows whose WHERE, key and inputs carry no
// validity bitmaps: each row is its loads, a compare per leaf, one probe-
// table lookup and its shared adds.  RPT rows a thread issue their loads
// together.  Anything else keeps the interpreted kernels.

enum : int { kLeanNone = 0, kLeanSumI32 = 1, kLeanSumI64 = 2, kLeanSumF64 = 3 };

struct LeanPlan {
    int nleaves;  // 0..2, over probe columns without validity
    int leaf_width[2];
    int leaf_f64[2];
    int leaf_mask[2];  // the comparison as the outcomes it keeps: bit 0 a < lit, 1 a == lit, 2 a > lit
    const void* acc_values[2];
    int acc_arr[2];  // CTA/HBM array of each sum
    int acc_j[2];    // its accumulator in the program
    int acc_off[2];  // acc_arr * S: the sum's CTA array, in 64-bit words from the table's base
    int fix[2];      // the program's DevAcc::fix and fix_lo of each sum
    int fix_lo[2];
    int acc_leaf[2];  // the WHERE leaf that reads the same column as the sum (its values reused), or -1
};

// A comparison without branches: which of a < b, a == b, a > b holds picks
// a bit of the leaf's mask.
__device__ __forceinline__ bool lean_cmp(int mask, long long a, long long b) {
    const int idx = (a >= b ? 1 : 0) + (a > b ? 1 : 0);
    return (mask >> idx) & 1;
}

template <int KIND>
__device__ __forceinline__ long long lean_load(const void* values, long long i) {
    if (KIND == kLeanSumI32) return (long long)__ldcs((const int*)values + i);
    return __ldcs((const long long*)values + i);
}

template <int KIND>
__device__ __forceinline__ void lean_fold(const AggProgram& P, const LeanPlan& L, int q, unsigned long long* tab, int S,
                                          int cs, long long raw) {
    if (KIND == kLeanNone) return;
    unsigned long long* col = tab + L.acc_off[q];
    if (KIND == kLeanSumF64) {
        const double x = __longlong_as_double(raw);
        long long X;
        if (L.fix[q] && fixed_of(x, L.fix_lo[q], &X)) {
            if (X) shared_add_i128((unsigned*)col, S, cs, X);
        } else if (L.fix[q]) {
            fused_f64_to_hbm(P, P.acc[L.acc_j[q]], cs, x);
        } else {
            const double old = atomicAdd((double*)&col[cs], x);
            double c = 0.0;
            two_sum_into(old, x, &c);
            if (c != 0.0) atomicAdd((double*)&col[S + cs], c);
        }
    } else if (raw) {
        shared_add_u64(&col[cs], (unsigned long long)raw);
    }
}

// One request's columns as the lean kernels read them: the probe key, up to
// two WHERE columns with their literals (the comparisons are the plan's),
// and up to two sum inputs.
struct LeanCols {
    const void* pk;
    const void* leaf[2];
    long long lit[2];
    const void* acc[2];
};

// Rows base + r * kFusedThreads (r < RPT, below n) of one request, folded
// into the CTA table: every load first, then the lookups, then the folds.
template <int A0, int A1, bool DENSE, int RPT>
__device__ __forceinline__ void lean_rows(const AggProgram& P, const DevPredicate& pred, const LeanPlan& L,
                                          const LeanCols& C, const AggKey& gkey, int pk_type, const JoinTableDev& jt,
                                          const FusedTab& ft, long long base, long long n, unsigned int* rows,
                                          unsigned long long* tab, int S, unsigned long long keep) {
    const unsigned int cap_mask = jt.capacity - 1u;
    long long key[RPT], v0[RPT], v1[RPT], lv0[RPT], lv1[RPT];
#pragma unroll
    for (int r = 0; r < RPT; r++) {
        const long long i = base + r * (long long)kFusedThreads;
        const bool in = i < n;
        key[r] = !in ? 0 : pk_type == kInt64 ? __ldcs((const long long*)C.pk + i) : (long long)__ldcs((const int*)C.pk + i);
        lv0[r] = lv1[r] = v0[r] = v1[r] = 0;
        if (!in) continue;
        if (L.nleaves > 0)
            lv0[r] = L.leaf_width[0] == 8 ? __ldcs((const long long*)C.leaf[0] + i) : (long long)__ldcs((const int*)C.leaf[0] + i);
        if (L.nleaves > 1)
            lv1[r] = L.leaf_width[1] == 8 ? __ldcs((const long long*)C.leaf[1] + i) : (long long)__ldcs((const int*)C.leaf[1] + i);
        if (A0 != kLeanNone) v0[r] = lean_load<A0>(C.acc[0], i);
        if (A1 != kLeanNone) v1[r] = lean_load<A1>(C.acc[1], i);
    }
    int cs[RPT];
#pragma unroll
    for (int r = 0; r < RPT; r++) {
        cs[r] = kDenseNone;
        const long long i = base + r * (long long)kFusedThreads;
        if (i >= n) continue;
        if (L.nleaves > 0) {
            const long long a = L.leaf_f64[0] ? filter_order_key(__longlong_as_double(lv0[r])) : lv0[r];
            if (!lean_cmp(L.leaf_mask[0], a, C.lit[0])) continue;
        }
        if (L.nleaves > 1) {
            const long long a = L.leaf_f64[1] ? filter_order_key(__longlong_as_double(lv1[r])) : lv1[r];
            if (!lean_cmp(L.leaf_mask[1], a, C.lit[1])) continue;
        }
        if (key[r] == kEmptyKey) {
            if (jt.special_count) cs[r] = kDenseSlow;
            continue;
        }
        if (DENSE) {
            const unsigned long long d = (unsigned long long)key[r] - (unsigned long long)ft.dense_lo;
            if (d < ft.dense_n) cs[r] = (int)ld_keep_u32(ft.dense + d, keep);
        } else {
            unsigned int sl = (unsigned int)(fmix64((unsigned long long)key[r]) & cap_mask);
            for (unsigned int q = 0; q <= cap_mask; q++) {
                const int4 e = ld_keep_v4(&ft.slots[sl], keep);
                const long long kk = ((long long)(unsigned int)e.y << 32) | (unsigned int)e.x;
                if (kk == key[r]) {
                    cs[r] = ((unsigned int)e.w == 1u && e.z >= 0) ? e.z : kDenseSlow;
                    break;
                }
                if (kk == kEmptyKey) break;
                sl = (sl + 1u) & cap_mask;
            }
        }
    }
#pragma unroll
    for (int r = 0; r < RPT; r++) {
        if (cs[r] >= 0) {
            atomicAdd(&rows[cs[r]], 1u);
            lean_fold<A0>(P, L, 0, tab, S, cs[r], v0[r]);
            lean_fold<A1>(P, L, 1, tab, S, cs[r], v1[r]);
        } else if (cs[r] == kDenseSlow) {
            const long long i = base + r * (long long)kFusedThreads;
            fused_slow(P, gkey, jt, key[r] == kEmptyKey ? -1 : jt_find_slot(jt, key[r]), i);
        }
    }
}

#ifndef OXB_LEAN_PAIRS
#define OXB_LEAN_PAIRS 2
#endif
// The paired-row kernels give a thread kLeanPairs pairs of rows: rows
// i + 64p and i + 64p + 1 for p < kLeanPairs, i = base + 2 * lane, so a
// warp covers a chunk of 64 * kLeanPairs consecutive rows.
constexpr int kLeanPairs = OXB_LEAN_PAIRS;
constexpr int kLeanPairRows = 2 * kLeanPairs;
constexpr int kLeanChunk = 64 * kLeanPairs;

// Row r of a thread's group starting at i.
__device__ __forceinline__ long long pair_row(long long i, int r) { return i + (r & 1) + (r >> 1) * 64; }

// A thread's rows of a 4- or 8-byte column (i even, the column 16-byte
// aligned), one vector load a pair: a warp reads 256 or 512 contiguous
// bytes per load.  Int32 values are sign-extended.
__device__ __forceinline__ void load_pairs(const void* col, int width, long long i, long long (&v)[kLeanPairRows]) {
#pragma unroll
    for (int p = 0; p < kLeanPairs; p++) {
        if (width == 8) {
            const longlong2 a = __ldcs((const longlong2*)((const long long*)col + i + 64 * p));
            v[2 * p] = a.x;
            v[2 * p + 1] = a.y;
        } else {
            const int2 a = __ldcs((const int2*)((const int*)col + i + 64 * p));
            v[2 * p] = a.x;
            v[2 * p + 1] = a.y;
        }
    }
}

// The same values in the chunk that holds the last row: one plain load per
// row below n, nothing read past it.
__device__ __forceinline__ void load_pairs_tail(const void* col, int width, long long i, long long n,
                                                long long (&v)[kLeanPairRows]) {
#pragma unroll
    for (int r = 0; r < kLeanPairRows; r++) {
        const long long j = pair_row(i, r);
        v[r] = j >= n ? 0 : width == 8 ? __ldcs((const long long*)col + j) : (long long)__ldcs((const int*)col + j);
    }
}

// lean_rows over a thread's paired rows of one request (i even, every
// column 16-byte aligned): vector loads inside full chunks, plain loads in
// the chunk that holds the last row.
template <int A0, int A1, bool DENSE>
__device__ __forceinline__ void lean_rows4(const AggProgram& P, const DevPredicate& pred, const LeanPlan& L,
                                           const LeanCols& C, const AggKey& gkey, int pk_type, const JoinTableDev& jt,
                                           const FusedTab& ft, long long i, long long n, bool full, unsigned int* rows,
                                           unsigned long long* tab, int S, unsigned long long keep) {
    const unsigned int cap_mask = jt.capacity - 1u;
    constexpr int R = kLeanPairRows;
    long long key[R], v0[R], v1[R], lv0[R], lv1[R];
#pragma unroll
    for (int r = 0; r < R; r++) v0[r] = v1[r] = lv0[r] = lv1[r] = 0;
    if (full) {
        load_pairs(C.pk, pk_type == kInt64 ? 8 : 4, i, key);
        if (L.nleaves > 0) load_pairs(C.leaf[0], L.leaf_width[0], i, lv0);
        if (L.nleaves > 1) load_pairs(C.leaf[1], L.leaf_width[1], i, lv1);
        if (A0 != kLeanNone && L.acc_leaf[0] < 0) load_pairs(C.acc[0], A0 == kLeanSumI32 ? 4 : 8, i, v0);
        if (A1 != kLeanNone && L.acc_leaf[1] < 0) load_pairs(C.acc[1], A1 == kLeanSumI32 ? 4 : 8, i, v1);
#pragma unroll
        for (int r = 0; r < R; r++) {
            if (A0 != kLeanNone && L.acc_leaf[0] >= 0) v0[r] = L.acc_leaf[0] == 0 ? lv0[r] : lv1[r];
            if (A1 != kLeanNone && L.acc_leaf[1] >= 0) v1[r] = L.acc_leaf[1] == 0 ? lv0[r] : lv1[r];
        }
    } else {
        load_pairs_tail(C.pk, pk_type == kInt64 ? 8 : 4, i, n, key);
        if (L.nleaves > 0) load_pairs_tail(C.leaf[0], L.leaf_width[0], i, n, lv0);
        if (L.nleaves > 1) load_pairs_tail(C.leaf[1], L.leaf_width[1], i, n, lv1);
        if (A0 != kLeanNone) load_pairs_tail(C.acc[0], A0 == kLeanSumI32 ? 4 : 8, i, n, v0);
        if (A1 != kLeanNone) load_pairs_tail(C.acc[1], A1 == kLeanSumI32 ? 4 : 8, i, n, v1);
    }
    int cs[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
        cs[r] = kDenseNone;
        if (pair_row(i, r) >= n) continue;
        if (L.nleaves > 0) {
            const long long a = L.leaf_f64[0] ? filter_order_key(__longlong_as_double(lv0[r])) : lv0[r];
            if (!lean_cmp(L.leaf_mask[0], a, C.lit[0])) continue;
        }
        if (L.nleaves > 1) {
            const long long a = L.leaf_f64[1] ? filter_order_key(__longlong_as_double(lv1[r])) : lv1[r];
            if (!lean_cmp(L.leaf_mask[1], a, C.lit[1])) continue;
        }
        if (key[r] == kEmptyKey) {
            if (jt.special_count) cs[r] = kDenseSlow;
            continue;
        }
        if (DENSE) {
            const unsigned long long d = (unsigned long long)key[r] - (unsigned long long)ft.dense_lo;
            if (d < ft.dense_n) cs[r] = (int)ld_keep_u32(ft.dense + d, keep);
        } else {
            unsigned int sl = (unsigned int)(fmix64((unsigned long long)key[r]) & cap_mask);
            for (unsigned int q = 0; q <= cap_mask; q++) {
                const int4 e = ld_keep_v4(&ft.slots[sl], keep);
                const long long kk = ((long long)(unsigned int)e.y << 32) | (unsigned int)e.x;
                if (kk == key[r]) {
                    cs[r] = ((unsigned int)e.w == 1u && e.z >= 0) ? e.z : kDenseSlow;
                    break;
                }
                if (kk == kEmptyKey) break;
                sl = (sl + 1u) & cap_mask;
            }
        }
    }
#pragma unroll
    for (int r = 0; r < R; r++) {
        if (cs[r] >= 0) {
            atomicAdd(&rows[cs[r]], 1u);
            lean_fold<A0>(P, L, 0, tab, S, cs[r], v0[r]);
            lean_fold<A1>(P, L, 1, tab, S, cs[r], v1[r]);
        } else if (cs[r] == kDenseSlow) {
            fused_slow(P, gkey, jt, key[r] == kEmptyKey ? -1 : jt_find_slot(jt, key[r]), pair_row(i, r));
        }
    }
}

__device__ __forceinline__ void fused_table_init(const AggProgram& P, unsigned int* rows, unsigned long long* tab,
                                                 int S) {
    for (int i = threadIdx.x; i < S; i += blockDim.x) rows[i] = 0;
    for (int i = threadIdx.x; i < S * (P.narrays - 1); i += blockDim.x) tab[S + i] = init_value(P.init[1 + i / S]);
}

#ifndef OXB_LEAN1_BLOCKS
#define OXB_LEAN1_BLOCKS 8  // resident CTAs an SM the one-row lean kernels are compiled for
#endif
#ifndef OXB_LEAN_BLOCKS
#define OXB_LEAN_BLOCKS 4  // ... the two- and four-row ones
#endif

template <int A0, int A1, bool DENSE, int RPT>
__global__ void __launch_bounds__(kFusedThreads, RPT == 1 ? OXB_LEAN1_BLOCKS : OXB_LEAN_BLOCKS) agg_lean_join_kernel(
    const __grid_constant__ AggProgram P, const __grid_constant__ DevPredicate pred, const __grid_constant__ LeanPlan L,
    const __grid_constant__ AggKey gkey, const void* __restrict__ pk, int pk_type, const __grid_constant__ JoinTableDev jt,
    const __grid_constant__ FusedTab ft, long long n) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int S = P.smem_slots;
    unsigned int* rows = (unsigned int*)smem;
    unsigned long long* tab = (unsigned long long*)(smem + fused_counts_bytes(S)) - S;
    fused_table_init(P, rows, tab, S);
    __syncthreads();
    LeanCols C;
    C.pk = pk;
    for (int l = 0; l < 2; l++) {
        C.leaf[l] = l < L.nleaves ? pred.leaves[l].values : nullptr;
        C.lit[l] = l < L.nleaves ? pred.leaves[l].lit : 0;
        C.acc[l] = L.acc_values[l];
    }
    const unsigned long long keep = policy_evict_last();
    const long long step = (long long)gridDim.x * blockDim.x * RPT;
    for (long long base = blockIdx.x * (long long)blockDim.x * RPT + threadIdx.x; base < n; base += step)
        lean_rows<A0, A1, DENSE, RPT>(P, pred, L, C, gkey, pk_type, jt, ft, base, n, rows, tab, S, keep);
    __syncthreads();
    fused_flush(P, rows, tab, S);
}

// The compiled fused kernel with four rows a thread in two pairs, each pair
// of a column one vector load (lean_rows4): half the load instructions and
// address arithmetic of four scalar rows, and four rows' loads in flight per
// thread.  Every column must start on a 16-byte boundary.
#ifndef OXB_LEAN4_BLOCKS
#define OXB_LEAN4_BLOCKS 4  // ... the paired-row ones
#endif

template <int A0, int A1, bool DENSE>
__global__ void __launch_bounds__(kFusedThreads, OXB_LEAN4_BLOCKS) agg_lean4_join_kernel(
    const __grid_constant__ AggProgram P, const __grid_constant__ DevPredicate pred, const __grid_constant__ LeanPlan L,
    const __grid_constant__ AggKey gkey, const void* __restrict__ pk, int pk_type, const __grid_constant__ JoinTableDev jt,
    const __grid_constant__ FusedTab ft, long long n) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int S = P.smem_slots;
    unsigned int* rows = (unsigned int*)smem;
    unsigned long long* tab = (unsigned long long*)(smem + fused_counts_bytes(S)) - S;
    fused_table_init(P, rows, tab, S);
    __syncthreads();
    LeanCols C;
    C.pk = pk;
    for (int l = 0; l < 2; l++) {
        C.leaf[l] = l < L.nleaves ? pred.leaves[l].values : nullptr;
        C.lit[l] = l < L.nleaves ? pred.leaves[l].lit : 0;
        C.acc[l] = L.acc_values[l];
    }
    const unsigned long long keep = policy_evict_last();
    // Warp w takes the chunks w, w + warps, ...; its lane l the rows 2l,
    // 2l + 1, 2l + 64, 2l + 65, ... of each.
    const long long warps = (long long)gridDim.x * (blockDim.x / 32);
    const int lane = threadIdx.x & 31;
    for (long long c = blockIdx.x * (long long)(blockDim.x / 32) + threadIdx.x / 32; c * kLeanChunk < n; c += warps)
        lean_rows4<A0, A1, DENSE>(P, pred, L, C, gkey, pk_type, jt, ft, c * kLeanChunk + 2 * lane, n,
                                  c * kLeanChunk + kLeanChunk <= n, rows, tab, S, keep);
    __syncthreads();
    fused_flush(P, rows, tab, S);
}

// ---- many join-aggregate requests in one launch ----------------------------
//
// Requests that differ only in their probe batch and WHERE literals (the
// same join table, group key, aggregates and comparisons) share one launch:
// their rows are cut into kLeanTile-row tiles laid end to end in one work
// queue, a CTA folds the tiles it takes into its CTA table, and when the
// next tile belongs to another request it flushes the table into that
// request's own HBM table first.  Each request's result equals its own call's.

constexpr long long kLeanTile = 8192;

struct LeanReq {
    LeanCols cols;
    long long n;
    long long tile0;  // the request's first tile in the queue
    long long* keys;  // its HBM table
    unsigned long long* arr;
    unsigned* status;
};

template <int A0, int A1, bool DENSE, int RPT>
__global__ void __launch_bounds__(kFusedThreads, 4) agg_lean_multi_kernel(
    const __grid_constant__ AggProgram P, const __grid_constant__ DevPredicate pred, const __grid_constant__ LeanPlan L,
    const __grid_constant__ AggKey gkey, int pk_type, const __grid_constant__ JoinTableDev jt,
    const __grid_constant__ FusedTab ft, const LeanReq* __restrict__ reqs, int nreq, long long ntiles,
    unsigned long long* __restrict__ queue) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ AggProgram Ps;  // P with the current request's HBM table
    __shared__ long long s_tile;
    const int S = P.smem_slots;
    unsigned int* rows = (unsigned int*)smem;
    unsigned long long* tab = (unsigned long long*)(smem + fused_counts_bytes(S)) - S;
    for (int i = threadIdx.x; i < (int)(sizeof(AggProgram) / 4); i += blockDim.x)
        ((unsigned*)&Ps)[i] = ((const unsigned*)&P)[i];
    const unsigned long long keep = policy_evict_last();
    int cur = -1;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_tile = (long long)atomicAdd(queue, 1ull);
        __syncthreads();
        const long long t = s_tile;
        if (t >= ntiles) break;
        int lo = 0, hi = nreq - 1;  // the last request whose first tile is <= t
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (reqs[mid].tile0 <= t) lo = mid;
            else hi = mid - 1;
        }
        if (lo != cur) {
            if (cur >= 0) {
                fused_flush(Ps, rows, tab, S);
                __syncthreads();
            }
            if (threadIdx.x == 0) {
                Ps.keys = reqs[lo].keys;
                Ps.arr = reqs[lo].arr;
                Ps.status = reqs[lo].status;
                // the slow paths read a row's inputs through the program
                for (int j = 0; j < Ps.nacc && j < 2; j++) Ps.acc[j].values = reqs[lo].cols.acc[j];
            }
            fused_table_init(Ps, rows, tab, S);
            __syncthreads();
            cur = lo;
        }
        const LeanReq& q = reqs[lo];
        const long long t0 = (t - q.tile0) * kLeanTile;
        const long long end = t0 + kLeanTile < q.n ? t0 + kLeanTile : q.n;
        const LeanCols C = q.cols;
        for (long long base = t0 + threadIdx.x; base < end; base += (long long)kFusedThreads * RPT)
            lean_rows<A0, A1, DENSE, RPT>(Ps, pred, L, C, gkey, pk_type, jt, ft, base, end, rows, tab, S, keep);
    }
    __syncthreads();
    if (cur >= 0) fused_flush(Ps, rows, tab, S);
}

__global__ void agg_init_kernel(const __grid_constant__ AggProgram P) {
    const long long total = (long long)P.narrays * P.stride;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x)
        P.arr[i] = init_value(P.init[i / P.stride]);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P.capacity;
         i += (long long)gridDim.x * blockDim.x)
        P.keys[i] = kEmptyKey;
}

// Occupied slots (the NULL group aside) as 0/1 flags; also the key range.
__global__ void agg_flags_kernel(const __grid_constant__ AggProgram P, unsigned int* __restrict__ flags,
                                 unsigned long long* __restrict__ range /* min, max of ordered keys */) {
    unsigned long long lo = ~0ull, hi = 0;
    const long long m = (long long)P.capacity + 2;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < m;
         s += (long long)gridDim.x * blockDim.x) {
        bool occ;
        long long key;
        if (s < P.capacity) {
            key = P.keys[s];
            occ = key != kEmptyKey;
        } else if (s == P.capacity) {
            occ = false;
            key = 0;
        } else {
            key = kEmptyKey;
            occ = P.arr[s] > 0;  // rows of the kEmptyKey group
        }
        flags[s] = occ ? 1u : 0u;
        if (occ) {
            unsigned long long u = (unsigned long long)key ^ 0x8000000000000000ull;
            lo = u < lo ? u : lo;
            hi = u > hi ? u : hi;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long a = __shfl_down_sync(0xffffffffu, lo, o);
        unsigned long long b = __shfl_down_sync(0xffffffffu, hi, o);
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&range[0], lo);
        atomicMax(&range[1], hi);
    }
}

__global__ void agg_compact_kernel(const __grid_constant__ AggProgram P, const unsigned int* __restrict__ flags,
                                   const unsigned long long* __restrict__ pos, unsigned long long lo,
                                   unsigned long long* __restrict__ skeys, unsigned int* __restrict__ sslots) {
    const long long m = (long long)P.capacity + 2;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < m;
         s += (long long)gridDim.x * blockDim.x) {
        if (!flags[s]) continue;
        long long key = s < P.capacity ? P.keys[s] : kEmptyKey;
        skeys[pos[s]] = ((unsigned long long)key ^ 0x8000000000000000ull) - lo;
        sslots[pos[s]] = (unsigned int)s;
    }
}

struct OutCol {
    void* values;
    unsigned int* validity;  // u32 words, null when the column has no bitmap
};
struct AggOutput {
    OutCol key;
    int key_type;
    OutCol cols[kMaxOuts];
};

// One output row per thread: the group at sorted position r, the NULL group last.
__global__ void agg_emit_kernel(const __grid_constant__ AggProgram P, const __grid_constant__ AggOutput O, const unsigned long long* __restrict__ skeys,
                                const unsigned int* __restrict__ sslots, unsigned long long lo, long long G,
                                long long rows) {
    const int lane = threadIdx.x & 31;
    for (long long r0 = blockIdx.x * (long long)blockDim.x; r0 < rows; r0 += (long long)gridDim.x * blockDim.x) {
        const long long r = r0 + threadIdx.x;
        const bool live = r < rows;
        const bool is_null_group = r >= G;
        long long slot = 0;
        if (live) slot = is_null_group ? (long long)P.capacity : (long long)sslots[r];
        if (live) {
            long long key = is_null_group ? 0 : (long long)((skeys[r] + lo) ^ 0x8000000000000000ull);
            if (O.key_type == kInt64) ((long long*)O.key.values)[r] = key;
            else ((int*)O.key.values)[r] = (int)key;
        }
        if (O.key.validity) {
            unsigned int bits = __ballot_sync(0xffffffffu, live && !is_null_group);
            if (lane == 0 && r < rows) O.key.validity[r >> 5] = bits;
        }
        const unsigned long long* A = P.arr;
        const long long st = P.stride;
        for (int j = 0; j < P.nout; j++) {
            const DevOut& o = P.out[j];
            bool valid = true;
            if (live) {
                const unsigned long long a0 = A[o.arr * st + slot];
                const unsigned long long nn = A[o.nn * st + slot];
                switch (o.func) {
                    case OXB_AGG_COUNT:
                    case OXB_AGG_COUNT_STAR:
                        ((unsigned long long*)O.cols[j].values)[r] = a0;
                        break;
                    case OXB_AGG_SUM:
                        valid = nn > 0;
                        if (o.in_type == kFloat64) {
                            double s = as_f64(a0), c = as_f64(A[(o.arr + 1) * st + slot]);
                            ((double*)O.cols[j].values)[r] = isfinite(s) ? __dadd_rn(s, c) : s;
                        } else {
                            ((unsigned long long*)O.cols[j].values)[r] = a0;
                        }
                        break;
                    case OXB_AGG_AVG: {
                        double s = as_f64(a0), c = as_f64(A[(o.arr + 1) * st + slot]);
                        double t = isfinite(s) ? __dadd_rn(s, c) : s;
                        ((double*)O.cols[j].values)[r] = nn ? __ddiv_rn(t, (double)nn) : 0.0;
                        valid = nn > 0;
                        break;
                    }
                    default: {
                        valid = nn > 0;
                        long long k = (long long)a0;
                        if (o.in_type == kFloat64)
                            ((double*)O.cols[j].values)[r] = valid ? from_total_order_key(k) : 0.0;
                        else if (o.in_type == kInt64)
                            ((long long*)O.cols[j].values)[r] = valid ? k : 0;
                        else
                            ((int*)O.cols[j].values)[r] = valid ? (int)k : 0;
                        break;
                    }
                }
            }
            if (O.cols[j].validity) {
                unsigned int bits = __ballot_sync(0xffffffffu, live && valid);
                if (lane == 0 && r < rows) O.cols[j].validity[r >> 5] = bits;
            }
        }
    }
}

// Distinct keys, and their range, among a strided sample of rows.
__global__ void agg_sample_kernel(const __grid_constant__ AggKey key, long long n, long long samples, long long* __restrict__ table,
                                  unsigned int tcap, unsigned long long* __restrict__ out /* distinct, min, max */) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < samples;
         i += (long long)gridDim.x * blockDim.x) {
        long long row = (long long)((double)i * (double)n / (double)samples);
        if (row >= n) row = n - 1;
        if (!valid_at(key.validity, row)) continue;
        long long k = load_int(key.values, key.type, row);
        if (k == kEmptyKey) continue;
        atomicMin((long long*)&out[1], k);
        atomicMax((long long*)&out[2], k);
        unsigned int h = (unsigned int)(fmix64((unsigned long long)k) & (tcap - 1u));
        for (unsigned int p = 0; p < tcap; p++) {
            unsigned long long old =
                atomicCAS((unsigned long long*)&table[h], (unsigned long long)kEmptyKey, (unsigned long long)k);
            if (old == (unsigned long long)kEmptyKey) {
                atomicAdd(&out[0], 1ull);
                break;
            }
            if ((long long)old == k) break;
            h = (h + 1u) & (tcap - 1u);
        }
    }
}

// The largest finite |x| over a strided sample of a Float64 column, as the
// bits of a non-negative double (whose integer order is its value order).
__global__ void f64_absmax_sample_kernel(const double* __restrict__ v, const uint8_t* __restrict__ valid, long long n,
                                         long long samples, unsigned long long* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < samples;
         i += (long long)gridDim.x * blockDim.x) {
        long long row = (long long)((double)i * (double)n / (double)samples);
        if (row >= n) row = n - 1;
        if (!valid_at(valid, row)) continue;
        const double x = fabs(__ldg(v + row));
        if (isfinite(x) && x != 0.0) atomicMax(out, as_u64(x));
    }
}

__global__ void fill_i64_kernel(long long* p, long long n, long long v) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = v;
}

unsigned int next_pow2(long long v, long long floor_v) {
    long long c = floor_v;
    while (c < v) c <<= 1;
    if (c > (1ll << 31)) fail(OXB_UNSUPPORTED, "aggregate of more than 2^30 groups");
    return (unsigned int)c;
}

// One aggregate as the kernels read it: a column of the input (side 0) or of
// the build side (side 1); no column for COUNT(*).
struct AggInputCol {
    const Column* col;
    int side;
    int index = -1;  // the column's index when it names a column of many batches
};

struct AggPlan {
    AggProgram P{};
    int acc_index[kMaxAccs];  // each accumulator's column index (-1 when not given)
    std::vector<int> out_types;
    int key_type = kInt64;
    long long acc_rows = 0;  // rows of the side the accumulators read (fused join kernels)
};

AggPlan plan_aggregate(const std::vector<int>& funcs, const std::vector<AggInputCol>& inputs, int key_type) {
    AggPlan plan;
    AggProgram& P = plan.P;
    int na = 1;  // array 0: rows per group
    P.init[0] = kInitZero;
    P.merge[0] = kMergeAddU64;
    auto add_array = [&](unsigned char init, unsigned char merge) {
        P.init[na] = init;
        P.merge[na] = merge;
        return na++;
    };
    // Accumulators are shared by every aggregate that needs the same one.
    // By column index when given (batches whose buffers differ), else by buffer.
    auto acc_for = [&](int kind, const Column* c, int side, int index) -> int {
        for (int j = 0; j < P.nacc; j++) {
            const bool same = index >= 0 ? plan.acc_index[j] == index
                                         : P.acc[j].values == c->values && P.acc[j].validity == c->validity;
            if (P.acc[j].kind == kind && same && P.acc[j].side == side && P.acc[j].in_type == c->type)
                return P.acc[j].arr;
        }
        if (P.nacc == kMaxAccs) fail(OXB_UNSUPPORTED, "too many distinct aggregate inputs");
        plan.acc_index[P.nacc] = index;
        DevAcc& a = P.acc[P.nacc++];
        a.values = c->values;
        a.validity = c->validity;
        a.kind = kind;
        a.in_type = c->type;
        a.side = side;
        switch (kind) {
            case kAccSumF64:
                a.arr = add_array(kInitZero, kMergeAddF64Comp);
                add_array(kInitZero, kMergeAddF64);
                break;
            case kAccMin: a.arr = add_array(kInitMax, kMergeMin); break;
            case kAccMax: a.arr = add_array(kInitMin, kMergeMax); break;
            default: a.arr = add_array(kInitZero, kMergeAddU64); break;
        }
        return a.arr;
    };
    P.nout = (int)funcs.size();
    for (int j = 0; j < P.nout; j++) {
        DevOut& o = P.out[j];
        o.func = funcs[j];
        const Column* c = inputs[j].col;
        const int side = inputs[j].side;
        o.in_type = c ? c->type : kInt64;
        // Rows with a non-NULL input: the group's rows when the column has no bitmap.
        const int index = inputs[j].index;
        auto nn = [&]() { return c && c->validity ? acc_for(kAccCount, c, side, index) : 0; };
        int out_type = kInt64;
        switch (o.func) {
            case OXB_AGG_COUNT_STAR:
                o.arr = 0;
                o.nn = 0;
                break;
            case OXB_AGG_COUNT:
                o.arr = nn();
                o.nn = 0;
                break;
            case OXB_AGG_SUM:
                o.arr = acc_for(o.in_type == kFloat64 ? kAccSumF64 : kAccSumInt, c, side, index);
                o.nn = nn();
                out_type = o.in_type == kFloat64 ? kFloat64 : kInt64;
                break;
            case OXB_AGG_AVG:
                o.arr = acc_for(kAccSumF64, c, side, index);
                o.nn = nn();
                out_type = kFloat64;
                break;
            case OXB_AGG_MIN:
                o.arr = acc_for(kAccMin, c, side, index);
                o.nn = nn();
                out_type = o.in_type;
                break;
            case OXB_AGG_MAX:
                o.arr = acc_for(kAccMax, c, side, index);
                o.nn = nn();
                out_type = o.in_type;
                break;
            default:
                fail(OXB_PLAN, "unknown aggregate function " + std::to_string(o.func));
        }
        plan.out_types.push_back(out_type);
    }
    P.narrays = na;
    plan.key_type = key_type;
    return plan;
}

void check_agg_input(int func, const Column* c, int index) {
    if (func == OXB_AGG_COUNT_STAR) return;
    if (!c) fail(OXB_PLAN, "aggregate input column missing");
    if (c->type != kInt64 && c->type != kFloat64 && c->type != kInt32)
        fail(OXB_UNSUPPORTED, "aggregate input column " + std::to_string(index) + " has type " +
                                  std::to_string(c->type) + "; Int64, Int32 and Float64 run on the device");
}

// One compiled shape of the row-loop kernels: the accumulator bound, warp
// combining, and rows per thread per step.  The autotuner picks among them.
struct AggVariant {
    int maxacc;
    bool combine;
    int rpt;
    bool tile;    // the tile sort-reduce kernels (combine/rpt unused)
    bool stream = false;  // the streamed kernels (combine/rpt unused)
    bool stile = false;   // the streamed tile sort-reduce kernels
    bool fused = false;   // the fused probe-table join kernel (rpt used)
    bool dense = false;   // ... with the dense lookup table
    bool vec = false;     // ... interpreted a vector of rows at a time (rpt 4 or 8)
    bool fstream = false; // ... fed by streamed columns (agg_fstream_join_kernel)
    bool lean = false;    // ... compiled per accumulator shape (agg_lean_join_kernel)
    bool lean4 = false;   // ... four rows a thread in two vector-loaded pairs (agg_lean4_join_kernel)
};

// The streamed kernels' plan: the probe-side columns (deduplicated) with
// their places in a stage, and the slot-major CTA-table layout (Float64
// (sum, compensation) pairs first, on even words).  False when a column
// cannot be streamed (a base not 16-byte aligned, too many columns).
bool plan_stream(const AggProgram& P, const DevPredicate& pred, const void* key_values, const uint8_t* key_validity,
                 int key_type, long long n, StreamPlan* SP) {
    *SP = StreamPlan{};
    auto add = [&](const void* values, const uint8_t* validity, int type) -> int {
        for (int c = 0; c < SP->ncols; c++)
            if (SP->cols[c].values == values && SP->cols[c].validity == validity) return c;
        if (SP->ncols == kMaxStreamCols) return -2;
        if (((uintptr_t)values & 15) || ((uintptr_t)validity & 15)) return -2;
        if (type != kInt64 && type != kFloat64 && type != kInt32) return -2;
        StreamCol& c = SP->cols[SP->ncols];
        c.values = values;
        c.validity = validity;
        c.type = type;
        c.width = type_width(type, 1);
        return SP->ncols++;
    };
    for (int l = 0; l < pred.nleaves; l++) {
        SP->leaf_col[l] = add(pred.leaves[l].values, pred.leaves[l].validity, pred.leaves[l].type);
        if (SP->leaf_col[l] < 0) return false;
    }
    SP->key_col = add(key_values, key_validity, key_type);
    if (SP->key_col < 0) return false;
    for (int j = 0; j < P.nacc; j++) {
        SP->acc_col[j] = -1;
        if (P.acc[j].side != 0) continue;
        SP->acc_col[j] = add(P.acc[j].values, P.acc[j].validity, P.acc[j].in_type);
        if (SP->acc_col[j] < 0) return false;
    }
    int off = 0;
    SP->tx_bytes = 0;
    for (int c = 0; c < SP->ncols; c++) {
        SP->cols[c].voff = off;
        off += kStreamT * SP->cols[c].width;
        SP->tx_bytes += kStreamT * SP->cols[c].width + (SP->cols[c].validity ? kStreamT / 8 : 0);
        SP->cols[c].boff = -1;
        if (SP->cols[c].validity) {
            SP->cols[c].boff = off;
            off += kStreamT / 8;
        }
        off = (off + 127) & ~127;
    }
    SP->stage_bytes = off;
    SP->n = n;
    SP->ntiles = (n + kStreamT - 1) / kStreamT;
    int w = 0;
    for (int a = 0; a < P.narrays; a++)
        if (P.merge[a] == kMergeAddF64Comp) {
            SP->aos_idx[a] = w;
            SP->aos_idx[a + 1] = w + 1;
            w += 2;
        }
    for (int a = 0; a < P.narrays; a++) {
        if (P.merge[a] == kMergeAddF64Comp) {
            a++;
            continue;
        }
        SP->aos_idx[a] = w++;
    }
    SP->aos = (w + 1) & ~1;
    return true;
}


// ---- many batches, one persistent launch ----------------------------------
//
// GpuAggregateExec folds every RecordBatch of a partition into one result
// (compute/src/exec/aggregate.rs:35-321); the reference runs one device
// aggregate per batch and merges on the host.  Here every batch's columns
// are described once in HBM and a persistent kernel takes 4096-row tiles of
// all batches from one work queue (uneven batch sizes cost nothing extra),
// folding into one HBM table sized from a HyperLogLog count of the keys.

struct BatchCols {
    long long n;      // rows
    long long tile0;  // the batch's first tile in the queue
    long long ptile0; // ... in the partitioning passes' queue (kPartTile rows per tile)
    const void* key;
    const uint8_t* key_valid;
    const void* vals[kMaxAccs];
    const uint8_t* valid[kMaxAccs];
    const void* lvals[kMaxLeaves];
    const uint8_t* lvalid[kMaxLeaves];
};

constexpr int kBatchTile = 4096;

template <int MAXACC>
__global__ void __launch_bounds__(kThreads) agg_batches_kernel(const __grid_constant__ AggProgram P,
                                                               const __grid_constant__ DevPredicate pred, int key_type,
                                                               const BatchCols* __restrict__ batches, int nb,
                                                               long long ntiles,
                                                               unsigned long long* __restrict__ queue) {
    __shared__ long long s_tile;
    __shared__ int s_b;
    // The first tiles of the first kTile0Cache batches, searched in shared
    // memory (the descriptors are large: a search in HBM costs a round trip
    // a step); a tile of a later batch searches HBM.
    constexpr int kTile0Cache = 2048;
    __shared__ long long s_tile0[kTile0Cache];
    const int cached = nb < kTile0Cache ? nb : kTile0Cache;
    for (int i = threadIdx.x; i < cached; i += blockDim.x) s_tile0[i] = batches[i].tile0;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            const long long t = (long long)atomicAdd(queue, 1ull);
            const bool far = cached < nb && batches[cached].tile0 <= t;
            int lo = far ? cached : 0, hi = far ? nb - 1 : cached - 1;  // the last batch whose first tile is <= t
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if ((far ? batches[mid].tile0 : s_tile0[mid]) <= t) lo = mid;
                else hi = mid - 1;
            }
            s_tile = t;
            s_b = lo;
        }
        __syncthreads();
        const long long t = s_tile;
        if (t >= ntiles) break;
        const BatchCols& B = batches[s_b];
        const long long base = (t - B.tile0) * kBatchTile;
        for (int i = threadIdx.x; i < kBatchTile; i += blockDim.x) {
            const long long r = base + i;
            if (r >= B.n) break;
            bool keep = true;
            for (int l = 0; l < pred.nleaves; l++) {
                const DevLeaf& lf = pred.leaves[l];
                if (!valid_at(B.lvalid[l], r)) {
                    keep = false;
                    break;
                }
                const long long a = lf.type == kFloat64 ? filter_order_key(__ldg((const double*)B.lvals[l] + r))
                                    : lf.type == kInt64 ? __ldg((const long long*)B.lvals[l] + r)
                                                        : (long long)__ldg((const int*)B.lvals[l] + r);
                if (!cmp_holds(lf.op, a, lf.lit)) {
                    keep = false;
                    break;
                }
            }
            if (!keep) continue;
            const bool kv = valid_at(B.key_valid, r);
            const long long key = kv ? load_int(B.key, key_type, r) : 0;
            const long long g = global_slot(P, kv, key);
            if (g < 0) continue;
            unsigned long long val[MAXACC];
            double comp[MAXACC];
#pragma unroll
            for (int j = 0; j < MAXACC; j++) {
                comp[j] = 0.0;
                if (j >= P.nacc) break;
                const DevAcc& a = P.acc[j];
                const bool v = valid_at(B.valid[j], r);
                long long raw = 0;
                if (v && a.kind != kAccCount)
                    raw = a.in_type == kInt32 ? (long long)__ldg((const int*)B.vals[j] + r)
                                              : __ldg((const long long*)B.vals[j] + r);
                val[j] = contribution_raw(a.kind, a.in_type, v, raw);
            }
            apply_vals<MAXACC>(P, P.arr, P.stride, g, 1, val, comp);
        }
    }
}

// HyperLogLog registers of the non-NULL keys (4096 registers: about 1.6 %
// standard error), to size the table before the fold.
constexpr int kHllBits = 12;
constexpr int kHllRegs = 1 << kHllBits;

double as_f64_host(unsigned long long u) {
    double d;
    std::memcpy(&d, &u, sizeof d);
    return d;
}

double hll_estimate(const std::vector<unsigned>& regs) {
    double sum = 0.0;
    int zeros = 0;
    for (unsigned r : regs) {
        sum += std::ldexp(1.0, -(int)r);
        zeros += r == 0;
    }
    const double m = (double)regs.size();
    double e = 0.7213 / (1.0 + 1.079 / m) * m * m / sum;
    if (e <= 2.5 * m && zeros > 0) e = m * std::log(m / zeros);
    return e;
}


// ---- hash-partitioned folding, for many groups ------------------------------
// With millions of groups the HBM table does not fit in L2 and the direct
// fold costs about six random HBM accesses per row.  Instead the kept rows
// are partitioned by the top bits of their key's hash, so that each final
// partition holds a few hundred groups, and each partition is folded in a
// shared-memory table of its own keys; each group then reaches the HBM table
// once.  Partitions split the key space, so no two CTAs fold the same group.
//
//   count   kept rows per final partition (a shared histogram per CTA)
//   split1  rows -> records (key, stored columns, validity byte) in F1 <= 128
//           level-1 partitions: each 2048-row sub-tile reserves its slice of
//           a partition with one atomic, so concurrent writes stay adjacent
//   split2  each level-1 partition -> its F2 final partitions, alike
//   fold    one final partition at a time in shared memory; keys that do not
//           fit fold into HBM directly
//
// NULL keys and the key INT64_MIN fold into their HBM slots during split1.
// A record is a whole number of 16-byte units: word 0 the key, then for one
// Int32 column its value and the validity byte in word 1 (16 bytes), else
// one word per column and a word of validity bits.

constexpr int kPartTile = 8192;  // rows per tile of the count pass and the HLL
constexpr int kSplitRows = 8;    // rows per thread in a split sub-tile
constexpr int kSplitTile = kThreads * kSplitRows;
constexpr int kMaxParts = 32768;
constexpr int kMaxF1 = 128;
constexpr int kMaxF2 = kMaxParts / kMaxF1;
constexpr int kPartKeys = 256;   // keys per final partition the sizing aims at
constexpr int kPartSlots = 1024; // shared slots of the fold (3/4 may fill)
constexpr int kPartSlotBits = 10;
static_assert(kPartSlots == 1 << kPartSlotBits, "the fold's slots are a power of two");
constexpr int kFoldRows = 4;     // rows in flight per thread in the fold
constexpr int kScanThreads = 1024;  // the scan pass: one CTA per SM (shared fine histogram)
constexpr int kFineBits = 15;       // fine histogram buckets: the top 15 bits of the partition hash
constexpr int kFine = 1 << kFineBits;
static_assert(kMaxParts == kFine, "final partitions are unions of fine buckets");
constexpr unsigned long long kPartSeed = 0x5BD1E9955BD1E995ull;

struct PartPlan {
    int nparts;   // final partitions: a power of two
    int shift;    // 64 - log2(nparts)
    int f2_bits;  // log2(F2): final partition = level-1 partition * F2 + p2
    int fstride;  // fine buckets per final partition: partition p starts at offs[p * fstride]
    int ncols;    // input columns stored per record
    bool compact; // one Int32 column: 16-byte records
    int col_of_acc[kMaxAccs];  // the stored column an accumulator reads
    int width[kMaxAccs];       // bytes per stored column (4 or 8)
    int src_of_col[kMaxAccs];  // an accumulator reading each stored column
    uint4* recs;   // level-1 partitions
    uint4* recs2;  // final partitions (recs again when F2 == 1)
};

__device__ __forceinline__ unsigned long long part_hash(long long key) {
    return fmix64((unsigned long long)key ^ kPartSeed);
}

__device__ __forceinline__ int part_of(const PartPlan& pp, long long key) { return (int)(part_hash(key) >> pp.shift); }

// The batch holding partitioning tile t: the last whose first tile is <= t.
__device__ __forceinline__ int batch_of_tile(const BatchCols* batches, int nb, long long t) {
    int lo = 0, hi = nb - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (batches[mid].ptile0 <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The same search over a shared copy of the first 2048 batches' first tiles
// (`cached` of them): a tile whose batch is past them searches HBM.
constexpr int kTileCache = 2048;
__device__ __forceinline__ int batch_of_tile_cached(const long long* ptile0, int cached, const BatchCols* batches,
                                                    int nb, long long t) {
    if (cached < nb && batches[cached].ptile0 <= t) return cached + batch_of_tile(batches + cached, nb - cached, t);
    int lo = 0, hi = cached - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (ptile0[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Rows r0 + j * T (j < R, below `end`) that pass the WHERE and have a
// valid key, with their keys.  The keys are loaded with the first leaf's
// values, before any test: one memory round trip instead of two, for
// 8 bytes more a row that the WHERE drops.
template <int R, int T = kThreads>
__device__ __forceinline__ unsigned kept_keys(const DevPredicate& pred, const BatchCols& B, int key_type, long long r0,
                                              long long end, long long* key, unsigned* nullkey) {
    unsigned live = 0;
#pragma unroll
    for (int j = 0; j < R; j++)
        if (r0 + (long long)j * T < end) live |= 1u << j;
    unsigned kvalid = 0;
#pragma unroll
    for (int j = 0; j < R; j++) {
        const long long r = r0 + (long long)j * T;
        key[j] = 0;
        if (!((live >> j) & 1u)) continue;
        if (valid_at(B.key_valid, r)) {
            kvalid |= 1u << j;
            key[j] = load_int(B.key, key_type, r);
        }
    }
    unsigned keep = live;
    for (int l = 0; l < pred.nleaves; l++) {
        const DevLeaf& lf = pred.leaves[l];
        long long a[R];
#pragma unroll
        for (int j = 0; j < R; j++) {
            const long long r = r0 + (long long)j * T;
            a[j] = 0;
            if (!((keep >> j) & 1u)) continue;
            if (!valid_at(B.lvalid[l], r)) {
                keep &= ~(1u << j);
                continue;
            }
            a[j] = lf.type == kFloat64 ? filter_order_key(__ldg((const double*)B.lvals[l] + r))
                   : lf.type == kInt64 ? __ldg((const long long*)B.lvals[l] + r)
                                       : (long long)__ldg((const int*)B.lvals[l] + r);
        }
#pragma unroll
        for (int j = 0; j < R; j++)
            if (((keep >> j) & 1u) && !cmp_holds(lf.op, a[j], lf.lit)) keep &= ~(1u << j);
    }
    unsigned nk = keep & ~kvalid;
#pragma unroll
    for (int j = 0; j < R; j++)
        if (((keep & kvalid) >> j) & 1u && key[j] == kEmptyKey) nk |= 1u << j;
    *nullkey = nk;  // kept rows whose key is NULL or INT64_MIN
    return keep & ~nk;
}

// kept_keys for the dense passes, with every load issued up front: a row
// index past `end` is clamped to end - 1 (in bounds, its result masked
// off), so the loads of all R rows are unconditional and independent, and
// each column's type and bitmap test sits outside the loops over rows.
// With X, accumulator q's Int32 values and validity come in the same batch
// (values of rows without a valid value read as 0).
template <int R, int T, bool X>
__device__ __forceinline__ unsigned kept_keys_eager(const DevPredicate& pred, const BatchCols& B, int key_type,
                                                    long long r0, long long end, long long* key, unsigned* nullkey,
                                                    int q, int* xv, unsigned* xvalid) {
    unsigned live = 0;
#pragma unroll
    for (int j = 0; j < R; j++)
        if (r0 + (long long)j * T < end) live |= 1u << j;
    *nullkey = 0;
    if (!live) return 0;
    const long long last = end - 1;
#define OXB_ROW(j) (r0 + (long long)(j) * T < last ? r0 + (long long)(j) * T : last)
    if (key_type == kInt64) {
        const long long* kp = (const long long*)B.key;
#pragma unroll
        for (int j = 0; j < R; j++) key[j] = __ldg(kp + OXB_ROW(j));
    } else {
        const int* kp = (const int*)B.key;
#pragma unroll
        for (int j = 0; j < R; j++) key[j] = (long long)__ldg(kp + OXB_ROW(j));
    }
    if (X) {
        const int* xp = (const int*)B.vals[q];
#pragma unroll
        for (int j = 0; j < R; j++) xv[j] = __ldg(xp + OXB_ROW(j));
    }
    unsigned kvalid = live;
    if (B.key_valid) {
#pragma unroll
        for (int j = 0; j < R; j++)
            if (!valid_at(B.key_valid, OXB_ROW(j))) kvalid &= ~(1u << j);
    }
    unsigned keep = live;
    for (int l = 0; l < pred.nleaves; l++) {
        const DevLeaf& lf = pred.leaves[l];
        if (lf.type == kInt32) {
            const int* ap = (const int*)B.lvals[l];
            int a[R];
#pragma unroll
            for (int j = 0; j < R; j++) a[j] = __ldg(ap + OXB_ROW(j));
#pragma unroll
            for (int j = 0; j < R; j++)
                if (!cmp_holds(lf.op, (long long)a[j], lf.lit)) keep &= ~(1u << j);
        } else {
            const long long* ap = (const long long*)B.lvals[l];
            long long a[R];
#pragma unroll
            for (int j = 0; j < R; j++) a[j] = __ldg(ap + OXB_ROW(j));
            if (lf.type == kFloat64) {
#pragma unroll
                for (int j = 0; j < R; j++) a[j] = filter_order_key(__longlong_as_double(a[j]));
            }
#pragma unroll
            for (int j = 0; j < R; j++)
                if (!cmp_holds(lf.op, a[j], lf.lit)) keep &= ~(1u << j);
        }
        if (B.lvalid[l]) {
#pragma unroll
            for (int j = 0; j < R; j++)
                if (!valid_at(B.lvalid[l], OXB_ROW(j))) keep &= ~(1u << j);
        }
    }
    if (X) {
        unsigned xm = keep;
        if (B.valid[q]) {
#pragma unroll
            for (int j = 0; j < R; j++)
                if (!valid_at(B.valid[q], OXB_ROW(j))) xm &= ~(1u << j);
        }
#pragma unroll
        for (int j = 0; j < R; j++)
            if (!((xm >> j) & 1u)) xv[j] = 0;
        *xvalid = xm;
    }
#undef OXB_ROW
    unsigned nk = keep & ~kvalid;
#pragma unroll
    for (int j = 0; j < R; j++)
        if (((keep & kvalid) >> j) & 1u && key[j] == kEmptyKey) nk |= 1u << j;
    *nullkey = nk;
    return keep & ~nk;
}

// The one pass over the input before the fold: for the kept rows with a
// valid key (not INT64_MIN), (1) HyperLogLog registers of their keys
// (2^kHllBits registers: a key's register is the top bits of its partition
// hash, its rank the leading zeros of the rest plus one), which size the
// HBM table and pick the path; (2) their count; (3) their histogram over
// kFine buckets (the top kFineBits bits of the same hash), from which the
// partitioned path takes every partition's size.
__global__ void __launch_bounds__(kScanThreads) part_scan_kernel(const __grid_constant__ DevPredicate pred, int key_type,
                                                                 const BatchCols* __restrict__ batches, int nb,
                                                                 long long ntiles, unsigned* __restrict__ regs,
                                                                 unsigned int* __restrict__ fine,
                                                                 unsigned long long* __restrict__ kept) {
    extern __shared__ unsigned int scan_smem[];
    unsigned* sr = scan_smem;             // kHllRegs
    unsigned* hist = scan_smem + kHllRegs;  // kFine
    for (int i = threadIdx.x; i < kHllRegs + kFine; i += blockDim.x) scan_smem[i] = 0;
    __syncthreads();
    unsigned n = 0;
    // A contiguous range of tiles a CTA, stepping from batch to batch (no
    // search per tile).
    const long long t0 = ntiles * blockIdx.x / gridDim.x, t1 = ntiles * (blockIdx.x + 1) / gridDim.x;
    int bi = t0 < t1 ? batch_of_tile(batches, nb, t0) : 0;
    for (long long t = t0; t < t1; t++) {
        while (bi + 1 < nb && batches[bi + 1].ptile0 <= t) bi++;
        const BatchCols& B = batches[bi];
        const long long base = (t - B.ptile0) * kPartTile;
        const long long end = base + kPartTile < B.n ? base + kPartTile : B.n;
        for (long long r0 = base + threadIdx.x; r0 < end; r0 += (long long)kScanThreads * 4) {
            long long key[4];
            unsigned nk;
            const unsigned m = kept_keys<4, kScanThreads>(pred, B, key_type, r0, end, key, &nk);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (!((m >> j) & 1u)) continue;
                const unsigned long long h = part_hash(key[j]);
                const unsigned rank = (unsigned)__clzll((h << kHllBits) | (1ull << (kHllBits - 1))) + 1u;
                atomicMax(&sr[h >> (64 - kHllBits)], rank);
                atomicAdd(&hist[h >> (64 - kFineBits)], 1u);
                n++;
            }
        }
    }
    // kept rows: a warp sum, then one atomic a warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(kept, (unsigned long long)n);
    __syncthreads();
    for (int i = threadIdx.x; i < kHllRegs; i += blockDim.x)
        if (sr[i]) atomicMax(&regs[i], sr[i]);
    for (int i = threadIdx.x; i < kFine; i += blockDim.x)
        if (hist[i]) atomicAdd(&fine[i], hist[i]);
}

// Split pass 1: tiles of rows from a queue; each sub-tile of kSplitTile rows
// ranks its kept rows per level-1 partition in shared memory, reserves each
// partition's slice with one atomic on cursor1, and writes the records.
// A kept row whose group key is NULL or INT64_MIN: straight into its HBM
// slot (out of line: rare, and kept out of the split's instruction cache).
template <int MAXACC>
__device__ __noinline__ void part_null_row_to_hbm(const AggProgram& P, const BatchCols& B, long long r) {
    const bool kv = valid_at(B.key_valid, r);
    unsigned long long val[MAXACC];
    double comp[MAXACC];
#pragma unroll
    for (int q = 0; q < MAXACC; q++) {
        val[q] = 0;
        comp[q] = 0.0;
        if (q >= P.nacc) continue;
        const DevAcc& a = P.acc[q];
        const bool v = valid_at(B.valid[q], r);
        long long raw = 0;
        if (v && a.kind != kAccCount)
            raw = a.in_type == kInt32 ? (long long)__ldg((const int*)B.vals[q] + r) : __ldg((const long long*)B.vals[q] + r);
        val[q] = contribution_raw(a.kind, a.in_type, v, raw);
    }
    const long long g = global_slot(P, kv, kv ? kEmptyKey : 0);
    if (g >= 0) apply_vals<MAXACC>(P, P.arr, P.stride, g, 1, val, comp);
}

#ifndef OXB_SPLIT1_BLOCKS
#define OXB_SPLIT1_BLOCKS 4  // resident CTAs an SM split1 is compiled for (64 registers)
#endif
// COMPACT: 16-byte records of one Int32 column (PartPlan::compact), else wider ones.
template <int MAXACC, bool COMPACT>
__global__ void __launch_bounds__(kThreads, OXB_SPLIT1_BLOCKS) part_split1_kernel(const __grid_constant__ AggProgram P,
                                                               const __grid_constant__ DevPredicate pred, int key_type,
                                                               const BatchCols* __restrict__ batches, int nb,
                                                               long long ntiles, unsigned long long* __restrict__ queue,
                                                               const __grid_constant__ PartPlan pp,
                                                               unsigned long long* __restrict__ cursor1) {
    __shared__ unsigned int hist[kMaxF1];
    __shared__ unsigned long long base1[kMaxF1];
    __shared__ long long s_tile;
    __shared__ long long s_ptile0[kTileCache];
    const int f1 = pp.nparts >> pp.f2_bits;
    const int cached = nb < kTileCache ? nb : kTileCache;
    for (int i = threadIdx.x; i < cached; i += blockDim.x) s_ptile0[i] = batches[i].ptile0;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_tile = (long long)atomicAdd(queue, 1ull);
        __syncthreads();
        const long long t = s_tile;
        if (t >= ntiles) break;
        const BatchCols& B = batches[batch_of_tile_cached(s_ptile0, cached, batches, nb, t)];
        const long long tbase = (t - B.ptile0) * kPartTile;
        const long long tend = tbase + kPartTile < B.n ? tbase + kPartTile : B.n;
        for (long long sub = tbase; sub < tend; sub += kSplitTile) {
            if (threadIdx.x < kMaxF1) hist[threadIdx.x] = 0;
            __syncthreads();
            long long key[kSplitRows];
            unsigned nk;
            const unsigned m = kept_keys<kSplitRows>(pred, B, key_type, sub + threadIdx.x, tend, key, &nk);
            // One Int32 column (16-byte records): its values and validity
            // are loaded now, while the partition cursors are reserved.
            int xv[kSplitRows];
            unsigned xvalid = 0;
            if (COMPACT) {
                const int q = pp.src_of_col[0];
#pragma unroll
                for (int j = 0; j < kSplitRows; j++) {
                    const long long r = sub + threadIdx.x + (long long)j * kThreads;
                    xv[j] = 0;
                    if (!((m >> j) & 1u) || !valid_at(B.valid[q], r)) continue;
                    xvalid |= 1u << j;
                    xv[j] = __ldg((const int*)B.vals[q] + r);
                }
            }
            unsigned rank[kSplitRows];
#pragma unroll
            for (int j = 0; j < kSplitRows; j++) {
                rank[j] = 0;
                if ((m >> j) & 1u) {
                    const int p1 = part_of(pp, key[j]) >> pp.f2_bits;
                    rank[j] = (unsigned)p1 << 24 | atomicAdd(&hist[p1], 1u);
                }
            }
            __syncthreads();
            if (threadIdx.x < f1 && hist[threadIdx.x])
                base1[threadIdx.x] = atomicAdd(&cursor1[threadIdx.x], (unsigned long long)hist[threadIdx.x]);
            __syncthreads();
            if (COMPACT) {
                // 16-byte records: a short store a row, unrolled.
#pragma unroll
                for (int j = 0; j < kSplitRows; j++) {
                    if ((nk >> j) & 1u) {
                        part_null_row_to_hbm<MAXACC>(P, B, sub + threadIdx.x + (long long)j * kThreads);
                    } else if ((m >> j) & 1u) {
                        const unsigned long long pos = base1[rank[j] >> 24] + (rank[j] & 0xFFFFFFu);
                        pp.recs[pos] = make_uint4((unsigned)key[j], (unsigned)((unsigned long long)key[j] >> 32),
                                                  (unsigned)xv[j], (xvalid >> j) & 1u);
                    }
                }
                continue;
            }
            // Wider records one row at a time from a register queue: a
            // single copy of the row code, which stays in the instruction cache.
            unsigned mm = m, nn = nk;
#pragma unroll 1
            for (int j = 0; j < kSplitRows && (mm | nn); j++) {
                const long long r = sub + threadIdx.x + (long long)j * kThreads;
                if (nn & 1u) {
                    part_null_row_to_hbm<MAXACC>(P, B, r);
                } else if (mm & 1u) {
                    const unsigned long long pos = base1[rank[0] >> 24] + (rank[0] & 0xFFFFFFu);
                    unsigned long long w[MAXACC + 2];  // key, columns, validity
                    unsigned long long flags = 0;
#pragma unroll
                    for (int i = 0; i < MAXACC + 2; i++) w[i] = 0;
                    w[0] = (unsigned long long)key[0];
#pragma unroll
                    for (int c = 0; c < MAXACC; c++) {
                        if (c >= pp.ncols) break;
                        const int q = pp.src_of_col[c];
                        const bool v = valid_at(B.valid[q], r);
                        flags |= (unsigned long long)v << c;
                        if (v)
                            w[1 + c] = pp.width[c] == 4 ? (unsigned long long)(long long)__ldg((const int*)B.vals[q] + r)
                                                        : (unsigned long long)__ldg((const long long*)B.vals[q] + r);
                    }
#pragma unroll
                    for (int i = 1; i < MAXACC + 2; i++)
                        if (i == 1 + pp.ncols) w[i] = flags;
                    const int units = (pp.ncols + 3) >> 1;
                    uint4* o = pp.recs + pos * units;
#pragma unroll
                    for (int u = 0; u < (MAXACC + 2) / 2; u++)
                        if (u < units)
                            o[u] = make_uint4((unsigned)w[2 * u], (unsigned)(w[2 * u] >> 32), (unsigned)w[2 * u + 1],
                                              (unsigned)(w[2 * u + 1] >> 32));
                }
                mm >>= 1;
                nn >>= 1;
#pragma unroll
                for (int t = 0; t + 1 < kSplitRows; t++) {
                    key[t] = key[t + 1];
                    rank[t] = rank[t + 1];
                }
            }
        }
    }
}

// The first split-2 tile of each level-1 partition (kSplitTile records a
// tile) and, at [f1], their total.
__global__ void part_tiles_kernel(const unsigned long long* __restrict__ offs, int f1, int f2, int fstride,
                                  long long* __restrict__ tstart) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    long long t = 0;
    const long long step = (long long)f2 * fstride;  // fine buckets a level-1 partition
    for (int i = 0; i < f1; i++) {
        tstart[i] = t;
        const unsigned long long n = offs[(i + 1) * step] - offs[i * step];
        t += (long long)((n + kSplitTile - 1) / kSplitTile);
    }
    tstart[f1] = t;
}

// Split pass 2: tiles of one level-1 partition's records from a queue, each
// ranked per final partition in shared memory, reserved with one atomic per
// final partition on cursor2 and copied.
template <int UNITS>
__global__ void __launch_bounds__(kThreads) part_split2_kernel(const __grid_constant__ PartPlan pp,
                                                               const unsigned long long* __restrict__ offs,
                                                               const long long* __restrict__ tstart,
                                                               unsigned long long* __restrict__ queue,
                                                               unsigned long long* __restrict__ cursor2) {
    __shared__ unsigned int hist[kMaxF2];
    __shared__ unsigned long long base2[kMaxF2];
    __shared__ long long s_tile;
    const int f2 = 1 << pp.f2_bits, f1 = pp.nparts >> pp.f2_bits;
    const long long ntiles = tstart[f1];
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_tile = (long long)atomicAdd(queue, 1ull);
        __syncthreads();
        const long long t = s_tile;
        if (t >= ntiles) break;
        int lo = 0, hi = f1 - 1;  // the last level-1 partition whose first tile is <= t
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (tstart[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const int p1 = lo;
        const long long step = (long long)f2 * pp.fstride;
        const unsigned long long first = offs[p1 * step] + (unsigned long long)(t - tstart[p1]) * kSplitTile;
        const unsigned long long last = offs[(p1 + 1) * step];
        const unsigned long long end = first + kSplitTile < last ? first + kSplitTile : last;
        for (int i = threadIdx.x; i < kMaxF2; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        uint4 rec[kSplitRows][UNITS];
        unsigned rank[kSplitRows];
#pragma unroll
        for (int j = 0; j < kSplitRows; j++) {
            const unsigned long long i = first + threadIdx.x + (unsigned long long)j * kThreads;
            rank[j] = 0xFFFFFFFFu;
            if (i >= end) continue;
#pragma unroll
            for (int u = 0; u < UNITS; u++) rec[j][u] = __ldcs(pp.recs + i * UNITS + u);
        }
#pragma unroll
        for (int j = 0; j < kSplitRows; j++) {
            const unsigned long long i = first + threadIdx.x + (unsigned long long)j * kThreads;
            if (i >= end) continue;
            const long long key = (long long)((unsigned long long)rec[j][0].x | (unsigned long long)rec[j][0].y << 32);
            const int p2 = part_of(pp, key) & (f2 - 1);
            rank[j] = (unsigned)p2 << 24 | atomicAdd(&hist[p2], 1u);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < f2; i += blockDim.x)
            if (hist[i]) base2[i] = atomicAdd(&cursor2[(long long)p1 * f2 + i], (unsigned long long)hist[i]);
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kSplitRows; j++) {
            if (rank[j] == 0xFFFFFFFFu) continue;
            const unsigned long long pos = base2[rank[j] >> 24] + (rank[j] & 0xFFFFFFu);
#pragma unroll
            for (int u = 0; u < UNITS; u++) pp.recs2[pos * UNITS + u] = rec[j][u];
        }
    }
}

// A record's input word for stored column c, and its validity bits.
template <int UNITS>
__device__ __forceinline__ long long rec_raw(const uint4* rec, int c) {
    if (UNITS == 1) return (long long)(int)rec[0].z;  // one Int32 column
    unsigned long long w = 0;
#pragma unroll
    for (int u = 0; u < UNITS; u++) {
        const unsigned long long lo = (unsigned long long)rec[u].x | (unsigned long long)rec[u].y << 32;
        const unsigned long long hi = (unsigned long long)rec[u].z | (unsigned long long)rec[u].w << 32;
        if (2 * u == 1 + c) w = lo;
        if (2 * u + 1 == 1 + c) w = hi;
    }
    return (long long)w;
}

template <int UNITS>
__device__ __forceinline__ unsigned rec_flags(const PartPlan& pp, const uint4* rec) {
    return UNITS == 1 ? rec[0].w : (unsigned)rec_raw<UNITS>(rec, pp.ncols);
}

// A fold record whose key found no shared slot, into the HBM table (out of
// line: the common path keeps only its own code in the instruction cache).
template <int MAXACC, int UNITS>
__device__ __noinline__ void part_rec_to_hbm(const AggProgram& P, const PartPlan& pp, uint4 u0, uint4 u1, uint4 u2) {
    const uint4 rec[3] = {u0, u1, u2};
    const long long key = (long long)((unsigned long long)rec[0].x | (unsigned long long)rec[0].y << 32);
    const unsigned flags = rec_flags<UNITS>(pp, rec);
    unsigned long long val[MAXACC];
    double comp[MAXACC];
#pragma unroll
    for (int q = 0; q < MAXACC; q++) {
        val[q] = 0;
        comp[q] = 0.0;
        if (q >= P.nacc) continue;
        const int c = pp.col_of_acc[q];
        val[q] = contribution_raw(P.acc[q].kind, P.acc[q].in_type, (flags >> c) & 1u, rec_raw<UNITS>(rec, c));
    }
    const long long g = global_slot(P, true, key);
    if (g >= 0) apply_vals<MAXACC>(P, P.arr, P.stride, g, 1, val, comp);
}

// The fold's accumulator operations (kind and input type together).
enum : unsigned {
    kFoldCount = 0, kFoldSumInt, kFoldSumF64, kFoldSumF64Int, kFoldMin32, kFoldMax32, kFoldMin64, kFoldMax64,
    kFoldMinF, kFoldMaxF
};

// Fold: one final partition at a time (records offs[p * fstride] ..
// offs[(p + 1) * fstride] of recs2) in a shared table of its keys.  Each
// thread loads kFoldRows records at once, then folds them one at a time from
// a register queue: one copy of the row code, which keeps it in the
// instruction cache (an unrolled copy per record and per accumulator kind
// stalled the warps on instruction fetch).  Keys that find no shared slot
// fold into HBM directly.
template <int MAXACC, int UNITS>
__global__ void __launch_bounds__(kThreads) part_fold_kernel(const __grid_constant__ AggProgram P,
                                                             const __grid_constant__ PartPlan pp,
                                                             const unsigned long long* __restrict__ offs) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int S = kPartSlots;
    long long* keys = (long long*)smem;
    unsigned int* rows = (unsigned int*)(keys + S);
    unsigned long long* tab = (unsigned long long*)(rows + S) - S;  // array a at tab + a * S
    __shared__ int fill;
    // MIN/MAX of an Int32 column: 32-bit shared atomics on the low word
    // (64-bit shared MIN/MAX/ADD are not single instructions).  A group's
    // value is only emitted when it has a non-NULL input, so the 32-bit
    // identity never reaches a result.
    unsigned narrow = 0;
    for (int q = 0; q < P.nacc; q++)
        if (P.acc[q].in_type == kInt32 && (P.acc[q].kind == kAccMin || P.acc[q].kind == kAccMax))
            narrow |= 1u << P.acc[q].arr;
    // The accumulator program as one word per accumulator: operation (kind
    // and input type together), stored column, array.  Every operation skips
    // a NULL input.
    __shared__ unsigned ops[kMaxAccs];
    if (threadIdx.x < P.nacc) {
        const DevAcc& a = P.acc[threadIdx.x];
        unsigned op;
        switch (a.kind) {
            case kAccCount: op = kFoldCount; break;
            case kAccSumInt: op = kFoldSumInt; break;
            case kAccSumF64: op = a.in_type == kFloat64 ? kFoldSumF64 : kFoldSumF64Int; break;
            case kAccMin: op = a.in_type == kInt32 ? kFoldMin32 : (a.in_type == kFloat64 ? kFoldMinF : kFoldMin64); break;
            default: op = a.in_type == kInt32 ? kFoldMax32 : (a.in_type == kFloat64 ? kFoldMaxF : kFoldMax64); break;
        }
        ops[threadIdx.x] = op | (unsigned)pp.col_of_acc[threadIdx.x] << 4 | (unsigned)a.arr << 8;
    }
    for (int part = blockIdx.x; part < pp.nparts; part += gridDim.x) {
        for (int i = threadIdx.x; i < S; i += blockDim.x) {
            keys[i] = kEmptyKey;
            rows[i] = 0;
        }
        for (int i = threadIdx.x; i < S * (P.narrays - 1); i += blockDim.x) {
            const int a = 1 + i / S;
            tab[S + i] = (narrow >> a) & 1u ? (P.init[a] == kInitMax ? 0x7fffffffull : 0x80000000ull)
                                            : init_value(P.init[a]);
        }
        if (threadIdx.x == 0) fill = 0;
        __syncthreads();
        const unsigned long long lo = offs[(long long)part * pp.fstride], hi = offs[(long long)(part + 1) * pp.fstride];
        for (unsigned long long b0 = lo + threadIdx.x; b0 < hi; b0 += (unsigned long long)kThreads * kFoldRows) {
            uint4 rec[kFoldRows][UNITS];
#pragma unroll
            for (int j = 0; j < kFoldRows; j++) {
                const unsigned long long i = b0 + (unsigned long long)j * kThreads;
                if (i < hi) {
#pragma unroll
                    for (int u = 0; u < UNITS; u++) rec[j][u] = __ldcs(pp.recs2 + i * UNITS + u);
                }
            }
            const int nrec = (int)min((unsigned long long)kFoldRows, (hi - b0 + kThreads - 1) / kThreads);
#pragma unroll 1
            for (int j = 0; j < nrec; j++) {
                const uint4* r0 = rec[0];
                const long long key = (long long)((unsigned long long)r0[0].x | (unsigned long long)r0[0].y << 32);
                const unsigned flags = rec_flags<UNITS>(pp, r0);
                // This partition's shared slot of the key; HBM when there is none.
                int slot = -1;
                unsigned int h = (unsigned int)(fmix64((unsigned long long)key) & (unsigned)(S - 1));
                for (int q = 0; q < 64; q++) {
                    const long long k = ((volatile long long*)keys)[h];
                    if (k == key) {
                        slot = (int)h;
                        break;
                    }
                    if (k == kEmptyKey) {
                        if (*(volatile int*)&fill >= S * 3 / 4) break;
                        const unsigned long long old = atomicCAS((unsigned long long*)&keys[h],
                                                                 (unsigned long long)kEmptyKey, (unsigned long long)key);
                        if (old == (unsigned long long)kEmptyKey) {
                            atomicAdd(&fill, 1);
                            slot = (int)h;
                            break;
                        }
                        if ((long long)old == key) {
                            slot = (int)h;
                            break;
                        }
                    }
                    h = (h + 1u) & (unsigned)(S - 1);
                }
                if (slot < 0) {
                    part_rec_to_hbm<MAXACC, UNITS>(P, pp, r0[0], UNITS > 1 ? r0[UNITS > 1 ? 1 : 0] : r0[0],
                                                   UNITS > 2 ? r0[UNITS > 2 ? 2 : 0] : r0[0]);
                } else {
                    atomicAdd(&rows[slot], 1u);
#pragma unroll 1
                    for (int q = 0; q < P.nacc; q++) {
                        const unsigned o = ops[q];
                        const int c = (o >> 4) & 15;
                        if (!((flags >> c) & 1u)) continue;
                        const long long raw = rec_raw<UNITS>(r0, c);
                        unsigned long long* p = tab + (o >> 8) * S + slot;
                        unsigned* w32 = (unsigned*)p;  // little-endian: [0] the low word
                        switch (o & 15) {
                            case kFoldCount:  // at most 2^32 rows a partition
                                atomicAdd(w32, 1u);
                                break;
                            case kFoldSumInt: {
                                // 64-bit wrapping add as a 32-bit add and its carry
                                const unsigned vlo = (unsigned)raw, vhi = (unsigned)((unsigned long long)raw >> 32);
                                const unsigned old = vlo ? atomicAdd(w32, vlo) : 0u;
                                const unsigned up = vhi + (old + vlo < old ? 1u : 0u);
                                if (up) atomicAdd(w32 + 1, up);
                                break;
                            }
                            case kFoldSumF64:
                            case kFoldSumF64Int: {
                                const double x = (o & 15) == kFoldSumF64 ? __longlong_as_double(raw) : (double)raw;
                                const double old = atomicAdd((double*)p, x);
                                double cc = 0.0;
                                two_sum_into(old, x, &cc);
                                if (cc != 0.0) atomicAdd((double*)(p + S), cc);
                                break;
                            }
                            case kFoldMin32: atomicMin((int*)w32, (int)raw); break;
                            case kFoldMax32: atomicMax((int*)w32, (int)raw); break;
                            case kFoldMin64: atomicMin((long long*)p, raw); break;
                            case kFoldMax64: atomicMax((long long*)p, raw); break;
                            case kFoldMinF: atomicMin((long long*)p, total_order_key(__longlong_as_double(raw))); break;
                            default: atomicMax((long long*)p, total_order_key(__longlong_as_double(raw))); break;
                        }
                    }
                }
                // the next record to the front of the queue
#pragma unroll
                for (int t = 0; t + 1 < kFoldRows; t++)
#pragma unroll
                    for (int u = 0; u < UNITS; u++) rec[t][u] = rec[t + 1][u];
            }
        }
        __syncthreads();
        fused_flush(P, rows, tab, S, keys, narrow);
        __syncthreads();
    }
}

// The fold for 16-byte records (one Int32 column) whose accumulators are
// among COUNT, SUM, MIN and MAX of that column: the program fixed at compile
// time (OPS: bit 0 COUNT, 1 SUM, 2 MIN, 3 MAX), kFoldRows records a thread
// loaded together and folded straight from their registers, no interpreter.
// part_fold_kernel folds every other shape.
struct CompactOps {
    int count_arr, sum_arr, min_arr, max_arr;
};

template <int OPS>
__global__ void __launch_bounds__(kThreads) part_fold_compact_kernel(const __grid_constant__ AggProgram P,
                                                                     const __grid_constant__ PartPlan pp,
                                                                     const __grid_constant__ CompactOps ops,
                                                                     const unsigned long long* __restrict__ offs) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int S = kPartSlots;
    long long* keys = (long long*)smem;
    unsigned int* rows = (unsigned int*)(keys + S);
    unsigned long long* tab = (unsigned long long*)(rows + S) - S;  // array a at tab + a * S
    __shared__ int fill;
    unsigned narrow = 0;  // MIN/MAX of the Int32 column live in their arrays' low words
    if (OPS & 4) narrow |= 1u << ops.min_arr;
    if (OPS & 8) narrow |= 1u << ops.max_arr;
    for (int part = blockIdx.x; part < pp.nparts; part += gridDim.x) {
        for (int i = threadIdx.x; i < S; i += blockDim.x) {
            keys[i] = kEmptyKey;
            rows[i] = 0;
        }
        for (int i = threadIdx.x; i < S * (P.narrays - 1); i += blockDim.x) {
            const int a = 1 + i / S;
            tab[S + i] = (narrow >> a) & 1u ? (P.init[a] == kInitMax ? 0x7fffffffull : 0x80000000ull)
                                            : init_value(P.init[a]);
        }
        if (threadIdx.x == 0) fill = 0;
        __syncthreads();
        const unsigned long long lo = offs[(long long)part * pp.fstride], hi = offs[(long long)(part + 1) * pp.fstride];
        for (unsigned long long b0 = lo + threadIdx.x; b0 < hi; b0 += (unsigned long long)kThreads * kFoldRows) {
            uint4 rec[kFoldRows];
#pragma unroll
            for (int j = 0; j < kFoldRows; j++) {
                const unsigned long long i = b0 + (unsigned long long)j * kThreads;
                rec[j] = i < hi ? __ldcs(pp.recs2 + i) : make_uint4(0, 0, 0, 0);
            }
#pragma unroll
            for (int j = 0; j < kFoldRows; j++) {
                if (b0 + (unsigned long long)j * kThreads >= hi) break;
                const long long key = (long long)((unsigned long long)rec[j].x | (unsigned long long)rec[j].y << 32);
                int slot = -1;
                // the slot: multiply-shift (Fibonacci) hashing of the key, the
                // top log2(S) bits of key * 2^64 / phi
                unsigned int h = (unsigned int)(((unsigned long long)key * 0x9E3779B97F4A7C15ull) >> (64 - kPartSlotBits));
                for (int q = 0; q < 64; q++) {
                    const long long k = ((volatile long long*)keys)[h];
                    if (k == key) {
                        slot = (int)h;
                        break;
                    }
                    if (k == kEmptyKey) {
                        if (*(volatile int*)&fill >= S * 3 / 4) break;
                        const unsigned long long old = atomicCAS((unsigned long long*)&keys[h],
                                                                 (unsigned long long)kEmptyKey, (unsigned long long)key);
                        if (old == (unsigned long long)kEmptyKey) {
                            atomicAdd(&fill, 1);
                            slot = (int)h;
                            break;
                        }
                        if ((long long)old == key) {
                            slot = (int)h;
                            break;
                        }
                    }
                    h = (h + 1u) & (unsigned)(S - 1);
                }
                if (slot < 0) {
                    part_rec_to_hbm<4, 1>(P, pp, rec[j], rec[j], rec[j]);
                    continue;
                }
                atomicAdd(&rows[slot], 1u);
                if (!(rec[j].w & 1u)) continue;  // a NULL value: the row counts, nothing else
                const int x = (int)rec[j].z;
                if (OPS & 1) atomicAdd((unsigned*)(tab + ops.count_arr * S + slot), 1u);
                if (OPS & 2) {
                    // the Int64 sum as a 32-bit add and its carry (x sign-extended)
                    unsigned* w32 = (unsigned*)(tab + ops.sum_arr * S + slot);
                    const unsigned vlo = (unsigned)x, vhi = x < 0 ? 0xffffffffu : 0u;
                    const unsigned old = vlo ? atomicAdd(w32, vlo) : 0u;
                    const unsigned up = vhi + (old + vlo < old ? 1u : 0u);
                    if (up) atomicAdd(w32 + 1, up);
                }
                if (OPS & 4) atomicMin((int*)(tab + ops.min_arr * S + slot), x);
                if (OPS & 8) atomicMax((int*)(tab + ops.max_arr * S + slot), x);
            }
        }
        __syncthreads();
        fused_flush(P, rows, tab, S, keys, narrow);
        __syncthreads();
    }
}

using CompactFold = void (*)(const AggProgram, const PartPlan, const CompactOps, const unsigned long long*);
CompactFold compact_fold_for(int ops) {
    switch (ops) {
#define OXB_CF(m) \
    case m: return part_fold_compact_kernel<m>;
        OXB_CF(1) OXB_CF(2) OXB_CF(3) OXB_CF(4) OXB_CF(5) OXB_CF(6) OXB_CF(7) OXB_CF(8) OXB_CF(9) OXB_CF(10)
        OXB_CF(11) OXB_CF(12) OXB_CF(13) OXB_CF(14) OXB_CF(15)
#undef OXB_CF
        default: return nullptr;
    }
}

// The compact fold's program for P (records of one Int32 column), or 0 when
// an accumulator is outside it.
int compact_ops_of(const AggProgram& P, CompactOps* ops) {
    int m = 0;
    *ops = CompactOps{0, 0, 0, 0};
    for (int q = 0; q < P.nacc; q++) {
        const DevAcc& a = P.acc[q];
        if (a.in_type != kInt32) return 0;
        int bit;
        switch (a.kind) {
            case kAccCount: bit = 1; ops->count_arr = a.arr; break;
            case kAccSumInt: bit = 2; ops->sum_arr = a.arr; break;
            case kAccMin: bit = 4; ops->min_arr = a.arr; break;
            case kAccMax: bit = 8; ops->max_arr = a.arr; break;
            default: return 0;
        }
        if (m & bit) return 0;
        m |= bit;
    }
    return m;
}

// ---- dense key ranges ----------------------------------------------------
// When the kept keys fill a range of at most kDenseMaxParts * kDenseKeys
// values (a sampled estimate, then checked row by row by the count pass),
// the partitioned fold needs no hash at all: a key's partition is its offset
// from the range's low end divided by kDenseKeys, and its slot in the fold's
// shared table the remainder.  Records shrink to 8 bytes (the Int32 value;
// the offset shifted left once, with the value's validity in bit 0).  The
// count pass keeps one histogram per CTA, so every CTA of the split owns a
// known slice of every partition and reserves nothing with global atomics
// (which reach only about 80 G/s on random addresses on the B200).  The
// groups leave the fold compacted and already in key order, so the emit
// needs no sort.

constexpr int kDenseBits = 13;
constexpr int kDenseKeys = 1 << kDenseBits;  // keys a partition: the fold's shared table
constexpr int kDenseMaxParts = 4096;        // so a range of at most 2^25 keys
constexpr int kDenseThreads = 256;          // the count and split passes
constexpr int kDenseCtas = 4;               // their CTAs an SM (64 registers a thread)
constexpr int kDenseRows = 8;               // rows a thread in a split sub-tile
constexpr int kDenseSub = kDenseThreads * kDenseRows;
constexpr int kDenseFoldThreads = 1024;
constexpr int kDenseSamples = 16384;
constexpr int kDenseFanBits = 4;  // final partitions a first-level partition
constexpr int kDenseFan = 1 << kDenseFanBits;
constexpr int kDenseChunk = 2048;  // records a chunk of the second split
constexpr unsigned long long kSignBit = 0x8000000000000000ull;
static_assert(kDenseSub <= 65536 && kDenseMaxParts <= 65536, "ranks and partitions pack into 16 bits each");

struct DensePlan {
    unsigned long long lo;    // the range's low end as an ordered key (key ^ sign bit)
    unsigned long long span;  // keys in the range: np * kDenseKeys
    int np;                   // final partitions (the fold's)
    int np1;                  // first-level partitions: kDenseFan final partitions each
    int grid;                 // CTAs of the count and first split passes (the same tile ranges)
    int q;                    // the accumulator whose Int32 column the records carry
    unsigned int* counts1;    // [np1][grid]: kept rows a first-level partition and CTA
    unsigned int* totals;     // [np]: kept rows a final partition
    const unsigned long long* offs1;  // exclusive scan of counts1, [np1 * grid + 1]
    const unsigned long long* offs;   // exclusive scan of totals, [np + 1]
    uint2* recs1;             // records by first-level partition: the value, offset << 1 | validity
    uint2* recs;              // the same records by final partition
    unsigned long long nrecs;
    unsigned int* status;
};

// The columns a dense pass reads for partitioning tile t of batch B (the
// key, every WHERE column and, when q >= 0, accumulator q's Int32 column),
// prefetched into L2 while the CTA works on the tile before it.
__device__ __forceinline__ void prefetch_tile(const DevPredicate& pred, const BatchCols& B, int key_type, long long t,
                                              int q) {
    const long long base = (t - B.ptile0) * kPartTile;
    const long long n = B.n - base < kPartTile ? B.n - base : kPartTile;
    if (n <= 0) return;
    const int kw = type_width(key_type, 1);
    prefetch_l2_range((const char*)B.key + base * kw, (unsigned long long)(n * kw));
    for (int l = 0; l < pred.nleaves; l++) {
        const int w = type_width(pred.leaves[l].type, 1);
        prefetch_l2_range((const char*)B.lvals[l] + base * w, (unsigned long long)(n * w));
    }
    if (q >= 0) prefetch_l2_range((const char*)B.vals[q] + base * 4, (unsigned long long)(n * 4));
}

// Thread 0 prefetches tile t + 1 of the CTA's range [.., t1) (bi: tile t's batch).
__device__ __forceinline__ void prefetch_next_tile(const DevPredicate& pred, const BatchCols* batches, int nb, int bi,
                                                   int key_type, long long t, long long t1, int q) {
    if (threadIdx.x != 0 || t + 1 >= t1) return;
    while (bi + 1 < nb && batches[bi + 1].ptile0 <= t + 1) bi++;
    prefetch_tile(pred, batches[bi], key_type, t + 1, q);
}

// A strided sample of the rows, spread over the partitioning tiles.
// out[0] rows sampled, [1] rows the WHERE keeps, [2] and [3] the least and
// greatest ordered key (key ^ sign bit) of the kept rows with a valid key.
__global__ void part_dense_sample_kernel(const __grid_constant__ DevPredicate pred, int key_type,
                                         const BatchCols* __restrict__ batches, int nb, long long ntiles, int samples,
                                         unsigned long long* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < samples;
    bool kept = false, kv = false;
    unsigned long long ok = 0;
    if (live) {
        const long long t = (long long)i * ntiles / samples;
        const BatchCols& B = batches[batch_of_tile(batches, nb, t)];
        const long long base = (t - B.ptile0) * kPartTile;
        const long long rows = B.n - base < kPartTile ? B.n - base : kPartTile;
        const long long r = base + (long long)(fmix64((unsigned long long)i + 1u) % (unsigned long long)rows);
        long long key[1];
        unsigned nk;
        const unsigned m = kept_keys<1, 1>(pred, B, key_type, r, r + 1, key, &nk);
        kept = ((m | nk) & 1u) != 0;
        kv = (m & 1u) != 0;
        ok = (unsigned long long)key[0] ^ kSignBit;
    }
    unsigned long long lo = kv ? ok : ~0ull, hi = kv ? ok : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long a = __shfl_xor_sync(0xffffffffu, lo, o), c = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = a < lo ? a : lo;
        hi = c > hi ? c : hi;
    }
    const unsigned nlive = __popc(__ballot_sync(0xffffffffu, live)), nkept = __popc(__ballot_sync(0xffffffffu, kept));
    const bool any = __ballot_sync(0xffffffffu, kv) != 0;
    if ((threadIdx.x & 31) == 0) {
        if (nlive) atomicAdd(&out[0], (unsigned long long)nlive);
        if (nkept) atomicAdd(&out[1], (unsigned long long)nkept);
        if (any) {
            atomicMin(&out[2], lo);
            atomicMax(&out[3], hi);
        }
    }
}

// The end of a count pass: the CTA's kept rows per first-level partition
// (its slice of each), and its share of every final partition's total.
__device__ __forceinline__ void dense_count_store(const DensePlan& dp, const unsigned* dhist) {
    for (int k = threadIdx.x; k < dp.np1; k += blockDim.x) {
        unsigned n = 0;
        for (int p = k << kDenseFanBits; p < ((k + 1) << kDenseFanBits) && p < dp.np; p++) n += dhist[p];
        dp.counts1[(long long)k * gridDim.x + blockIdx.x] = n;
    }
    for (int p = threadIdx.x; p < dp.np; p += blockDim.x)
        if (dhist[p]) atomicAdd(&dp.totals[p], dhist[p]);
}

// The count pass, over a contiguous range of tiles a CTA (the first split
// takes the same ranges): the kept rows with a valid key in each partition
// (dense_count_store).  out[0] gets their number, out[1] the number of
// kept rows whose key falls outside the range (the host then takes the
// hashed passes instead).
__global__ void __launch_bounds__(kDenseThreads, kDenseCtas) part_dense_count_kernel(const __grid_constant__ DevPredicate pred,
                                                                         int key_type,
                                                                         const BatchCols* __restrict__ batches, int nb,
                                                                         long long ntiles,
                                                                         const __grid_constant__ DensePlan dp,
                                                                         unsigned long long* __restrict__ out) {
    extern __shared__ unsigned int dhist[];
    for (int i = threadIdx.x; i < dp.np; i += blockDim.x) dhist[i] = 0;
    __syncthreads();
    unsigned n = 0, outside = 0;
    const long long t0 = ntiles * blockIdx.x / gridDim.x, t1 = ntiles * (blockIdx.x + 1) / gridDim.x;
    int bi = t0 < t1 ? batch_of_tile(batches, nb, t0) : 0;
    for (long long t = t0; t < t1; t++) {
        while (bi + 1 < nb && batches[bi + 1].ptile0 <= t) bi++;
        const BatchCols& B = batches[bi];
        if (t == t0 && threadIdx.x == 0) prefetch_tile(pred, B, key_type, t, -1);
        prefetch_next_tile(pred, batches, nb, bi, key_type, t, t1, -1);
        const long long base = (t - B.ptile0) * kPartTile;
        const long long end = base + kPartTile < B.n ? base + kPartTile : B.n;
        for (long long sub = base; sub < end; sub += kDenseSub) {
            long long key[kDenseRows];
            unsigned nk;
            const unsigned m = kept_keys_eager<kDenseRows, kDenseThreads, false>(pred, B, key_type, sub + threadIdx.x,
                                                                                end, key, &nk, 0, nullptr, nullptr);
#pragma unroll
            for (int j = 0; j < kDenseRows; j++) {
                if (!((m >> j) & 1u)) continue;
                const unsigned long long rel = ((unsigned long long)key[j] ^ kSignBit) - dp.lo;
                if (rel < dp.span) {
                    atomicAdd(&dhist[rel >> kDenseBits], 1u);
                    n++;
                } else {
                    outside++;
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n += __shfl_xor_sync(0xffffffffu, n, o);
        outside += __shfl_xor_sync(0xffffffffu, outside, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (n) atomicAdd(&out[0], (unsigned long long)n);
        if (outside) atomicAdd(&out[1], (unsigned long long)outside);
    }
    __syncthreads();
    dense_count_store(dp, dhist);
}

// Exclusive scan of in[0, n) into out[0, n) by the whole block (a multiple
// of 32 threads, at most 1024); *total gets the sum.  Ends synchronised.
__device__ void block_exclusive_scan(const unsigned* in, unsigned* out, int n, unsigned* wsum, unsigned* total) {
    const int per = (n + (int)blockDim.x - 1) / (int)blockDim.x;
    const int b0 = threadIdx.x * per;
    unsigned s = 0;
    for (int i = 0; i < per; i++)
        if (b0 + i < n) s += in[b0 + i];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned inc = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    if (w == 0) {
        const int nw = (int)blockDim.x >> 5;
        const unsigned v = lane < nw ? wsum[lane] : 0u;
        unsigned vi = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, vi, o);
            if (lane >= o) vi += y;
        }
        if (lane < nw) wsum[lane] = vi - v;
        if (lane == 31) *total = vi;
    }
    __syncthreads();
    unsigned run = wsum[w] + inc - s;
    for (int i = 0; i < per; i++)
        if (b0 + i < n) {
            out[b0 + i] = run;
            run += in[b0 + i];
        }
    __syncthreads();
}

// A sub-tile's records staged in shared memory, ordered by first-level
// partition, so that each partition's run reaches HBM as whole 32-byte
// sectors: a sector written in part is first filled from DRAM by L2, which
// (measured) doubled the split's DRAM reads when each row was stored alone.
struct DenseStage {
    uint2* rec;             // kDenseSub records, by partition
    unsigned* cursor;       // np1: the CTA's next record in each first-level partition
    unsigned* hist;         // np1: the sub-tile's records a partition
    unsigned* start;        // np1: their exclusive scan
    unsigned short* part;   // kDenseSub: each ordered record's partition
};

size_t dense_split_smem(int np1) { return (size_t)kDenseSub * (8 + 2) + (size_t)np1 * 12; }

__device__ __forceinline__ DenseStage dense_stage(unsigned char* smem, int np1) {
    DenseStage st;
    st.rec = (uint2*)smem;
    st.cursor = (unsigned*)(st.rec + kDenseSub);
    st.hist = st.cursor + np1;
    st.start = st.hist + np1;
    st.part = (unsigned short*)(st.start + np1);
    return st;
}

// After the records are ordered (and a barrier): each partition's run to
// the CTA's cursor into it, consecutive threads on consecutive records; then
// the cursors advance and the counts clear.  Ends synchronised.
__device__ __forceinline__ void dense_stage_store(const DenseStage& st, const DensePlan& dp, unsigned total) {
    for (unsigned sidx = threadIdx.x; sidx < total; sidx += blockDim.x) {
        const unsigned k = st.part[sidx];
        const unsigned long long pos = (unsigned long long)st.cursor[k] + (sidx - st.start[k]);
        if (pos < dp.nrecs) dp.recs1[pos] = st.rec[sidx];
        else atomicOr(dp.status, kStatusBounds);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < dp.np1; k += blockDim.x) {
        st.cursor[k] += st.hist[k];
        st.hist[k] = 0;
    }
    __syncthreads();
}

// The first split, over the count pass's tile ranges: each sub-tile of
// kDenseSub rows ranks its kept rows per first-level partition (kDenseFan
// final partitions each) in shared memory, orders their records there, and
// stores each partition's run at the CTA's own cursor into it (the CTA's
// slice, from the count pass).  Kept rows whose key is NULL or INT64_MIN
// fold straight into their HBM slots.
template <int MAXACC>
__global__ void __launch_bounds__(kDenseThreads, kDenseCtas) part_dense_split_kernel(const __grid_constant__ AggProgram P,
                                                                            const __grid_constant__ DevPredicate pred,
                                                                            int key_type,
                                                                            const BatchCols* __restrict__ batches,
                                                                            int nb, long long ntiles,
                                                                            const __grid_constant__ DensePlan dp) {
    extern __shared__ __align__(16) unsigned char dsm[];
    DenseStage st = dense_stage(dsm, dp.np1);
    __shared__ unsigned wsum[kDenseThreads / 32];
    __shared__ unsigned s_total;
    for (int k = threadIdx.x; k < dp.np1; k += blockDim.x) {
        st.cursor[k] = (unsigned)dp.offs1[(long long)k * gridDim.x + blockIdx.x];
        st.hist[k] = 0;
    }
    __syncthreads();
    const long long t0 = ntiles * blockIdx.x / gridDim.x, t1 = ntiles * (blockIdx.x + 1) / gridDim.x;
    int bi = t0 < t1 ? batch_of_tile(batches, nb, t0) : 0;
    for (long long t = t0; t < t1; t++) {
        while (bi + 1 < nb && batches[bi + 1].ptile0 <= t) bi++;
        const BatchCols& B = batches[bi];
        if (t == t0 && threadIdx.x == 0) prefetch_tile(pred, B, key_type, t, dp.q);
        prefetch_next_tile(pred, batches, nb, bi, key_type, t, t1, dp.q);
        const long long base = (t - B.ptile0) * kPartTile;
        const long long end = base + kPartTile < B.n ? base + kPartTile : B.n;
        for (long long sub = base; sub < end; sub += kDenseSub) {
            long long key[kDenseRows];
            int xv[kDenseRows];
            unsigned nk, xvalid = 0;
            unsigned m = kept_keys_eager<kDenseRows, kDenseThreads, true>(pred, B, key_type, sub + threadIdx.x, end, key,
                                                                          &nk, dp.q, xv, &xvalid);
            unsigned rel[kDenseRows], pr[kDenseRows];
#pragma unroll
            for (int j = 0; j < kDenseRows; j++) {
                pr[j] = 0;
                const unsigned long long r64 = ((unsigned long long)key[j] ^ kSignBit) - dp.lo;
                rel[j] = (unsigned)r64;
                if (!((m >> j) & 1u)) continue;
                if (r64 >= dp.span) {  // the count pass found none; never written out of range
                    atomicOr(dp.status, kStatusBounds);
                    m &= ~(1u << j);
                    continue;
                }
                const unsigned k = rel[j] >> (kDenseBits + kDenseFanBits);
                pr[j] = k << 16 | atomicAdd(&st.hist[k], 1u);
            }
#pragma unroll
            for (int j = 0; j < kDenseRows; j++)
                if ((nk >> j) & 1u) part_null_row_to_hbm<MAXACC>(P, B, sub + threadIdx.x + (long long)j * kDenseThreads);
            __syncthreads();
            block_exclusive_scan(st.hist, st.start, dp.np1, wsum, &s_total);
#pragma unroll
            for (int j = 0; j < kDenseRows; j++) {
                if (!((m >> j) & 1u)) continue;
                const unsigned k = pr[j] >> 16;
                const unsigned sidx = st.start[k] + (pr[j] & 0xFFFFu);
                st.rec[sidx] = make_uint2((unsigned)xv[j], rel[j] << 1 | ((xvalid >> j) & 1u));
                st.part[sidx] = (unsigned short)k;
            }
            __syncthreads();
            dense_stage_store(st, dp, s_total);
        }
    }
}

// The compiled form of the dense count and split passes, for the common
// shape: no validity bitmap on the key or the WHERE columns, at most two
// WHERE leaves, and every column of every batch starting on a 16-byte
// boundary.  A thread takes four consecutive rows a load (one 128-bit load
// of an Int32 column, two of a 64-bit one), so loads, index arithmetic and
// loop overhead a row shrink fourfold, and each comparison is lean_cmp's
// branch-free mask.  The rows a thread takes are quads g and g + kDenseThreads
// of a sub-tile, so a warp's loads stay contiguous.
struct DenseLean {
    int nleaves;
    int leaf_w8[2];   // the leaf's column is 64-bit (Int64 or Float64)
    int leaf_f64[2];
    int leaf_mask[2];
    long long lit[2];
};

// The 64-bit values of rows 4g .. 4g+3 (below end; the others read 0).
__device__ __forceinline__ void quad_load64(const void* col, long long g, long long end, long long v[4]) {
    const long long r = 4 * g;
    if (r + 4 <= end) {
        const longlong2 a = __ldg((const longlong2*)col + 2 * g), b = __ldg((const longlong2*)col + 2 * g + 1);
        v[0] = a.x;
        v[1] = a.y;
        v[2] = b.x;
        v[3] = b.y;
    } else {
#pragma unroll
        for (int i = 0; i < 4; i++) v[i] = r + i < end ? __ldg((const long long*)col + r + i) : 0;
    }
}

// The Int32 values of rows 4g .. 4g+3 (below end; the others read 0).
__device__ __forceinline__ void quad_load32(const void* col, long long g, long long end, int v[4]) {
    const long long r = 4 * g;
    if (r + 4 <= end) {
        const int4 a = __ldg((const int4*)col + g);
        v[0] = a.x;
        v[1] = a.y;
        v[2] = a.z;
        v[3] = a.w;
    } else {
#pragma unroll
        for (int i = 0; i < 4; i++) v[i] = r + i < end ? __ldg((const int*)col + r + i) : 0;
    }
}

// Rows 4g .. 4g+3 for q in {0, 1}, g = g0 + q * kDenseThreads: their keys
// (key[4q + i]) and a mask (bit 4q + i) of the live rows the WHERE keeps.
// *minkey gets those whose key is INT64_MIN, left out of the mask.
template <bool K8>
__device__ __forceinline__ unsigned lean_rows(const DenseLean& L, const BatchCols& B, long long g0, long long end,
                                              long long key[8], unsigned* minkey) {
    unsigned live = 0;
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const long long r = 4 * (g0 + q * kDenseThreads);
#pragma unroll
        for (int i = 0; i < 4; i++)
            if (r + i < end) live |= 1u << (4 * q + i);
    }
    if (!live) {
        *minkey = 0;
        return 0;
    }
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const long long g = g0 + q * kDenseThreads;
        if (K8) {
            quad_load64(B.key, g, end, key + 4 * q);
        } else {
            int k32[4];
            quad_load32(B.key, g, end, k32);
#pragma unroll
            for (int i = 0; i < 4; i++) key[4 * q + i] = k32[i];
        }
    }
    unsigned keep = live;
#pragma unroll
    for (int l = 0; l < 2; l++) {
        if (l >= L.nleaves) break;
        const void* col = B.lvals[l];
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const long long g = g0 + q * kDenseThreads;
            long long a[4];
            if (L.leaf_w8[l]) {
                quad_load64(col, g, end, a);
                if (L.leaf_f64[l]) {
#pragma unroll
                    for (int i = 0; i < 4; i++) a[i] = filter_order_key(__longlong_as_double(a[i]));
                }
            } else {
                int a32[4];
                quad_load32(col, g, end, a32);
#pragma unroll
                for (int i = 0; i < 4; i++) a[i] = a32[i];
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
                if (!lean_cmp(L.leaf_mask[l], a[i], L.lit[l])) keep &= ~(1u << (4 * q + i));
        }
    }
    unsigned mk = 0;
#pragma unroll
    for (int j = 0; j < 8; j++)
        if (((keep >> j) & 1u) && key[j] == kEmptyKey) mk |= 1u << j;
    *minkey = mk;
    return keep & ~mk;
}

// The count pass, compiled (part_dense_count_kernel's contract).
template <bool K8>
__global__ void __launch_bounds__(kDenseThreads, kDenseCtas) part_dense_count_lean_kernel(const __grid_constant__ DenseLean L,
                                                                              const BatchCols* __restrict__ batches,
                                                                              int nb, long long ntiles,
                                                                              const __grid_constant__ DensePlan dp,
                                                                              unsigned long long* __restrict__ out) {
    extern __shared__ unsigned int dhist[];
    for (int i = threadIdx.x; i < dp.np; i += blockDim.x) dhist[i] = 0;
    __syncthreads();
    unsigned n = 0, outside = 0;
    const long long t0 = ntiles * blockIdx.x / gridDim.x, t1 = ntiles * (blockIdx.x + 1) / gridDim.x;
    int bi = t0 < t1 ? batch_of_tile(batches, nb, t0) : 0;
    for (long long t = t0; t < t1; t++) {
        while (bi + 1 < nb && batches[bi + 1].ptile0 <= t) bi++;
        const BatchCols& B = batches[bi];
        const long long base = (t - B.ptile0) * kPartTile;
        const long long end = base + kPartTile < B.n ? base + kPartTile : B.n;
        for (long long sub = base; sub < end; sub += kDenseSub) {
            long long key[8];
            unsigned mk;
            const unsigned m = lean_rows<K8>(L, B, sub / 4 + threadIdx.x, end, key, &mk);
#pragma unroll
            for (int j = 0; j < 8; j++) {
                if (!((m >> j) & 1u)) continue;
                const unsigned long long rel = ((unsigned long long)key[j] ^ kSignBit) - dp.lo;
                if (rel < dp.span) {
                    atomicAdd(&dhist[rel >> kDenseBits], 1u);
                    n++;
                } else {
                    outside++;
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n += __shfl_xor_sync(0xffffffffu, n, o);
        outside += __shfl_xor_sync(0xffffffffu, outside, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (n) atomicAdd(&out[0], (unsigned long long)n);
        if (outside) atomicAdd(&out[1], (unsigned long long)outside);
    }
    __syncthreads();
    dense_count_store(dp, dhist);
}

// The first split, compiled (part_dense_split_kernel's contract; rows
// whose key is INT64_MIN fold into their HBM slot).
template <int MAXACC, bool K8>
__global__ void __launch_bounds__(kDenseThreads, kDenseCtas) part_dense_split_lean_kernel(
    const __grid_constant__ AggProgram P, const __grid_constant__ DenseLean L, const BatchCols* __restrict__ batches,
    int nb, long long ntiles, const __grid_constant__ DensePlan dp) {
    extern __shared__ __align__(16) unsigned char dsm[];
    DenseStage st = dense_stage(dsm, dp.np1);
    __shared__ unsigned wsum[kDenseThreads / 32];
    __shared__ unsigned s_total;
    for (int k = threadIdx.x; k < dp.np1; k += blockDim.x) {
        st.cursor[k] = (unsigned)dp.offs1[(long long)k * gridDim.x + blockIdx.x];
        st.hist[k] = 0;
    }
    __syncthreads();
    const long long t0 = ntiles * blockIdx.x / gridDim.x, t1 = ntiles * (blockIdx.x + 1) / gridDim.x;
    int bi = t0 < t1 ? batch_of_tile(batches, nb, t0) : 0;
    for (long long t = t0; t < t1; t++) {
        while (bi + 1 < nb && batches[bi + 1].ptile0 <= t) bi++;
        const BatchCols& B = batches[bi];
        const long long base = (t - B.ptile0) * kPartTile;
        const long long end = base + kPartTile < B.n ? base + kPartTile : B.n;
        for (long long sub = base; sub < end; sub += kDenseSub) {
            const long long g0 = sub / 4 + threadIdx.x;
            // the carried values first, so they load with the keys and the WHERE columns
            int xv[8];
            unsigned xvalid = 0xFFu;
            const uint8_t* xbits = B.valid[dp.q];
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const long long g = g0 + q * kDenseThreads;
                quad_load32(B.vals[dp.q], g, end, xv + 4 * q);
                if (xbits && 4 * g < end)
                    xvalid &= ~(0xFu << (4 * q)) | ((unsigned)(__ldg(xbits + ((4 * g) >> 3)) >> ((4 * g) & 7)) & 0xFu)
                                                       << (4 * q);
            }
            unsigned rel[8], mk, m;
            {
                long long key[8];
                m = lean_rows<K8>(L, B, g0, end, key, &mk);
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const unsigned long long r64 = ((unsigned long long)key[j] ^ kSignBit) - dp.lo;
                    rel[j] = (unsigned)r64;
                    if (((m >> j) & 1u) && r64 >= dp.span) {  // the count pass found none; never written out of range
                        atomicOr(dp.status, kStatusBounds);
                        m &= ~(1u << j);
                    }
                }
            }
            unsigned pr[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                pr[j] = 0;
                if (!((m >> j) & 1u)) continue;
                const unsigned k = rel[j] >> (kDenseBits + kDenseFanBits);
                pr[j] = k << 16 | atomicAdd(&st.hist[k], 1u);
                xv[j] = ((xvalid >> j) & 1u) ? xv[j] : 0;
            }
            if (mk) {
#pragma unroll
                for (int j = 0; j < 8; j++)
                    if ((mk >> j) & 1u)
                        part_null_row_to_hbm<MAXACC>(P, B, 4 * (g0 + (j >> 2) * kDenseThreads) + (j & 3));
            }
            __syncthreads();
            block_exclusive_scan(st.hist, st.start, dp.np1, wsum, &s_total);
#pragma unroll
            for (int j = 0; j < 8; j++) {
                if (!((m >> j) & 1u)) continue;
                const unsigned k = pr[j] >> 16;
                const unsigned sidx = st.start[k] + (pr[j] & 0xFFFFu);
                st.rec[sidx] = make_uint2((unsigned)xv[j], rel[j] << 1 | ((xvalid >> j) & 1u));
                st.part[sidx] = (unsigned short)k;
            }
            __syncthreads();
            dense_stage_store(st, dp, s_total);
        }
    }
}

// The first chunk of each first-level partition's records (kDenseChunk a
// chunk) and, at [np1], their total: one block of 256 threads (np1 is at
// most kDenseMaxParts / kDenseFan = 256) and one block scan.
static_assert(kDenseMaxParts / kDenseFan <= 256, "one thread a first-level partition");
__global__ void __launch_bounds__(256) dense_chunks_kernel(const __grid_constant__ DensePlan dp,
                                                           long long* __restrict__ cstart) {
    __shared__ unsigned cnt[256], pre[256], wsum[8], total;
    for (int k = threadIdx.x; k < dp.np1; k += blockDim.x) {
        const unsigned long long n = dp.offs1[(long long)(k + 1) * dp.grid] - dp.offs1[(long long)k * dp.grid];
        cnt[k] = (unsigned)((n + kDenseChunk - 1) / kDenseChunk);
    }
    __syncthreads();
    block_exclusive_scan(cnt, pre, dp.np1, wsum, &total);
    for (int k = threadIdx.x; k < dp.np1; k += blockDim.x) cstart[k] = pre[k];
    if (threadIdx.x == 0) cstart[dp.np1] = total;
}

// Each final partition's next record in the second split: its start.
__global__ void dense_cursor_kernel(const __grid_constant__ DensePlan dp, unsigned int* __restrict__ gcursor) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < dp.np; p += gridDim.x * blockDim.x)
        gcursor[p] = (unsigned)dp.offs[p];
}

// The second split: chunks of one first-level partition's records from a
// queue, each spread over its kDenseFan final partitions.  A record's rank
// among the chunk's records of its final partition comes from a warp-wide
// match and one shared atomic a group; the chunk then reserves each final
// partition's run with one global atomic, and the records are stored from
// shared memory in run order (runs of about kDenseChunk / kDenseFan records,
// whole sectors).
constexpr int kSplit2Rows = kDenseChunk / kDenseThreads;
__global__ void __launch_bounds__(kDenseThreads, kDenseCtas) part_dense_split2_kernel(const __grid_constant__ DensePlan dp,
                                                                          const long long* __restrict__ cstart,
                                                                          unsigned long long* __restrict__ queue,
                                                                          unsigned int* __restrict__ gcursor) {
    __shared__ unsigned hist[kDenseFan], gbase[kDenseFan], start[kDenseFan];
    __shared__ __align__(16) uint2 srec[kDenseChunk];
    __shared__ long long s_c;
    const int lane = threadIdx.x & 31;
    const long long nchunks = cstart[dp.np1];
    for (;;) {
        if (threadIdx.x < kDenseFan) hist[threadIdx.x] = 0;
        if (threadIdx.x == 0) s_c = (long long)atomicAdd(queue, 1ull);
        __syncthreads();
        const long long c = s_c;
        if (c >= nchunks) break;
        int a = 0, b = dp.np1 - 1;  // the first-level partition holding chunk c
        while (a < b) {
            const int mid = (a + b + 1) >> 1;
            if (cstart[mid] <= c) a = mid;
            else b = mid - 1;
        }
        const unsigned long long r0 = dp.offs1[(long long)a * dp.grid] + (unsigned long long)(c - cstart[a]) * kDenseChunk;
        const unsigned long long rend = dp.offs1[(long long)(a + 1) * dp.grid];
        uint2 rec[kSplit2Rows];
        unsigned rank[kSplit2Rows];
#pragma unroll
        for (int j = 0; j < kSplit2Rows; j++) {
            const unsigned long long i = r0 + threadIdx.x + (unsigned long long)j * kDenseThreads;
            rec[j] = i < rend && i < r0 + kDenseChunk ? __ldcs(dp.recs1 + i) : make_uint2(0u, 0xFFFFFFFFu);
        }
#pragma unroll
        for (int j = 0; j < kSplit2Rows; j++) {
            const unsigned long long i = r0 + threadIdx.x + (unsigned long long)j * kDenseThreads;
            const bool live = i < rend && i < r0 + kDenseChunk;
            // a lane without a record matches no other (a tag of its own above the bins)
            const unsigned bin = live ? ((rec[j].y >> (1 + kDenseBits)) & (kDenseFan - 1)) : (unsigned)(kDenseFan + lane);
            const unsigned peers = __match_any_sync(0xffffffffu, bin);
            const int leader = __ffs(peers) - 1;
            unsigned base = 0;
            if (live && lane == leader) base = atomicAdd(&hist[bin], (unsigned)__popc(peers));
            base = __shfl_sync(0xffffffffu, base, leader);
            rank[j] = base + (unsigned)__popc(peers & ((1u << lane) - 1u));
        }
        __syncthreads();
        if (threadIdx.x < 32) {  // the runs' places in shared memory
            const unsigned h = threadIdx.x < kDenseFan ? hist[threadIdx.x] : 0u;
            unsigned inc = h;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += y;
            }
            if (threadIdx.x < kDenseFan) start[threadIdx.x] = inc - h;
        }
        __syncthreads();
        // ... and in HBM: the reservations' round trip overlaps the other
        // warps' ordering of the records
        if (threadIdx.x < kDenseFan && hist[threadIdx.x])
            gbase[threadIdx.x] = atomicAdd(&gcursor[(a << kDenseFanBits) + threadIdx.x], hist[threadIdx.x]);
#pragma unroll
        for (int j = 0; j < kSplit2Rows; j++) {
            const unsigned long long i = r0 + threadIdx.x + (unsigned long long)j * kDenseThreads;
            if (!(i < rend && i < r0 + kDenseChunk)) continue;
            const unsigned bin = (rec[j].y >> (1 + kDenseBits)) & (kDenseFan - 1);
            srec[start[bin] + rank[j]] = rec[j];
        }
        __syncthreads();
        // consecutive threads store consecutive records of a run: whole sectors
        const unsigned n = (unsigned)((rend < r0 + kDenseChunk ? rend : r0 + kDenseChunk) - r0);
        for (unsigned sidx = threadIdx.x; sidx < n; sidx += blockDim.x) {
            const uint2 r = srec[sidx];
            const unsigned bin = (r.y >> (1 + kDenseBits)) & (kDenseFan - 1);
            const unsigned long long pos = (unsigned long long)gbase[bin] + (sidx - start[bin]);
            if (pos < dp.nrecs) dp.recs[pos] = r;
            else atomicOr(dp.status, kStatusBounds);
        }
        __syncthreads();
    }
}

// Slots [capacity] (the NULL group) and [capacity + 1] (the key INT64_MIN)
// of every array: the only HBM slots the dense path folds into with atomics.
__global__ void dense_special_init_kernel(const __grid_constant__ AggProgram P) {
    for (int a = threadIdx.x; a < P.narrays; a += blockDim.x) {
        P.arr[(long long)a * P.stride + P.capacity] = init_value(P.init[a]);
        P.arr[(long long)a * P.stride + P.capacity + 1] = init_value(P.init[a]);
    }
}

size_t dense_fold_smem(int ops) {
    int arrays = 2 + ((ops & 2) ? 2 : 0) + ((ops & 4) ? 1 : 0) + ((ops & 8) ? 1 : 0);
    return (size_t)arrays * kDenseKeys * 4;
}

// The fold, one partition a CTA at a time, into a shared table indexed by
// the key's offset: 32-bit shared atomics only (the rows with a NULL value
// or else the rows with a value, which is COUNT; the Int64 SUM as a 32-bit
// add and its carry; MIN and MAX, each only after a plain read shows the
// value would change it), so one counting atomic a record.  The
// partition's groups then go to the HBM table compacted and in key order,
// at the partition's own slots [p * kDenseKeys, ...), and their number to
// gcount[p].  OPS: bit 0 COUNT, 1 SUM, 2 MIN, 3 MAX (CompactOps).
template <int OPS>
__global__ void __launch_bounds__(kDenseFoldThreads, 1) part_dense_fold_kernel(const __grid_constant__ AggProgram P,
                                                                               const __grid_constant__ DensePlan dp,
                                                                               const __grid_constant__ CompactOps ops,
                                                                               unsigned int* __restrict__ gcount) {
    extern __shared__ __align__(16) unsigned int fsm[];
    unsigned* nul = fsm;                // rows whose value is NULL
    unsigned* cnt = nul + kDenseKeys;   // rows whose value is not: a group's rows are their sum
    unsigned* slo = cnt + kDenseKeys;
    unsigned* shi = slo + ((OPS & 2) ? kDenseKeys : 0);
    int* mn = (int*)(shi + ((OPS & 2) ? kDenseKeys : 0));
    int* mx = mn + ((OPS & 4) ? kDenseKeys : 0);
    __shared__ unsigned wsum[32];
    __shared__ unsigned s_total;
    constexpr int kPer = kDenseKeys / kDenseFoldThreads;  // slots a thread in the flush
    constexpr int kInFlight = 4;                            // record pairs a thread loads together
    const long long st = P.stride;
    for (int part = blockIdx.x; part < dp.np; part += gridDim.x) {
        for (int i = threadIdx.x; i < kDenseKeys; i += blockDim.x) {
            nul[i] = 0;
            cnt[i] = 0;
            if (OPS & 2) {
                slo[i] = 0;
                shi[i] = 0;
            }
            if (OPS & 4) mn[i] = 0x7fffffff;
            if (OPS & 8) mx[i] = (int)0x80000000;
        }
        __syncthreads();
        const unsigned long long lo = dp.offs[part], hi = dp.offs[part + 1];
        // Records in pairs (one 128-bit load) from the first even index at
        // or below lo, kInFlight pairs a thread in flight; the pairs' halves
        // outside [lo, hi) are skipped.  Thread 0 keeps the L2 prefetch four
        // iterations (256 KB) ahead of the loads.
        const unsigned long long p0 = lo >> 1, p1 = (hi + 1) >> 1;
        const uint4* pairs = (const uint4*)dp.recs;
        constexpr unsigned long long kStep = (unsigned long long)kDenseFoldThreads * kInFlight;  // pairs an iteration
        if (threadIdx.x == 0 && p0 < p1)
            prefetch_l2_range(pairs + p0, (p1 - p0 < 4 * kStep ? p1 - p0 : 4 * kStep) * sizeof(uint4));
        for (unsigned long long b0 = p0 + threadIdx.x; b0 < p1; b0 += kStep) {
            if (threadIdx.x == 0 && b0 + 4 * kStep < p1) {
                const unsigned long long a = b0 + 4 * kStep;
                prefetch_l2_range(pairs + a, (p1 - a < kStep ? p1 - a : kStep) * sizeof(uint4));
            }
            uint4 pr2[kInFlight];
#pragma unroll
            for (int j = 0; j < kInFlight; j++) {
                const unsigned long long i = b0 + (unsigned long long)j * kDenseFoldThreads;
                pr2[j] = i < p1 ? __ldcs(pairs + i) : make_uint4(0u, 0u, 0u, 0u);
            }
#pragma unroll
            for (int h = 0; h < 2 * kInFlight; h++) {
                const unsigned long long idx = 2 * (b0 + (unsigned long long)(h >> 1) * kDenseFoldThreads) + (h & 1);
                if (idx < lo || idx >= hi) continue;
                const uint2 r = (h & 1) ? make_uint2(pr2[h >> 1].z, pr2[h >> 1].w) : make_uint2(pr2[h >> 1].x, pr2[h >> 1].y);
                const unsigned off = (r.y >> 1) & (unsigned)(kDenseKeys - 1);
                if (!(r.y & 1u)) {  // a NULL value: the row counts, nothing else
                    atomicAdd(&nul[off], 1u);
                    continue;
                }
                const int x = (int)r.x;
                atomicAdd(&cnt[off], 1u);
                if (OPS & 2) {
                    // x sign-extended to 64 bits: a 32-bit add and its carry
                    const unsigned vlo = (unsigned)x, vhi = x < 0 ? 0xffffffffu : 0u;
                    const unsigned old = vlo ? atomicAdd(&slo[off], vlo) : 0u;
                    const unsigned up = vhi + (old + vlo < old ? 1u : 0u);
                    if (up) atomicAdd(&shi[off], up);
                }
                if (OPS & 4)
                    if (x < ((volatile int*)mn)[off]) atomicMin(&mn[off], x);
                if (OPS & 8)
                    if (x > ((volatile int*)mx)[off]) atomicMax(&mx[off], x);
            }
        }
        __syncthreads();
        // Flush in kPer rounds of kDenseFoldThreads consecutive slots, a slot a
        // thread: the occupied ones, ranked by a block prefix each round, go
        // to consecutive groups, so consecutive lanes store whole sectors.
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        const unsigned long long kbase = dp.lo + (unsigned long long)part * kDenseKeys;
        unsigned done = 0;  // groups of the rounds before
#pragma unroll 1
        for (int k = 0; k < kPer; k++) {
            const int sl = k * kDenseFoldThreads + threadIdx.x;
            const unsigned nrows = nul[sl] + cnt[sl];
            const unsigned ball = __ballot_sync(0xffffffffu, nrows != 0u);
            if (lane == 0) wsum[w] = __popc(ball);
            __syncthreads();
            if (w == 0) {
                const unsigned v = lane < (kDenseFoldThreads >> 5) ? wsum[lane] : 0u;
                unsigned vi = v;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned y = __shfl_up_sync(0xffffffffu, vi, o);
                    if (lane >= o) vi += y;
                }
                if (lane < (kDenseFoldThreads >> 5)) wsum[lane] = vi - v;
                if (lane == 31) s_total = vi;
            }
            __syncthreads();
            if (nrows) {
                const long long g = (long long)part * kDenseKeys + done + wsum[w] + __popc(ball & ((1u << lane) - 1u));
                P.keys[g] = (long long)((kbase + (unsigned long long)sl) ^ kSignBit);
                P.arr[g] = nrows;
                if (OPS & 1) P.arr[ops.count_arr * st + g] = cnt[sl];
                if (OPS & 2) P.arr[ops.sum_arr * st + g] = (unsigned long long)shi[sl] << 32 | slo[sl];
                if (OPS & 4) P.arr[ops.min_arr * st + g] = (unsigned long long)(long long)mn[sl];
                if (OPS & 8) P.arr[ops.max_arr * st + g] = (unsigned long long)(long long)mx[sl];
            }
            done += s_total;
            __syncthreads();
        }
        if (threadIdx.x == 0) gcount[part] = done;
        __syncthreads();
    }
}

using DenseFold = void (*)(const AggProgram, const DensePlan, const CompactOps, unsigned int*);
DenseFold dense_fold_for(int ops) {
    switch (ops) {
#define OXB_DF(m) \
    case m: return part_dense_fold_kernel<m>;
        OXB_DF(1) OXB_DF(2) OXB_DF(3) OXB_DF(4) OXB_DF(5) OXB_DF(6) OXB_DF(7) OXB_DF(8) OXB_DF(9) OXB_DF(10)
        OXB_DF(11) OXB_DF(12) OXB_DF(13) OXB_DF(14) OXB_DF(15)
#undef OXB_DF
        default: return nullptr;
    }
}

// The dense fold's groups in key order for agg_emit_kernel (whose key is
// skeys[r] ^ sign bit, with lo = 0): the key INT64_MIN first when its slot
// [capacity + 1] holds rows, then every partition's compacted groups, one
// block a partition, so each group's row is its partition's first plus its
// index there.
__global__ void dense_order_kernel(const __grid_constant__ AggProgram P, const unsigned long long* __restrict__ gpre,
                                   int np, int has_min, unsigned long long* __restrict__ skeys,
                                   unsigned int* __restrict__ sslots) {
    if (has_min && blockIdx.x == 0 && threadIdx.x == 0) {
        skeys[0] = 0;  // INT64_MIN ^ sign bit
        sslots[0] = (unsigned)(P.capacity + 1);
    }
    for (int p = blockIdx.x; p < np; p += gridDim.x) {
        const unsigned long long r0 = gpre[p] + (unsigned long long)has_min;
        const long long n = (long long)(gpre[p + 1] - gpre[p]);
        for (long long i = threadIdx.x; i < n; i += blockDim.x) {
            const long long slot = (long long)p * kDenseKeys + i;
            sslots[r0 + i] = (unsigned)slot;
            skeys[r0 + i] = (unsigned long long)P.keys[slot] ^ kSignBit;
        }
    }
}

size_t part_fold_smem(int narrays) { return (size_t)kPartSlots * (8 + 4 + 8 * (narrays - 1)); }

int maxacc_for(int nacc) { return nacc <= 2 ? 2 : (nacc <= 4 ? 4 : kMaxAccs); }

using RowsKernel = void (*)(const AggProgram, const DevPredicate, const AggKey, long long);
using JoinKernel = void (*)(const AggProgram, const DevPredicate, const AggKey, const void*, const uint8_t*, int,
                            const JoinTableDev, long long);

#define OXB_AGG_VARIANTS(X)                                                                                    \
    X(2, false, 1) X(2, false, 2) X(2, true, 1) X(2, true, 2) X(4, false, 1) X(4, false, 2) X(4, true, 1)      \
        X(4, true, 2) X(16, false, 1) X(16, false, 2)

RowsKernel rows_kernel_for(const AggVariant& v) {
    if (v.tile) {
        if (v.maxacc == 2) return agg_tile_rows_kernel<2>;
        if (v.maxacc == 4) return agg_tile_rows_kernel<4>;
    }
#define OXB_PICK(M, C, R) \
    if (v.maxacc == M && v.combine == C && v.rpt == R) return agg_rows_kernel<M, C, R>;
    OXB_AGG_VARIANTS(OXB_PICK)
#undef OXB_PICK
    fail(OXB_EXECUTION, "no aggregate kernel for this variant");
}

JoinKernel join_kernel_for(const AggVariant& v) {
    if (v.tile) {
        if (v.maxacc == 2) return agg_tile_join_kernel<2>;
        if (v.maxacc == 4) return agg_tile_join_kernel<4>;
    }
#define OXB_PICK(M, C, R) \
    if (v.maxacc == M && v.combine == C && v.rpt == R) return agg_join_kernel<M, C, R>;
    OXB_AGG_VARIANTS(OXB_PICK)
#undef OXB_PICK
    fail(OXB_EXECUTION, "no join-aggregate kernel for this variant");
}

using StreamRowsKernel = void (*)(const AggProgram, const DevPredicate, const StreamPlan);
using StreamJoinKernel = void (*)(const AggProgram, const DevPredicate, const StreamPlan, const AggKey,
                                  const JoinTableDev);

using StileKernel = void (*)(const AggProgram, const DevPredicate, const StreamPlan, const AggKey, const JoinTableDev);

StileKernel stile_kernel_for(int maxacc, bool join) {
    if (join) return maxacc == 2 ? agg_stile_kernel<2, true> : agg_stile_kernel<4, true>;
    return maxacc == 2 ? agg_stile_kernel<2, false> : agg_stile_kernel<4, false>;
}

StreamRowsKernel stream_rows_kernel_for(int maxacc) {
    if (maxacc == 2) return agg_stream_rows_kernel<2>;
    if (maxacc == 4) return agg_stream_rows_kernel<4>;
    return agg_stream_rows_kernel<kMaxAccs>;
}

StreamJoinKernel stream_join_kernel_for(int maxacc) {
    if (maxacc == 2) return agg_stream_join_kernel<2>;
    if (maxacc == 4) return agg_stream_join_kernel<4>;
    return agg_stream_join_kernel<kMaxAccs>;
}

using FusedKernel = void (*)(const AggProgram, const DevPredicate, const AggKey, const void*, const uint8_t*, int,
                             const JoinTableDev, const FusedTab, long long);

FusedKernel fused_kernel_for(const AggVariant& v) {
    if (v.vec) {
        if (v.dense) return v.rpt == 4 ? agg_fusedv_join_kernel<4, true> : agg_fusedv_join_kernel<8, true>;
        return v.rpt == 4 ? agg_fusedv_join_kernel<4, false> : agg_fusedv_join_kernel<8, false>;
    }
#define OXB_PICK(M, R, D) \
    if (v.maxacc == M && v.rpt == R && v.dense == D) return agg_fused_join_kernel<M, R, D>;
    OXB_PICK(2, 2, false) OXB_PICK(2, 4, false) OXB_PICK(4, 2, false) OXB_PICK(4, 4, false)
    OXB_PICK(2, 2, true) OXB_PICK(2, 4, true) OXB_PICK(4, 2, true) OXB_PICK(4, 4, true)
#undef OXB_PICK
    fail(OXB_EXECUTION, "no fused join kernel for this variant");
}

using FStreamKernel = void (*)(const AggProgram, const DevPredicate, const StreamPlan, const AggKey,
                               const JoinTableDev, const FusedTab);
FStreamKernel fstream_kernel_for(const AggVariant& v) {
    if (v.maxacc == 2) return v.dense ? agg_fstream_join_kernel<2, true> : agg_fstream_join_kernel<2, false>;
    return v.dense ? agg_fstream_join_kernel<4, true> : agg_fstream_join_kernel<4, false>;
}

// The lean kernels' accumulator shape for a program, or false when the
// program or its columns need the interpreted kernels.
bool lean_shape(const AggProgram& P, const DevPredicate& pred, const uint8_t* key_validity, int* a0, int* a1) {
    if (key_validity || P.nacc > 2 || pred.nleaves > 2) return false;
    for (int l = 0; l < pred.nleaves; l++)
        if (pred.leaves[l].validity) return false;
    int k[2] = {kLeanNone, kLeanNone};
    for (int j = 0; j < P.nacc; j++) {
        const DevAcc& a = P.acc[j];
        if (a.side != 0 || a.validity) return false;
        if (a.kind == kAccSumInt) k[j] = a.in_type == kInt32 ? kLeanSumI32 : kLeanSumI64;
        else if (a.kind == kAccSumF64 && a.in_type == kFloat64) k[j] = kLeanSumF64;
        else return false;
    }
    *a0 = k[0];
    *a1 = k[1];
    return true;
}

LeanPlan lean_plan(const AggProgram& P, const DevPredicate& pred) {
    LeanPlan L{};
    L.nleaves = pred.nleaves;
    static const int kMask[5] = {2, 1, 3, 4, 6};  // ==, <, <=, >, >= (cmp_holds' codes)
    for (int l = 0; l < pred.nleaves; l++) {
        L.leaf_width[l] = pred.leaves[l].type == kInt32 ? 4 : 8;
        L.leaf_f64[l] = pred.leaves[l].type == kFloat64;
        L.leaf_mask[l] = kMask[pred.leaves[l].op < 0 || pred.leaves[l].op > 4 ? 4 : pred.leaves[l].op];
    }
    for (int j = 0; j < P.nacc; j++) {
        L.acc_values[j] = P.acc[j].values;
        L.acc_arr[j] = P.acc[j].arr;
        L.acc_j[j] = j;
        L.acc_off[j] = P.acc[j].arr * P.smem_slots;
        L.fix[j] = P.acc[j].fix;
        L.fix_lo[j] = P.acc[j].fix_lo;
        L.acc_leaf[j] = -1;
        const int width = P.acc[j].in_type == kInt32 ? 4 : 8;
        for (int l = 0; l < pred.nleaves && l < 2; l++)
            if (pred.leaves[l].values == P.acc[j].values && L.leaf_width[l] == width) L.acc_leaf[j] = l;
    }
    return L;
}

using LeanKernel = void (*)(const AggProgram, const DevPredicate, const LeanPlan, const AggKey, const void*, int,
                            const JoinTableDev, const FusedTab, long long);

template <int A0, int A1>
LeanKernel lean_kernel_pick(bool dense, int rpt) {
    if (dense)
        return rpt >= 4 ? agg_lean_join_kernel<A0, A1, true, 4>
                        : (rpt == 1 ? agg_lean_join_kernel<A0, A1, true, 1> : agg_lean_join_kernel<A0, A1, true, 2>);
    return rpt >= 4 ? agg_lean_join_kernel<A0, A1, false, 4>
                    : (rpt == 1 ? agg_lean_join_kernel<A0, A1, false, 1> : agg_lean_join_kernel<A0, A1, false, 2>);
}

template <int A0>
LeanKernel lean_kernel_a1(int a1, bool dense, int rpt) {
    switch (a1) {
        case kLeanSumI32: return lean_kernel_pick<A0, kLeanSumI32>(dense, rpt);
        case kLeanSumI64: return lean_kernel_pick<A0, kLeanSumI64>(dense, rpt);
        case kLeanSumF64: return lean_kernel_pick<A0, kLeanSumF64>(dense, rpt);
        default: return lean_kernel_pick<A0, kLeanNone>(dense, rpt);
    }
}

template <int A0, int A1>
LeanKernel lean4_pick(bool dense) {
    return dense ? agg_lean4_join_kernel<A0, A1, true> : agg_lean4_join_kernel<A0, A1, false>;
}

template <int A0>
LeanKernel lean4_a1(int a1, bool dense) {
    switch (a1) {
        case kLeanSumI32: return lean4_pick<A0, kLeanSumI32>(dense);
        case kLeanSumI64: return lean4_pick<A0, kLeanSumI64>(dense);
        case kLeanSumF64: return lean4_pick<A0, kLeanSumF64>(dense);
        default: return lean4_pick<A0, kLeanNone>(dense);
    }
}

LeanKernel lean4_kernel_for(int a0, int a1, bool dense) {
    switch (a0) {
        case kLeanSumI32: return lean4_a1<kLeanSumI32>(a1, dense);
        case kLeanSumI64: return lean4_a1<kLeanSumI64>(a1, dense);
        case kLeanSumF64: return lean4_a1<kLeanSumF64>(a1, dense);
        default: return lean4_pick<kLeanNone, kLeanNone>(dense);
    }
}

LeanKernel lean_kernel_for(int a0, int a1, bool dense, int rpt) {
    switch (a0) {
        case kLeanSumI32: return lean_kernel_a1<kLeanSumI32>(a1, dense, rpt);
        case kLeanSumI64: return lean_kernel_a1<kLeanSumI64>(a1, dense, rpt);
        case kLeanSumF64: return lean_kernel_a1<kLeanSumF64>(a1, dense, rpt);
        default: return lean_kernel_pick<kLeanNone, kLeanNone>(dense, rpt);
    }
}

using LeanMultiKernel = void (*)(const AggProgram, const DevPredicate, const LeanPlan, const AggKey, int,
                                 const JoinTableDev, const FusedTab, const LeanReq*, int, long long,
                                 unsigned long long*);

template <int A0, int A1>
LeanMultiKernel lean_multi_pick(bool dense) {
    return dense ? agg_lean_multi_kernel<A0, A1, true, 2> : agg_lean_multi_kernel<A0, A1, false, 2>;
}

template <int A0>
LeanMultiKernel lean_multi_a1(int a1, bool dense) {
    switch (a1) {
        case kLeanSumI32: return lean_multi_pick<A0, kLeanSumI32>(dense);
        case kLeanSumI64: return lean_multi_pick<A0, kLeanSumI64>(dense);
        case kLeanSumF64: return lean_multi_pick<A0, kLeanSumF64>(dense);
        default: return lean_multi_pick<A0, kLeanNone>(dense);
    }
}

LeanMultiKernel lean_multi_kernel_for(int a0, int a1, bool dense) {
    switch (a0) {
        case kLeanSumI32: return lean_multi_a1<kLeanSumI32>(a1, dense);
        case kLeanSumI64: return lean_multi_a1<kLeanSumI64>(a1, dense);
        case kLeanSumF64: return lean_multi_a1<kLeanSumF64>(a1, dense);
        default: return lean_multi_pick<kLeanNone, kLeanNone>(dense);
    }
}

std::string variant_name(const char* base, const AggVariant& v) {
    if (v.fused && v.lean4)
        return std::string(base) + "<" + std::to_string(v.maxacc) + (v.dense ? ",fused-dense," : ",fused,") + "lean4>";
    if (v.fused && v.lean)
        return std::string(base) + "<" + std::to_string(v.maxacc) + (v.dense ? ",fused-dense," : ",fused,") + "lean," +
               std::to_string(v.rpt) + ">";
    if (v.fused && v.fstream)
        return std::string(base) + "<" + std::to_string(v.maxacc) + (v.dense ? ",fused-dense," : ",fused,") + "stream>";
    if (v.fused)
        return std::string(base) + "<" + std::to_string(v.maxacc) + (v.dense ? ",fused-dense," : ",fused,") +
               (v.vec ? "vec," : "") + std::to_string(v.rpt) + ">";
    if (v.stile) return std::string(base) + "<" + std::to_string(v.maxacc) + ",stream-tile>";
    if (v.stream) return std::string(base) + "<" + std::to_string(v.maxacc) + ",stream>";
    if (v.tile) return std::string(base) + "<" + std::to_string(v.maxacc) + ",tile>";
    return std::string(base) + "<" + std::to_string(v.maxacc) + (v.combine ? ",combine," : ",atomic,") +
           std::to_string(v.rpt) + ">";
}

oxb_batch* emit_ordered(const StreamRef& s, const Backend& b, const AggPlan& plan, const AggProgram& P,
                        const unsigned long long* okeys, const unsigned int* oslots, unsigned long long lo, long long G,
                        bool has_null);

// Collects the occupied slots of a filled table into the output batch: the
// groups sorted by key with the NULL group last (aggregate.rs:35-66), one
// column per aggregate.  nullptr when the table overflowed and the caller
// may retry with a bigger one.
oxb_batch* emit_groups(const StreamRef& s, const Backend& b, const AggPlan& plan, const AggProgram& P, unsigned int cap,
                       const unsigned int* status, bool allow_retry) {
    // Collect the occupied slots and their key range.
    const long long m = (long long)cap + 2;
    Scratch<unsigned int> flags(s, m);
    Scratch<unsigned long long> pos(s, m + 1);
    Scratch<unsigned long long> range(s, 2);
    unsigned long long init_range[2] = {~0ull, 0ull};
    OXB_CUDA(cudaMemcpyAsync(range.get(), init_range, sizeof init_range, cudaMemcpyHostToDevice, s->stream));
    note_launch(), agg_flags_kernel<<<grid_for(b, m, 256, 8), 256, 0, s->stream>>>(P, flags.get(), range.get());
    OXB_CUDA(cudaGetLastError());
    scan_u32_to_u64(s, b, flags.get(), pos.get(), m);
    struct {
        unsigned long long G, lo, hi, null_rows;
        uint32_t status;
    } h{};
    OXB_CUDA(cudaMemcpyAsync(&h.G, pos.get() + m, 8, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaMemcpyAsync(&h.lo, range.get(), 16, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaMemcpyAsync(&h.null_rows, P.arr + cap, 8, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaMemcpyAsync(&h.status, status, 4, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaStreamSynchronize(s->stream));
    if ((h.status & kStatusTableFull) && allow_retry) return nullptr;
    check_status_word(h.status, "aggregate");

    const long long G = (long long)h.G;
    const bool has_null = h.null_rows > 0;
    Scratch<unsigned long long> skeys(s, G + 1);
    Scratch<unsigned int> sslots(s, G + 1);
    unsigned long long lo = G > 0 ? h.lo : 0;
    const unsigned long long* okeys = skeys.get();  // the groups in key order
    const unsigned int* oslots = sslots.get();
    Scratch<unsigned long long> ukeys;
    Scratch<unsigned int> uslots;
    if (G > 0) {
        note_launch(), agg_compact_kernel<<<grid_for(b, m, 256, 8), 256, 0, s->stream>>>(P, flags.get(), pos.get(), lo,
                                                                                        skeys.get(), sslots.get());
        OXB_CUDA(cudaGetLastError());
        unsigned long long span = h.hi - h.lo;
        // Group keys are distinct: a narrow or well-filled span is ordered
        // by rank, without a sort.
        ukeys = Scratch<unsigned long long>(s, G + 1);
        uslots = Scratch<unsigned int>(s, G + 1);
        if (order_distinct_keys(s, b, skeys.get(), sslots.get(), G, span, ukeys.get(), uslots.get())) {
            okeys = ukeys.get();
            oslots = uslots.get();
        } else {
            int bits = 0;
            while (bits < 64 && (span >> bits) != 0) bits++;
            radix_sort_pairs(s, b, skeys.get(), sslots.get(), G, bits);
        }
    }
    return emit_ordered(s, b, plan, P, okeys, oslots, lo, G, has_null);
}

// The output batch from the groups in key order (okeys[r] + lo is the
// ordered key, oslots[r] the HBM slot of group r), the NULL group last.
oxb_batch* emit_ordered(const StreamRef& s, const Backend& b, const AggPlan& plan, const AggProgram& P,
                        const unsigned long long* okeys, const unsigned int* oslots, unsigned long long lo, long long G,
                        bool has_null) {
    const long long rows = G + (has_null ? 1 : 0);
    auto out = std::make_unique<oxb_batch>();
    out->rows = rows;
    AggOutput O{};
    O.key_type = plan.key_type;
    auto make_col = [&](int type, bool nullable) {
        Column c;
        c.type = type;
        c.length = rows;
        if (rows > 0) {
            c.owner_values = dev_alloc(s, rows * (size_t)type_width(type, 1), false);
            c.values = c.owner_values->ptr;
            if (nullable) {
                c.owner_validity = dev_alloc(s, ((rows + 31) / 32) * 4, true);
                c.validity = (uint8_t*)c.owner_validity->ptr;
            }
        }
        return c;
    };
    out->cols.push_back(make_col(plan.key_type, has_null));
    O.key = OutCol{out->cols[0].values, (unsigned int*)out->cols[0].validity};
    for (int j = 0; j < P.nout; j++) {
        const int f = P.out[j].func;
        const bool nullable = !(f == OXB_AGG_COUNT || f == OXB_AGG_COUNT_STAR);
        out->cols.push_back(make_col(plan.out_types[j], nullable));
        O.cols[j] = OutCol{out->cols.back().values, (unsigned int*)out->cols.back().validity};
    }
    if (rows > 0) {
        note_launch(), agg_emit_kernel<<<grid_for(b, rows, 256, 8), 256, 0, s->stream>>>(P, O, okeys, oslots, lo, G,
                                                                                        rows);
        OXB_CUDA(cudaGetLastError());
        OXB_CUDA(cudaStreamSynchronize(s->stream));
    }
    return out.release();
}

// Choices the autotuner made, per query shape, for this process.
std::mutex g_tune_mu;
std::map<std::string, AggVariant> g_tuned;

// Runs the planned aggregation kernel(s) and emits the sorted output batch.
// launch(P, smem, variant) launches the row-loop kernel of that variant.
template <typename Launch>
oxb_batch* run_aggregate(const StreamRef& s, const Backend& b, AggPlan& plan, const AggKey& key_for_sample,
                         long long sample_rows, long long max_groups, const char* kernel_name, const StreamPlan* SP,
                         int fusable, Launch&& launch) {
    AggProgram& P = plan.P;
    const int maxacc = maxacc_for(P.nacc);
    P.scratch_accs = maxacc <= 4 ? maxacc : 0;

    // Size the HBM table and the shared-memory levels from a strided sample:
    // a small HBM table when keys repeat, room for every row otherwise; warp
    // caches direct-mapped when the sampled keys span at most 64 keys (no
    // CTA table then), tagged otherwise; the CTA table direct-mapped when the
    // span fits it.  Keys outside a sampled span still fold correctly, one
    // level further out.
    unsigned int cap;
    long long sampled_distinct = 0;
    int fix_lo[kMaxAccs];
    unsigned long long span = ~0ull;
    long long span_lo = 0;
    {
        long long samples = sample_rows < 8192 ? sample_rows : 8192;
        // h[3 + j]: the sampled largest |x| of accumulator j's Float64 input,
        // which places its fixed-point window in the fused join kernels.
        unsigned long long h[3 + kMaxAccs] = {0, (unsigned long long)LLONG_MAX, (unsigned long long)LLONG_MIN};
        const long long fsamples = plan.acc_rows < 8192 ? plan.acc_rows : 8192;
        auto windowed = [&](int j) {
            const DevAcc& a = P.acc[j];
            return fusable && fsamples > 0 && a.kind == kAccSumF64 && a.in_type == kFloat64 && a.side == 0;
        };
        if (samples > 0) {
            const unsigned int tcap = 16384;
            Scratch<long long> t(s, tcap);
            Scratch<unsigned long long> out(s, 3 + kMaxAccs);
            OXB_CUDA(cudaMemcpyAsync(out.get(), h, sizeof h, cudaMemcpyHostToDevice, s->stream));
            note_launch(), fill_i64_kernel<<<16, 256, 0, s->stream>>>(t.get(), tcap, kEmptyKey);
            note_launch(), agg_sample_kernel<<<grid_for(b, samples, 256, 2), 256, 0, s->stream>>>(
                key_for_sample, sample_rows, samples, t.get(), tcap, out.get());
            for (int j = 0; j < P.nacc; j++)
                if (windowed(j))
                    note_launch(), f64_absmax_sample_kernel<<<grid_for(b, fsamples, 256, 2), 256, 0, s->stream>>>(
                        (const double*)P.acc[j].values, P.acc[j].validity, plan.acc_rows, fsamples, out.get() + 3 + j);
            OXB_CUDA(cudaGetLastError());
            OXB_CUDA(cudaMemcpyAsync(h, out.get(), sizeof h, cudaMemcpyDeviceToHost, s->stream));
            OXB_CUDA(cudaStreamSynchronize(s->stream));
        }
        // The window: |x| < 2^H with H one bit above the sampled largest
        // value's exponent (values up to twice it still fit), unit 2^(H - 63).
        for (int j = 0; j < P.nacc; j++) {
            fix_lo[j] = INT_MIN;
            if (!windowed(j) || h[3 + j] == 0) continue;
            int e = 0;
            std::frexp(as_f64_host(h[3 + j]), &e);  // |x| < 2^e
            const int lo = e + 1 - 63;
            if (lo >= -900 && lo <= 800) fix_lo[j] = lo;
        }
        const long long d = (long long)h[0];
        sampled_distinct = d;
        const long long full = max_groups < 1 ? 1 : max_groups;
        if (d * 8 <= samples) cap = next_pow2(std::min<long long>(2 * full, 64ll * d + 4096), 4096);
        else cap = next_pow2(2 * full, 4096);
        if (d > 0) {
            span_lo = (long long)h[1];
            span = (unsigned long long)(long long)h[2] - (unsigned long long)span_lo;
        }
    }
    // A base below the sampled minimum, leaving `room` slots of margin, that
    // does not wrap below the int64 range.
    auto direct_base = [&](int slots) {
        long long margin = (long long)(((unsigned long long)slots - 1 - span) / 2);
        return span_lo < LLONG_MIN + slots ? span_lo : span_lo - margin;
    };
    const size_t kBudget = 64 * 1024;
    // Shared-memory layout of the row-loop kernels (warp caches + CTA table)
    // and of the tile sort-reduce kernels (a bigger CTA table, no caches).
    struct SmemPlan {
        int S = 0, Sw = 0, direct = 0, wdirect = 0;
        long long direct_lo = 0, wdirect_lo = 0;
        size_t bytes = 0;
    };
    SmemPlan cp, tp;
    if (P.scratch_accs == 0) {
        // no combining, so no warp caches: the CTA table and HBM only
        for (cp.S = 2048; cp.S >= 64 && smem_bytes(cp.S, 0, P.narrays, 0) > kBudget; cp.S >>= 1) {
        }
    } else if (span < 64) {
        cp.Sw = 2;
        while ((unsigned long long)cp.Sw <= span) cp.Sw <<= 1;
        cp.wdirect = 1;
        cp.wdirect_lo = direct_base(cp.Sw);
    } else {
        for (cp.Sw = 64; cp.Sw > 8 && smem_bytes(0, cp.Sw, P.narrays, P.scratch_accs) > kBudget / 3; cp.Sw >>= 1) {
        }
        for (cp.S = 2048; cp.S >= 64 && smem_bytes(cp.S, cp.Sw, P.narrays, P.scratch_accs) > kBudget; cp.S >>= 1) {
        }
    }
    if (cp.S < 64) cp.S = 0;
    if (cp.S > 0 && span < (unsigned long long)cp.S) {
        cp.direct = 1;
        cp.direct_lo = direct_base(cp.S);
    }
    cp.bytes = smem_bytes(cp.S, cp.Sw, P.narrays, P.scratch_accs);
    if (maxacc <= 4) {
        for (tp.S = 2048; tp.S >= 64 && tile_smem_bytes(tp.S, P.narrays, maxacc) > kBudget; tp.S >>= 1) {
        }
        if (tp.S < 64) tp.S = 0;
        if (tp.S > 0 && span < (unsigned long long)tp.S) {
            tp.direct = 1;
            tp.direct_lo = direct_base(tp.S);
        }
        tp.bytes = tile_smem_bytes(tp.S, P.narrays, maxacc);
    }
    SmemPlan sp, stp;
    if (SP && SP->n >= 4ll * kStreamT && maxacc <= 4) {
        for (stp.S = 2048; stp.S >= 64 && stile_smem_bytes(stp.S, SP->stage_bytes, P.narrays, maxacc) > 110 * 1024;
             stp.S >>= 1) {
        }
        if (stp.S < 64) stp.S = 0;
        if (stp.S > 0 && span < (unsigned long long)stp.S) {
            stp.direct = 1;
            stp.direct_lo = direct_base(stp.S);
        }
        stp.bytes = stile_smem_bytes(stp.S, SP->stage_bytes, P.narrays, maxacc);
    }
    if (SP && SP->n >= 4ll * kStreamT) {
        for (sp.S = 2048; sp.S >= 64 && stream_smem_bytes(sp.S, SP->stage_bytes, SP->aos) > 110 * 1024; sp.S >>= 1) {
        }
        if (sp.S < 64) sp.S = 0;
        if (sp.S > 0 && span < (unsigned long long)sp.S) {
            sp.direct = 1;
            sp.direct_lo = direct_base(sp.S);
        }
        sp.bytes = stream_smem_bytes(sp.S, SP->stage_bytes, SP->aos);
    }
    // The fused join kernel: a direct-mapped CTA table over the sampled span
    // of the (build-side) group key, small enough for full occupancy.
    SmemPlan fp;
    if (fusable && maxacc <= 4 && span < 4096ull) {
        const size_t bytes = fused_smem_bytes((int)span + 1, P.narrays);
        if (bytes <= 48 * 1024) {
            fp.S = (int)span + 1;
            fp.direct = 1;
            fp.direct_lo = span_lo;
            fp.bytes = bytes;
        }
    }
    // ... and over streamed columns: the same table beside the stage ring.
    SmemPlan fsp;
    if (fp.S > 0 && SP && SP->n >= 4ll * kStreamT) {
        const size_t bytes = fstream_smem_bytes(fp.S, SP->stage_bytes, P.narrays);
        if (bytes <= 200 * 1024) {
            fsp = fp;
            fsp.bytes = bytes;
        }
    }
    auto configure = [&](const AggVariant& v) {
        const SmemPlan& p =
            v.fused ? (v.fstream ? fsp : fp) : (v.stile ? stp : (v.stream ? sp : (v.tile ? tp : cp)));
        for (int j = 0; j < P.nacc; j++) {  // fixed-point Float64 sums: the fused kernels only
            DevAcc& a = P.acc[j];
            a.fix = v.fused && fix_lo[j] != INT_MIN;
            a.fix_lo = a.fix ? fix_lo[j] : 0;
        }
        P.smem_slots = p.S;
        P.wslots = p.Sw;
        P.direct = p.direct;
        P.direct_lo = p.direct_lo;
        P.wdirect = p.wdirect;
        P.wdirect_lo = p.wdirect_lo;
        return p.bytes;
    };

    // The variant: the tuned one for this shape, else the default; the
    // autotuner (when on) times every candidate on this call's data once.
    // Warp caches need combining; without a CTA table the atomic-only path
    // would send every row to HBM, so it is no candidate then either.
    std::vector<AggVariant> candidates;
    // fusable: 1 the hashed probe table, 2 its dense form; bit 4 the lean
    // (compiled) kernels apply as well.
    const bool lean_ok = (fusable & 4) != 0;
    const bool lean4_ok = lean_ok && (fusable & 8) != 0;  // every column 16-byte aligned
    const bool dense_ok = (fusable & 3) == 2;
    for (int d = dense_ok ? 1 : 0; d >= 0 && fp.S > 0 && lean4_ok; d--) {
        AggVariant f{maxacc, false, kLeanPairRows, false};
        f.fused = f.lean = f.lean4 = true;
        f.dense = d == 1;
        candidates.push_back(f);
    }
    for (int d = dense_ok ? 1 : 0; d >= 0 && fp.S > 0 && lean_ok; d--)
        for (int r = 1; r <= 4; r *= 2) {
            AggVariant f{maxacc, false, r, false};
            f.fused = f.lean = true;
            f.dense = d == 1;
            candidates.push_back(f);
        }
    for (int d = dense_ok ? 1 : 0; d >= 0 && fp.S > 0; d--)
        for (int r = 2; r <= 8; r *= 2)
            for (int vec = 0; vec < 2; vec++) {
                if ((vec == 0 && r == 8) || (vec == 1 && r == 2)) continue;
                AggVariant f{maxacc, false, r, false};
                f.fused = true;
                f.vec = vec == 1;
                f.dense = d == 1;
                candidates.push_back(f);
            }
    for (int d = dense_ok ? 1 : 0; d >= 0 && fsp.S > 0; d--) {
        AggVariant f{maxacc, false, 1, false};
        f.fused = f.fstream = true;
        f.dense = d == 1;
        candidates.push_back(f);
    }
    if (stp.S > 0) candidates.push_back(AggVariant{maxacc, false, 1, false, false, true});
    if (sp.S > 0) candidates.push_back(AggVariant{maxacc, false, 1, false, true});
    if (tp.S > 0) candidates.push_back(AggVariant{maxacc, false, 1, true});
    for (int c = 0; c < (maxacc <= 4 ? 2 : 1); c++) {
        if (c == 0 && maxacc <= 4 && cp.S == 0) continue;
        for (int r = 1; r <= 2; r++) candidates.push_back(AggVariant{maxacc, c == 1, r, false});
    }
    int cap_class = 0;
    while ((1u << cap_class) < cap) cap_class++;
    const std::string shape = std::string(kernel_name) + "/" + std::to_string(maxacc) + "/" +
                              std::to_string(cp.wdirect) + std::to_string(cp.direct) + std::to_string(tp.direct) + "/" +
                              std::to_string(sampled_distinct * 8 <= 8192) + "/" + std::to_string(cap_class) + "/" +
                              std::to_string(fp.S > 0);
    AggVariant chosen{maxacc, maxacc <= 4, 2, tp.S > 0 && sp.S == 0, sp.S > 0 && stp.S == 0, stp.S > 0};
    if (fp.S > 0) {  // the compiled kernels where they apply: paired rows, else one row a thread
        chosen = AggVariant{maxacc, false, lean4_ok ? kLeanPairRows : lean_ok ? 1 : 2, false};
        chosen.fused = true;
        chosen.dense = dense_ok;
        chosen.lean = lean_ok;
        chosen.lean4 = lean4_ok;
    }
    bool tune = false;
    if (b.force_combine >= 0 || b.force_rpt > 0) {
        if (b.force_combine >= 0) {
            chosen.fused = ((b.force_combine >= 5 && b.force_combine <= 8) && fp.S > 0) ||
                           ((b.force_combine == 11 || b.force_combine == 12) && fsp.S > 0) ||
                           ((b.force_combine >= 13 && b.force_combine <= 16) && fp.S > 0);
            chosen.fstream = b.force_combine == 11 || b.force_combine == 12;
            chosen.lean = (b.force_combine >= 13 && b.force_combine <= 16) && lean_ok;
            chosen.lean4 = (b.force_combine == 15 || b.force_combine == 16) && lean4_ok;
            chosen.vec = b.force_combine == 7 || b.force_combine == 8;
            chosen.dense = (b.force_combine == 5 || b.force_combine == 7 || b.force_combine == 11 ||
                            b.force_combine == 13 || b.force_combine == 15) &&
                           dense_ok;
            chosen.stile = b.force_combine == 4 && stp.S > 0;
            chosen.stream = b.force_combine == 3 && sp.S > 0;
            chosen.tile = b.force_combine == 2 && tp.S > 0;
            chosen.combine = b.force_combine == 1 && maxacc <= 4;
        }
        if (b.force_rpt > 0) chosen.rpt = b.force_rpt;
        if (chosen.fstream) chosen.rpt = 1;
        else if (chosen.lean4) chosen.rpt = kLeanPairRows;
        else if (chosen.lean) chosen.rpt = chosen.rpt <= 1 ? 1 : (chosen.rpt <= 2 ? 2 : 4);
        else if (chosen.fused && chosen.vec) chosen.rpt = chosen.rpt <= 4 ? 4 : 8;
        else if (chosen.fused) chosen.rpt = chosen.rpt <= 2 ? 2 : 4;
        else if (chosen.rpt > 2) chosen.rpt = 2;
    } else {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(shape);
        if (it != g_tuned.end()) chosen = it->second;
        else tune = b.autotune;
    }

    for (int attempt = 0; attempt < 2; attempt++) {
        P.capacity = cap;
        P.probe_limit = attempt == 0 ? kMaxInsertProbes : cap;
        P.stride = (long long)cap + 2;
        AllocRef keys_mem = dev_alloc(s, (size_t)cap * 8, false);
        AllocRef arr_mem = dev_alloc(s, (size_t)P.narrays * P.stride * 8, false);
        Scratch<unsigned int> status(s, 1, true);
        P.keys = (long long*)keys_mem->ptr;
        P.arr = (unsigned long long*)arr_mem->ptr;
        P.status = status.get();
        auto init = [&]() {
            OXB_CUDA(cudaMemsetAsync(status.get(), 0, 4, s->stream));
            note_launch(), agg_init_kernel<<<grid_for(b, (long long)P.narrays * P.stride, 256, 8), 256, 0, s->stream>>>(P);
            OXB_CUDA(cudaGetLastError());
        };
        if (tune && attempt == 0) {
            // two rounds over the candidates, each kept at its faster time:
            // the first launch of a kernel also pays for its first touch
            std::vector<float> ms(candidates.size(), 1e30f);
            cudaEvent_t e0, e1;
            OXB_CUDA(cudaEventCreate(&e0));
            OXB_CUDA(cudaEventCreate(&e1));
            for (int round = 0; round < 2; round++)
                for (size_t c = 0; c < candidates.size(); c++) {
                    init();
                    OXB_CUDA(cudaEventRecord(e0, s->stream));
                    launch(P, configure(candidates[c]), candidates[c]);
                    OXB_CUDA(cudaEventRecord(e1, s->stream));
                    OXB_CUDA(cudaEventSynchronize(e1));
                    float t = 0.0f;
                    OXB_CUDA(cudaEventElapsedTime(&t, e0, e1));
                    ms[c] = std::min(ms[c], t);
                }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            size_t best = 0;
            for (size_t c = 1; c < candidates.size(); c++)
                if (ms[c] < ms[best]) best = c;
            if (!candidates.empty()) chosen = candidates[best];
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tuned[shape] = chosen;
        }
        init();
        {
            const std::string name = variant_name(kernel_name, chosen);
            KernelTimer timer(b, s, name.c_str());
            timer.begin();
            launch(P, configure(chosen), chosen);
            timer.end();
        }
        OXB_CUDA(cudaGetLastError());

        oxb_batch* out = emit_groups(s, b, plan, P, cap, status.get(), attempt == 0);
        if (!out) {
            cap = next_pow2(2 * (max_groups < 1 ? 1 : max_groups), 4096);
            continue;  // the small table overflowed: rerun with room for every row
        }
        return out;
    }
    fail(OXB_TABLE_FULL, "aggregate hash table full after a retry");
}

template <typename K>
void set_smem(K kernel, size_t smem) {
    allow_smem(kernel, smem);
}

// As many CTAs as fit on the GPU at once (the row loops are grid-strided),
// fewer when there is less work.
template <typename K>
int resident_grid(const Backend& b, K kernel, size_t smem, long long work) {
    int per_sm = 0;
    OXB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, smem));
    if (per_sm < 1) per_sm = 1;
    return grid_for(b, work, kThreads, per_sm);
}

}  // namespace


// The dense fold's output: groups numbered by a scan of the partitions'
// group counts, the key INT64_MIN first and the NULL group last.
oxb_batch* emit_dense(const StreamRef& s, const Backend& b, const AggPlan& plan, const AggProgram& P,
                      const DensePlan& dp, const unsigned int* gcount) {
    Scratch<unsigned long long> gpre(s, (size_t)dp.np + 1);
    scan_u32_to_u64(s, b, gcount, gpre.get(), dp.np);
    struct {
        unsigned long long G, null_rows, min_rows;
        uint32_t status;
    } h{};
    OXB_CUDA(cudaMemcpyAsync(&h.G, gpre.get() + dp.np, 8, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaMemcpyAsync(&h.null_rows, P.arr + P.capacity, 8, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaMemcpyAsync(&h.min_rows, P.arr + P.capacity + 1, 8, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaMemcpyAsync(&h.status, dp.status, 4, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaStreamSynchronize(s->stream));
    check_status_word(h.status, "aggregate");
    const int has_min = h.min_rows > 0 ? 1 : 0;
    const long long G = (long long)h.G + has_min;
    Scratch<unsigned long long> skeys(s, G + 1);
    Scratch<unsigned int> sslots(s, G + 1);
    if (G > 0) {
        note_launch(), dense_order_kernel<<<std::min(dp.np, b.sms * 8), 256, 0, s->stream>>>(P, gpre.get(), dp.np, has_min,
                                                                                           skeys.get(), sslots.get());
        OXB_CUDA(cudaGetLastError());
    }
    return emit_ordered(s, b, plan, P, skeys.get(), sslots.get(), 0, G, h.null_rows > 0);
}

// The dense-range passes (part_dense_*) when they apply: every accumulator
// reads one Int32 column and is among COUNT, SUM, MIN and MAX of it (with
// COUNT(*) beside them), the kept keys span at most 2^25 values, and, unless
// pinned (variant 17), enough rows are kept for the passes to pay.  nullptr
// otherwise, and the caller takes the direct or hashed passes.
// The compiled dense passes apply (DenseLean): no bitmap on the key or a
// WHERE column in any batch, at most two leaves, 16-byte aligned columns.
bool dense_lean_plan(const DevPredicate& pred, const std::vector<BatchCols>& hb, int q, DenseLean* L) {
    if (pred.nleaves > 2) return false;
    *L = DenseLean{};
    L->nleaves = pred.nleaves;
    static const int kMask[5] = {2, 1, 3, 4, 6};  // ==, <, <=, >, >= (cmp_holds' codes)
    for (int l = 0; l < pred.nleaves; l++) {
        const DevLeaf& lf = pred.leaves[l];
        if (lf.type != kInt32 && lf.type != kInt64 && lf.type != kFloat64) return false;
        L->leaf_w8[l] = lf.type != kInt32;
        L->leaf_f64[l] = lf.type == kFloat64;
        L->leaf_mask[l] = kMask[lf.op < 0 || lf.op > 4 ? 4 : lf.op];
        L->lit[l] = lf.lit;
    }
    auto aligned = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
    for (const BatchCols& c : hb) {
        if (c.n == 0) continue;
        if (c.key_valid || !aligned(c.key) || !aligned(c.vals[q])) return false;
        for (int l = 0; l < pred.nleaves; l++)
            if (c.lvalid[l] || !aligned(c.lvals[l])) return false;
    }
    return true;
}

oxb_batch* aggregate_dense(const StreamRef& s, const Backend& b, const AggPlan& plan, AggProgram P,
                           const DevPredicate& pred, int key_type, const BatchCols* dbatches,
                           const std::vector<BatchCols>& hb, long long nptiles, long long total, const int* acc_col,
                           KernelTimer& timer) {
    const int nb = (int)hb.size();
    const bool pinned = b.force_combine == 17;
    if (b.force_combine >= 0 && !pinned) return nullptr;
    if (nptiles == 0 || total >= (1ll << 32) || P.nacc < 1 || P.nacc > 4) return nullptr;
    for (int j = 1; j < P.nacc; j++)
        if (acc_col[j] != acc_col[0]) return nullptr;
    CompactOps ops;
    const int mask = compact_ops_of(P, &ops);
    if (!mask) return nullptr;

    // The sampled key range, widened by an eighth of it and a partition on
    // each side; the count pass then checks every kept key against it.
    Scratch<unsigned long long> smp(s, 4);
    unsigned long long hs[4] = {0, 0, ~0ull, 0};
    OXB_CUDA(cudaMemcpyAsync(smp.get(), hs, sizeof hs, cudaMemcpyHostToDevice, s->stream));
    note_launch(), part_dense_sample_kernel<<<kDenseSamples / 256, 256, 0, s->stream>>>(pred, key_type, dbatches, nb,
                                                                                      nptiles, kDenseSamples, smp.get());
    OXB_CUDA(cudaGetLastError());
    OXB_CUDA(cudaMemcpyAsync(hs, smp.get(), sizeof hs, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaStreamSynchronize(s->stream));
    if (hs[1] == 0 || hs[2] > hs[3]) return nullptr;
    const double kept_est = (double)hs[1] / (double)std::max<unsigned long long>(hs[0], 1) * (double)total;
    const unsigned long long margin = (hs[3] - hs[2]) / 8 + kDenseKeys;
    const unsigned long long lo = hs[2] > margin ? hs[2] - margin : 0ull;
    const unsigned long long hi = hs[3] < ~0ull - margin ? hs[3] + margin : ~0ull;
    const unsigned long long range = hi - lo;  // keys in the range, less one
    if (range >= (unsigned long long)kDenseMaxParts * kDenseKeys) return nullptr;
    const int np = (int)((range + kDenseKeys) / kDenseKeys);
    // Worth it from a million kept rows (below, the direct fold's table sits
    // in L2), unless the range's slots, which the fold initialises and scans
    // partition by partition, far outnumber the kept rows.  Measured at 200M
    // rows over 10M keys: 1.7 ms at 1 % kept against 3.0 ms for the direct
    // fold, whose HBM table misses L2 (about 80 G atomics/s there).
    auto worth = [&](double kept) {
        return pinned || (kept >= 1e6 && (double)np * kDenseKeys <= 16.0 * kept + (double)(1 << 22));
    };
    if (!worth(kept_est)) return nullptr;

    DensePlan dp{};
    dp.lo = lo;
    dp.span = (unsigned long long)np * kDenseKeys;
    dp.np = np;
    dp.np1 = (np + kDenseFan - 1) >> kDenseFanBits;
    dp.grid = b.sms * kDenseCtas;
    dp.q = 0;
    Scratch<unsigned int> counts1(s, (size_t)dp.np1 * dp.grid);
    Scratch<unsigned int> totals(s, (size_t)np, true);
    Scratch<unsigned long long> cnt_out(s, 2, true);
    dp.counts1 = counts1.get();
    dp.totals = totals.get();
    DenseLean L;
    const bool lean = dense_lean_plan(pred, hb, dp.q, &L);
    const bool k8 = key_type == kInt64;
    timer.begin();
    if (lean) {
        auto count = k8 ? part_dense_count_lean_kernel<true> : part_dense_count_lean_kernel<false>;
        note_launch(), count<<<dp.grid, kDenseThreads, (size_t)np * 4, s->stream>>>(L, dbatches, nb, nptiles, dp,
                                                                                    cnt_out.get());
    } else {
        note_launch(), part_dense_count_kernel<<<dp.grid, kDenseThreads, (size_t)np * 4, s->stream>>>(
            pred, key_type, dbatches, nb, nptiles, dp, cnt_out.get());
    }
    OXB_CUDA(cudaGetLastError());
    timer.end();
    unsigned long long hc[2] = {0, 0};
    OXB_CUDA(cudaMemcpyAsync(hc, cnt_out.get(), sizeof hc, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaStreamSynchronize(s->stream));
    if (hc[1] > 0 || !worth((double)hc[0])) return nullptr;

    Scratch<unsigned long long> offs1(s, (size_t)dp.np1 * dp.grid + 1);
    Scratch<unsigned long long> offs(s, (size_t)np + 1);
    scan_u32_to_u64(s, b, counts1.get(), offs1.get(), (long long)dp.np1 * dp.grid);
    scan_u32_to_u64(s, b, totals.get(), offs.get(), np);
    dp.offs1 = offs1.get();
    dp.offs = offs.get();
    dp.nrecs = hc[0];
    // an even number of records, so the fold's pair loads stay inside
    const size_t rec_bytes = (size_t)((hc[0] + 2) & ~1ull) * sizeof(uint2);
    AllocRef recs1_mem = dev_alloc(s, rec_bytes, false);
    AllocRef recs_mem = dev_alloc(s, rec_bytes, false);
    dp.recs1 = (uint2*)recs1_mem->ptr;
    dp.recs = (uint2*)recs_mem->ptr;
    Scratch<unsigned int> status(s, 1, true);
    dp.status = status.get();
    Scratch<unsigned int> gcount(s, (size_t)np);
    Scratch<long long> cstart(s, (size_t)dp.np1 + 1);
    Scratch<unsigned int> gcursor(s, (size_t)np);
    Scratch<unsigned long long> queue(s, 1, true);

    const long long cap = (long long)np * kDenseKeys;
    P.capacity = (unsigned int)cap;
    P.probe_limit = cap;
    P.stride = cap + 2;
    P.smem_slots = 0;
    P.wslots = 0;
    AllocRef keys_mem = dev_alloc(s, (size_t)cap * 8, false);
    AllocRef arr_mem = dev_alloc(s, (size_t)P.narrays * P.stride * 8, false);
    P.keys = (long long*)keys_mem->ptr;
    P.arr = (unsigned long long*)arr_mem->ptr;
    P.status = status.get();

    const int maxacc = maxacc_for(P.nacc);
    auto split = maxacc == 2 ? part_dense_split_kernel<2> : part_dense_split_kernel<4>;
    auto split_lean = maxacc == 2 ? (k8 ? part_dense_split_lean_kernel<2, true> : part_dense_split_lean_kernel<2, false>)
                                  : (k8 ? part_dense_split_lean_kernel<4, true> : part_dense_split_lean_kernel<4, false>);
    const size_t ssmem = dense_split_smem(dp.np1);
    set_smem(split, ssmem);
    set_smem(split_lean, ssmem);
    DenseFold fold = dense_fold_for(mask);
    const size_t fsmem = dense_fold_smem(mask);
    set_smem(fold, fsmem);
    int s2occ = 0;
    OXB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s2occ, part_dense_split2_kernel, kDenseThreads, 0));
    const long long chunks_max = (long long)(hc[0] / kDenseChunk) + dp.np1;
    const int s2grid = (int)std::max<long long>(1, std::min<long long>(chunks_max, (long long)b.sms * std::max(s2occ, 1)));
    timer.rename("agg_batches_dense");
    timer.begin();
    note_launch(), dense_special_init_kernel<<<1, 64, 0, s->stream>>>(P);
    if (lean)
        note_launch(), split_lean<<<dp.grid, kDenseThreads, ssmem, s->stream>>>(P, L, dbatches, nb, nptiles, dp);
    else
        note_launch(), split<<<dp.grid, kDenseThreads, ssmem, s->stream>>>(P, pred, key_type, dbatches, nb, nptiles, dp);
    note_launch(), dense_chunks_kernel<<<1, 256, 0, s->stream>>>(dp, cstart.get());
    note_launch(), dense_cursor_kernel<<<grid_for(b, np, 256, 4), 256, 0, s->stream>>>(dp, gcursor.get());
    note_launch(), part_dense_split2_kernel<<<s2grid, kDenseThreads, 0, s->stream>>>(dp, cstart.get(), queue.get(),
                                                                                    gcursor.get());
    note_launch(), fold<<<std::min(np, b.sms), kDenseFoldThreads, fsmem, s->stream>>>(P, dp, ops, gcount.get());
    OXB_CUDA(cudaGetLastError());
    timer.end();
    return emit_dense(s, b, plan, P, dp, gcount.get());
}

oxb_batch* aggregate_batches(const StreamRef& s, const Backend& b, const oxb_aggregate_batches_args& a) {
    if (a.ninputs < 1 || !a.inputs || !a.spec) fail(OXB_PLAN, "aggregate_batches: no inputs or no spec");
    for (int i = 0; i < a.ninputs; i++)
        if (!a.inputs[i]) fail(OXB_PLAN, "aggregate_batches: input batch " + std::to_string(i) + " is null");
    const oxb_batch& first = *a.inputs[0];
    const int ncols = (int)first.cols.size();
    for (int i = 1; i < a.ninputs; i++) {
        const oxb_batch& bt = *a.inputs[i];
        if ((int)bt.cols.size() != ncols) fail(OXB_PLAN, "input batches have different column counts");
        for (int c = 0; c < ncols; c++)
            if (bt.cols[c].type != first.cols[c].type || bt.cols[c].dim != first.cols[c].dim)
                fail(OXB_PLAN, "input batches differ in the type of column " + std::to_string(c));
    }
    const oxb_aggregate_spec& spec = *a.spec;
    if (spec.group_by < 0 || spec.group_by >= ncols) fail(OXB_PLAN, "group-by column out of range");
    // The plan's view of each column: a validity bitmap when any batch has
    // one (a batch without NULLs may carry none), so NULL-aware counts exist.
    std::vector<Column> rep(first.cols.begin(), first.cols.end());
    for (int c = 0; c < ncols; c++)
        for (int i = 0; i < a.ninputs && !rep[c].validity; i++) rep[c].validity = a.inputs[i]->cols[c].validity;
    const Column& key = rep[spec.group_by];
    if (key.type != kInt64 && key.type != kInt32)
        fail(OXB_UNSUPPORTED, "group key must be Int64 or Int32 on the device");
    if (spec.naggregates < 0 || spec.naggregates > kMaxOuts) fail(OXB_UNSUPPORTED, "too many aggregates");
    std::vector<int> funcs;
    std::vector<AggInputCol> inputs;
    for (int j = 0; j < spec.naggregates; j++) {
        const int f = spec.funcs[j];
        const Column* c = nullptr;
        if (f != OXB_AGG_COUNT_STAR) {
            if (spec.columns[j] < 0 || spec.columns[j] >= ncols) fail(OXB_PLAN, "aggregate column out of range");
            c = &rep[spec.columns[j]];
        }
        check_agg_input(f, c, spec.columns[j]);
        funcs.push_back(f);
        inputs.push_back(AggInputCol{c, 0, f == OXB_AGG_COUNT_STAR ? -1 : spec.columns[j]});
    }
    const DevPredicate pred = make_predicate(first, a.leaves, a.nleaves);
    AggPlan plan = plan_aggregate(funcs, inputs, key.type);
    AggProgram& P = plan.P;
    const int* acc_col = plan.acc_index;
    std::vector<BatchCols> hb(a.ninputs);
    long long ntiles = 0, nptiles = 0, total = 0;
    for (int i = 0; i < a.ninputs; i++) {
        const oxb_batch& bt = *a.inputs[i];
        BatchCols& c = hb[i];
        c = BatchCols{};
        c.n = bt.rows;
        c.tile0 = ntiles;
        c.ptile0 = nptiles;
        ntiles += (bt.rows + kBatchTile - 1) / kBatchTile;
        nptiles += (bt.rows + kPartTile - 1) / kPartTile;
        total += bt.rows;
        c.key = bt.cols[spec.group_by].values;
        c.key_valid = bt.cols[spec.group_by].validity;
        for (int j = 0; j < P.nacc; j++) {
            c.vals[j] = bt.cols[acc_col[j]].values;
            c.valid[j] = bt.cols[acc_col[j]].validity;
        }
        for (int l = 0; l < a.nleaves; l++) {
            c.lvals[l] = bt.cols[a.leaves[l].column].values;
            c.lvalid[l] = bt.cols[a.leaves[l].column].validity;
        }
    }
    Scratch<BatchCols> dbatches(s, hb.size());
    OXB_CUDA(cudaMemcpyAsync(dbatches.get(), hb.data(), hb.size() * sizeof(BatchCols), cudaMemcpyHostToDevice, s->stream));

    // One pass over the input: distinct keys and count of the kept rows, and
    // their fine partition histogram (KernelTimer: this pass plus the fold).
    KernelTimer timer(b, s, "agg_batches_kernel");
    if (oxb_batch* out = aggregate_dense(s, b, plan, P, pred, key.type, dbatches.get(), hb, nptiles, total, acc_col,
                                         timer))
        return out;
    Scratch<unsigned> regs(s, kHllRegs, true);
    Scratch<unsigned int> fine(s, kFine, true);
    Scratch<unsigned long long> kept_dev(s, 1, true);
    const size_t scan_smem = (size_t)(kHllRegs + kFine) * 4;
    set_smem(part_scan_kernel, scan_smem);
    timer.begin();
    if (nptiles > 0) {
        int socc = 0;
        OXB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&socc, part_scan_kernel, kScanThreads, scan_smem));
        const long long sgrid0 = std::max<long long>(1, std::min<long long>(nptiles, (long long)b.sms * std::max(socc, 1)));
        note_launch(), part_scan_kernel<<<(unsigned)sgrid0, kScanThreads, scan_smem, s->stream>>>(
            pred, key.type, dbatches.get(), a.ninputs, nptiles, regs.get(), fine.get(), kept_dev.get());
        OXB_CUDA(cudaGetLastError());
    }
    timer.end();
    std::vector<unsigned> hregs(kHllRegs);
    unsigned long long kept = 0;
    OXB_CUDA(cudaMemcpyAsync(hregs.data(), regs.get(), kHllRegs * 4, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaMemcpyAsync(&kept, kept_dev.get(), 8, cudaMemcpyDeviceToHost, s->stream));
    OXB_CUDA(cudaStreamSynchronize(s->stream));
    const double est = hll_estimate(hregs);
    const long long all_rows = next_pow2(2 * std::max<long long>(total, 1), 4096);
    unsigned int cap = next_pow2(std::max<long long>(4096, (long long)(est * 1.2 * 2.0) + 1), 4096);
    if ((long long)cap > all_rows) cap = (unsigned int)all_rows;

    const int maxacc = maxacc_for(P.nacc);
    auto kern = maxacc == 2 ? agg_batches_kernel<2> : (maxacc == 4 ? agg_batches_kernel<4> : agg_batches_kernel<kMaxAccs>);
    int per_sm = 0;
    OXB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, 0));
    const long long grid = std::max<long long>(1, std::min<long long>(ntiles, (long long)b.sms * std::max(per_sm, 1)));

    // The hash-partitioned passes pay two more passes over the kept rows and
    // a second read of the input; they win when the HBM table is well beyond
    // L2 (each kept row then costs the direct fold several random HBM
    // accesses) and enough rows are kept: measured on B200, about 0.22 ms per
    // million kept rows direct against 0.10 partitioned, plus about 9 us per
    // million input rows.  The stored columns are the distinct inputs of the
    // accumulators.  Pinned variants: 9 the partitioned passes as planned,
    // 10 with the fewest partitions (so that partitions overflow their shared
    // tables), 0..8 the direct kernel.
    PartPlan pp{};
    const bool pinned = b.force_combine >= 0;
    const double table_bytes = (double)cap * 8.0 * (1 + P.narrays);
    const bool worth = table_bytes > 64.0 * (1 << 20) && (double)kept >= (double)total / 12.0 + 4e6;
    bool partitioned = maxacc <= 4 && total < (1ll << 32) && nptiles > 0 &&
                       (pinned ? (b.force_combine == 9 || b.force_combine == 10) : worth);
    if (partitioned) {
        for (int j = 0; j < P.nacc; j++) {
            int c = 0;
            while (c < pp.ncols && plan.acc_index[pp.src_of_col[c]] != acc_col[j]) c++;
            if (c == pp.ncols) {
                pp.src_of_col[c] = j;
                pp.width[c] = rep[acc_col[j]].type == kInt32 ? 4 : 8;
                pp.ncols++;
            }
            pp.col_of_acc[j] = c;
        }
        int np = 64, lg = 6;
        while (b.force_combine != 10 && np < kMaxParts && (double)np * kPartKeys < est) {
            np <<= 1;
            lg++;
        }
        pp.nparts = np;
        pp.shift = 64 - lg;
        pp.fstride = kFine >> lg;
        pp.f2_bits = lg > 7 ? lg - 7 : 0;  // at most kMaxF1 level-1 partitions
        pp.compact = pp.ncols == 1 && pp.width[0] == 4;
    }
    const int units = pp.compact ? 1 : (pp.ncols + 3) >> 1;
    AllocRef recs_mem, recs2_mem;
    if (partitioned) {
        recs_mem = dev_alloc(s, (size_t)total * units * 16, false);
        pp.recs = (uint4*)recs_mem->ptr;
        pp.recs2 = pp.recs;
        if (pp.f2_bits > 0) {
            recs2_mem = dev_alloc(s, (size_t)total * units * 16, false);
            pp.recs2 = (uint4*)recs2_mem->ptr;
        }
        timer.rename("agg_batches_partitioned");
    }
    auto psplit1 = pp.compact ? (maxacc == 2 ? part_split1_kernel<2, true> : part_split1_kernel<4, true>)
                              : (maxacc == 2 ? part_split1_kernel<2, false> : part_split1_kernel<4, false>);
    auto psplit2 = units == 1 ? part_split2_kernel<1> : (units == 2 ? part_split2_kernel<2> : part_split2_kernel<3>);
    auto pfold = maxacc == 2 ? (units == 1 ? part_fold_kernel<2, 1> : part_fold_kernel<2, 2>)
                             : (units == 1 ? part_fold_kernel<4, 1>
                                           : (units == 2 ? part_fold_kernel<4, 2> : part_fold_kernel<4, 3>));
    for (int attempt = 0;; attempt++) {
        P.capacity = cap;
        P.probe_limit = (long long)cap < all_rows ? kMaxInsertProbes : cap;
        P.stride = (long long)cap + 2;
        P.smem_slots = 0;
        P.wslots = 0;
        AllocRef keys_mem = dev_alloc(s, (size_t)cap * 8, false);
        AllocRef arr_mem = dev_alloc(s, (size_t)P.narrays * P.stride * 8, false);
        Scratch<unsigned int> status(s, 1, true);
        Scratch<unsigned long long> queue(s, 1, true);
        P.keys = (long long*)keys_mem->ptr;
        P.arr = (unsigned long long*)arr_mem->ptr;
        P.status = status.get();
        timer.begin();
        note_launch(), agg_init_kernel<<<grid_for(b, (long long)P.narrays * P.stride, 256, 8), 256, 0, s->stream>>>(P);
        OXB_CUDA(cudaGetLastError());
        if (partitioned) {
            const int f1 = pp.nparts >> pp.f2_bits, f2 = 1 << pp.f2_bits;
            const size_t fsmem = part_fold_smem(P.narrays);
            set_smem(pfold, fsmem);
            // one CTA per unit of work (a tile, a partition) up to a full GPU
            const long long sgrid = resident_grid(b, psplit1, 0, nptiles * kThreads);
            const long long fgrid = resident_grid(b, pfold, fsmem, (long long)pp.nparts * kThreads);
            Scratch<unsigned long long> offs(s, kFine + 1);
            Scratch<unsigned long long> cursor1(s, f1);
            Scratch<unsigned long long> cursor2(s, pp.nparts);
            Scratch<long long> tstart(s, f1 + 1);
            Scratch<unsigned long long> queue2(s, 1, true);
            // every fine bucket's first record; partition p starts at bucket p * fstride
            scan_u32_to_u64(s, b, fine.get(), offs.get(), kFine);
            OXB_CUDA(cudaMemcpy2DAsync(cursor1.get(), 8, offs.get(), (size_t)f2 * pp.fstride * 8, 8, f1,
                                       cudaMemcpyDeviceToDevice, s->stream));
            note_launch(), psplit1<<<(unsigned)sgrid, kThreads, 0, s->stream>>>(P, pred, key.type, dbatches.get(), a.ninputs,
                                                                               nptiles, queue.get(), pp, cursor1.get());
            if (f2 > 1) {
                OXB_CUDA(cudaMemcpy2DAsync(cursor2.get(), 8, offs.get(), (size_t)pp.fstride * 8, 8, pp.nparts,
                                           cudaMemcpyDeviceToDevice, s->stream));
                note_launch(), part_tiles_kernel<<<1, 32, 0, s->stream>>>(offs.get(), f1, f2, pp.fstride, tstart.get());
                const long long grid2 = resident_grid(b, psplit2, 0, ((total + kSplitTile - 1) / kSplitTile + f1) * kThreads);
                note_launch(), psplit2<<<(unsigned)grid2, kThreads, 0, s->stream>>>(pp, offs.get(), tstart.get(),
                                                                                   queue2.get(), cursor2.get());
            }
            CompactOps cops;
            const int cmask = units == 1 ? compact_ops_of(P, &cops) : 0;
            if (cmask) {
                CompactFold cf = compact_fold_for(cmask);
                set_smem(cf, fsmem);
                note_launch(), cf<<<(unsigned)resident_grid(b, cf, fsmem, (long long)pp.nparts * kThreads), kThreads, fsmem,
                                    s->stream>>>(P, pp, cops, offs.get());
            } else {
                note_launch(), pfold<<<(unsigned)fgrid, kThreads, fsmem, s->stream>>>(P, pp, offs.get());
            }
            timer.end();
            OXB_CUDA(cudaGetLastError());
        } else {
            if (ntiles > 0)
                note_launch(), kern<<<(unsigned)grid, kThreads, 0, s->stream>>>(P, pred, key.type, dbatches.get(),
                                                                                a.ninputs, ntiles, queue.get());
            timer.end();
            OXB_CUDA(cudaGetLastError());
        }
        const bool can_retry = (long long)cap < all_rows;
        oxb_batch* out = emit_groups(s, b, plan, P, cap, status.get(), can_retry);
        if (out) return out;
        cap = (unsigned int)std::min<long long>(2ll * cap, all_rows);  // the estimate was low: double the table
    }
}

oxb_batch* aggregate(const StreamRef& s, const Backend& b, const oxb_aggregate_args& a) {
    if (!a.input || !a.spec) fail(OXB_PLAN, "aggregate: null input or spec");
    const oxb_batch& in = *a.input;
    const oxb_aggregate_spec& spec = *a.spec;
    const int ncols = (int)in.cols.size();
    if (spec.group_by < 0 || spec.group_by >= ncols)
        fail(OXB_PLAN, "column index " + std::to_string(spec.group_by) + " out of range for a batch with " +
                           std::to_string(ncols) + " columns");
    const Column& key = in.cols[spec.group_by];
    if (key.type != kInt64 && key.type != kInt32)
        fail(OXB_UNSUPPORTED, "group key column " + std::to_string(spec.group_by) + " has type " +
                                  std::to_string(key.type) + "; Int64 and Int32 run on the device");
    if (spec.naggregates < 0 || spec.naggregates > kMaxOuts) fail(OXB_UNSUPPORTED, "too many aggregates");
    std::vector<int> funcs;
    std::vector<AggInputCol> inputs;
    for (int j = 0; j < spec.naggregates; j++) {
        const int f = spec.funcs[j];
        const Column* c = nullptr;
        if (f != OXB_AGG_COUNT_STAR) {
            if (spec.columns[j] < 0 || spec.columns[j] >= ncols)
                fail(OXB_PLAN, "column index " + std::to_string(spec.columns[j]) + " out of range");
            c = &in.cols[spec.columns[j]];
        }
        check_agg_input(f, c, spec.columns[j]);
        funcs.push_back(f);
        inputs.push_back(AggInputCol{c, 0});
    }
    DevPredicate pred = make_predicate(in, a.leaves, a.nleaves);
    AggPlan plan = plan_aggregate(funcs, inputs, key.type);
    const long long n = in.rows;
    AggKey k{key.values, key.validity, key.type, 0};
    StreamPlan SP;
    const bool streamable = plan_stream(plan.P, pred, key.values, key.validity, key.type, n, &SP);
    return run_aggregate(s, b, plan, k, n, n, "agg_rows_kernel", streamable ? &SP : nullptr, 0,
                         [&](AggProgram& P, size_t smem, const AggVariant& v) {
        if (n == 0) return;
        if (v.stile) {
            StileKernel kern = stile_kernel_for(v.maxacc, false);
            set_smem(kern, smem);
            int per_sm = 0;
            OXB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kStreamThreads, smem));
            const long long grid = std::min<long long>(SP.ntiles, (long long)b.sms * std::max(per_sm, 1));
            note_launch(), kern<<<(unsigned)grid, kStreamThreads, smem, s->stream>>>(P, pred, SP, k, JoinTableDev{});
            return;
        }
        if (v.stream) {
            StreamRowsKernel kern = stream_rows_kernel_for(v.maxacc);
            set_smem(kern, smem);
            int per_sm = 0;
            OXB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kStreamThreads, smem));
            const long long grid = std::min<long long>(SP.ntiles, (long long)b.sms * std::max(per_sm, 1));
            note_launch(), kern<<<(unsigned)grid, kStreamThreads, smem, s->stream>>>(P, pred, SP);
            return;
        }
        RowsKernel kern = rows_kernel_for(v);
        set_smem(kern, smem);
        note_launch(), kern<<<resident_grid(b, kern, smem, (n + v.rpt - 1) / v.rpt), kThreads, smem, s->stream>>>(P, pred, k, n);
    });
}

oxb_batch* join_aggregate(const StreamRef& s, const Backend& b, const oxb_join_aggregate_args& a) {
    if (!a.probe || !a.table || !a.build) fail(OXB_PLAN, "join_aggregate: null probe, build or table");
    const oxb_batch& probe = *a.probe;
    const oxb_batch& build = *a.build;
    if (a.table->build_rows != build.rows)
        fail(OXB_EXECUTION, "the join table indexes " + std::to_string(a.table->build_rows) +
                                " build rows but the build batch has " + std::to_string(build.rows));
    if (a.probe_key < 0 || a.probe_key >= (int)probe.cols.size()) fail(OXB_PLAN, "probe key column out of range");
    const Column& pk = probe.cols[a.probe_key];
    if (pk.type != kInt64 && pk.type != kInt32) fail(OXB_UNSUPPORTED, "probe join key must be Int64 or Int32");
    auto side_col = [&](int side, int col) -> const Column* {
        if (side != 0 && side != 1) fail(OXB_PLAN, "side must be 0 (probe) or 1 (build)");
        const oxb_batch& bt = side ? build : probe;
        if (col < 0 || col >= (int)bt.cols.size()) fail(OXB_PLAN, "column index " + std::to_string(col) + " out of range");
        return &bt.cols[col];
    };
    const Column* gk = side_col(a.group_side, a.group_column);
    if (gk->type != kInt64 && gk->type != kInt32) fail(OXB_UNSUPPORTED, "group key must be Int64 or Int32");
    if (a.naggregates < 0 || a.naggregates > kMaxOuts) fail(OXB_UNSUPPORTED, "too many aggregates");
    std::vector<int> funcs;
    std::vector<AggInputCol> inputs;
    for (int j = 0; j < a.naggregates; j++) {
        const Column* c = a.funcs[j] == OXB_AGG_COUNT_STAR ? nullptr : side_col(a.sides[j], a.columns[j]);
        check_agg_input(a.funcs[j], c, a.columns[j]);
        funcs.push_back(a.funcs[j]);
        inputs.push_back(AggInputCol{c, a.sides[j]});
    }
    DevPredicate pred = make_predicate(probe, a.leaves, a.nleaves);
    AggPlan plan = plan_aggregate(funcs, inputs, gk->type);
    const long long n = probe.rows;
    AggKey k{gk->values, gk->validity, gk->type, a.group_side};
    // The groups are at most the distinct group keys of the side they come
    // from; the sample is taken over that side's column.
    const long long group_rows = a.group_side ? build.rows : probe.rows;
    plan.acc_rows = probe.rows;
    AggKey sample_key{gk->values, gk->validity, gk->type, 0};
    const JoinTableDev jt = a.table->t;
    StreamPlan SP;
    const bool streamable = plan_stream(plan.P, pred, pk.values, pk.validity, pk.type, n, &SP);
    // The fused probe-table kernel takes a build-side group key and
    // probe-side aggregate inputs.
    // Its CTA row counts are u32: with at least one CTA per SM, fewer than
    // 2^38 probe rows keep every CTA under 2^32.
    bool fusable = a.group_side == 1 && n < (1ll << 38);
    for (int j = 0; j < plan.P.nacc; j++) fusable = fusable && plan.P.acc[j].side == 0;
    // The dense lookup table when the build keys fill at least a quarter of
    // their range (and it stays under 256 MB).
    const unsigned long long key_span = (unsigned long long)jt.key_hi - (unsigned long long)jt.key_lo;
    const bool dense = jt.key_lo <= jt.key_hi && key_span < (1ull << 26) &&
                       (long long)key_span < 4 * jt.ndistinct + 4096;
    int la0 = kLeanNone, la1 = kLeanNone;
    const bool lean = fusable && lean_shape(plan.P, pred, pk.validity, &la0, &la1);
    bool aligned = ((uintptr_t)pk.values & 15) == 0;
    for (int l = 0; l < pred.nleaves && l < 2; l++) aligned = aligned && ((uintptr_t)pred.leaves[l].values & 15) == 0;
    for (int j = 0; j < plan.P.nacc; j++) aligned = aligned && ((uintptr_t)plan.P.acc[j].values & 15) == 0;
    return run_aggregate(s, b, plan, sample_key, group_rows, group_rows, "agg_join_kernel", streamable ? &SP : nullptr,
                         fusable ? (dense ? 2 : 1) | (lean ? 4 : 0) | (lean && aligned ? 8 : 0) : 0,
                         [&](AggProgram& P, size_t smem, const AggVariant& v) {
                             if (n == 0) return;
                             if (v.fused) {
                                 FusedTab ft{};
                                 AllocRef fs;
                                 const int grid = grid_for(b, jt.capacity, 256, 8);
                                 if (v.dense) {
                                     ft.dense_lo = jt.key_lo;
                                     ft.dense_n = key_span + 1;
                                     fs = dev_alloc(s, (size_t)ft.dense_n * 4, false);
                                     OXB_CUDA(cudaMemsetAsync(fs->ptr, 0xff, (size_t)ft.dense_n * 4, s->stream));
                                     ft.dense = (const int*)fs->ptr;
                                     note_launch(), fuse_dense_kernel<<<grid, 256, 0, s->stream>>>(
                                         jt, k, P.direct_lo, P.smem_slots, (int*)fs->ptr, ft.dense_lo);
                                 } else {
                                     fs = dev_alloc(s, (size_t)jt.capacity * sizeof(FusedSlot), false);
                                     ft.slots = (const FusedSlot*)fs->ptr;
                                     note_launch(), fuse_table_kernel<<<grid, 256, 0, s->stream>>>(
                                         jt, k, P.direct_lo, P.smem_slots, (FusedSlot*)fs->ptr);
                                 }
                                 if (v.lean) {
                                     LeanKernel kern = v.lean4 ? lean4_kernel_for(la0, la1, v.dense)
                                                               : lean_kernel_for(la0, la1, v.dense, v.rpt);
                                     set_smem(kern, smem);
                                     note_launch(), kern<<<resident_grid(b, kern, smem, (n + v.rpt - 1) / v.rpt),
                                                           kFusedThreads, smem, s->stream>>>(
                                         P, pred, lean_plan(P, pred), k, pk.values, pk.type, jt, ft, n);
                                     return;
                                 }
                                 if (v.fstream) {
                                     FStreamKernel kern = fstream_kernel_for(v);
                                     set_smem(kern, smem);
                                     int per_sm = 0;
                                     OXB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kStreamThreads,
                                                                                            smem));
                                     const long long grid =
                                         std::min<long long>(SP.ntiles, (long long)b.sms * std::max(per_sm, 1));
                                     note_launch(), kern<<<(unsigned)grid, kStreamThreads, smem, s->stream>>>(P, pred, SP, k,
                                                                                                             jt, ft);
                                     return;
                                 }
                                 FusedKernel kern = fused_kernel_for(v);
                                 set_smem(kern, smem);
                                 note_launch(), kern<<<resident_grid(b, kern, smem, (n + v.rpt - 1) / v.rpt), kFusedThreads,
                                                       smem, s->stream>>>(P, pred, k, pk.values, pk.validity, pk.type, jt, ft, n);
                                 return;
                             }
                             if (v.stile) {
                                 StileKernel kern = stile_kernel_for(v.maxacc, true);
                                 set_smem(kern, smem);
                                 int per_sm = 0;
                                 OXB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kStreamThreads, smem));
                                 const long long grid = std::min<long long>(SP.ntiles, (long long)b.sms * std::max(per_sm, 1));
                                 note_launch(), kern<<<(unsigned)grid, kStreamThreads, smem, s->stream>>>(P, pred, SP, k, jt);
                                 return;
                             }
                             if (v.stream) {
                                 StreamJoinKernel kern = stream_join_kernel_for(v.maxacc);
                                 set_smem(kern, smem);
                                 int per_sm = 0;
                                 OXB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kStreamThreads, smem));
                                 const long long grid = std::min<long long>(SP.ntiles, (long long)b.sms * std::max(per_sm, 1));
                                 note_launch(), kern<<<(unsigned)grid, kStreamThreads, smem, s->stream>>>(P, pred, SP, k, jt);
                                 return;
                             }
                             JoinKernel kern = join_kernel_for(v);
                             set_smem(kern, smem);
                             note_launch(), kern<<<resident_grid(b, kern, smem, (n + v.rpt - 1) / v.rpt), kThreads, smem,
                                                   s->stream>>>(P, pred, k, pk.values, pk.validity, pk.type, jt, n);
                         });
}

// True when two join-aggregate requests differ at most in their probe batch
// (same column types) and their WHERE literals.
bool same_join_shape(const oxb_join_aggregate_args& a, const oxb_join_aggregate_args& z) {
    if (a.table != z.table || a.build != z.build || a.probe_key != z.probe_key || a.group_side != z.group_side ||
        a.group_column != z.group_column || a.naggregates != z.naggregates || a.nleaves != z.nleaves || !a.probe ||
        !z.probe || a.probe->cols.size() != z.probe->cols.size())
        return false;
    for (size_t c = 0; c < a.probe->cols.size(); c++)
        if (a.probe->cols[c].type != z.probe->cols[c].type) return false;
    for (int j = 0; j < a.naggregates; j++)
        if (a.funcs[j] != z.funcs[j] || a.sides[j] != z.sides[j] || a.columns[j] != z.columns[j]) return false;
    for (int l = 0; l < a.nleaves; l++)
        if (a.leaves[l].column != z.leaves[l].column || a.leaves[l].op != z.leaves[l].op ||
            a.leaves[l].lit_type != z.leaves[l].lit_type)
            return false;
    return true;
}

// Several join-aggregates of one shape in one launch of the compiled fused
// kernel (agg_lean_multi_kernel); requests that cannot share it, and one
// whose small table overflows, run alone through join_aggregate.
std::vector<oxb_batch*> join_aggregate_many(const StreamRef& s, const Backend& b, const oxb_join_aggregate_args* all,
                                            int nall) {
    std::vector<oxb_batch*> res(nall, nullptr);
    try {
        // The requests that can share the launch: the compiled kernel's shape,
        // the first such request's; the others run alone.
        std::vector<int> idx;
        std::vector<AggPlan> plans;
        std::vector<DevPredicate> preds;
        int la0 = kLeanNone, la1 = kLeanNone;
        for (int r = 0; r < nall; r++) {
            const oxb_join_aggregate_args& ar = all[r];
            bool ok = ar.probe && ar.build && ar.table && ar.group_side == 1 && ar.probe->rows < (1ll << 38) &&
                      ar.group_column >= 0 && ar.group_column < (int)ar.build->cols.size() && ar.probe_key >= 0 &&
                      ar.probe_key < (int)ar.probe->cols.size() && ar.table->build_rows == ar.build->rows &&
                      ar.naggregates >= 0 && ar.naggregates <= kMaxOuts;
            if (ok && !idx.empty()) ok = same_join_shape(ar, all[idx[0]]);
            if (ok) {
                const Column& g = ar.build->cols[ar.group_column];
                ok = g.type == kInt64 || g.type == kInt32;
            }
            std::vector<int> funcs;
            std::vector<AggInputCol> inputs;
            for (int j = 0; ok && j < ar.naggregates; j++) {
                if (ar.funcs[j] != OXB_AGG_COUNT_STAR &&
                    (ar.sides[j] != 0 || ar.columns[j] < 0 || ar.columns[j] >= (int)ar.probe->cols.size())) {
                    ok = false;
                    break;
                }
                const Column* c = ar.funcs[j] == OXB_AGG_COUNT_STAR ? nullptr : &ar.probe->cols[ar.columns[j]];
                if (ar.funcs[j] != OXB_AGG_COUNT_STAR && c->type != kInt64 && c->type != kFloat64 && c->type != kInt32) ok = false;
                funcs.push_back(ar.funcs[j]);
                inputs.push_back(AggInputCol{c, 0});
            }
            if (ok) {
                AggPlan pl = plan_aggregate(funcs, inputs, ar.build->cols[ar.group_column].type);
                DevPredicate pr = make_predicate(*ar.probe, ar.leaves, ar.nleaves);
                const Column& pk = ar.probe->cols[ar.probe_key];
                int x0, x1;
                ok = (pk.type == kInt64 || pk.type == kInt32) && lean_shape(pl.P, pr, pk.validity, &x0, &x1);
                if (ok && !idx.empty()) ok = x0 == la0 && x1 == la1 && pl.P.narrays == plans[0].P.narrays;
                if (ok) {
                    if (idx.empty()) {
                        la0 = x0;
                        la1 = x1;
                    }
                    idx.push_back(r);
                    plans.push_back(pl);
                    preds.push_back(pr);
                }
            }
        }
        std::vector<bool> shared(nall, false);
        if (idx.size() > 1)
            for (int r : idx) shared[r] = true;
        for (int r = 0; r < nall; r++)
            if (!shared[r]) res[r] = join_aggregate(s, b, all[r]);
        if (idx.size() <= 1) return res;
        std::vector<oxb_join_aggregate_args> a;
        for (int r : idx) a.push_back(all[r]);
        const int n = (int)a.size();
        std::vector<oxb_batch*> out(n, nullptr);
        auto alone = [&](int q) { out[q] = join_aggregate(s, b, a[q]); };
        auto finish = [&]() {
            for (int q = 0; q < n; q++) {
                res[idx[q]] = out[q];
                out[q] = nullptr;
            }
            return res;
        };
        const oxb_join_aggregate_args& a0 = a[0];
        const Column* gk = &a0.build->cols[a0.group_column];
        AggPlan plan;
        DevPredicate pred{};
        try {
        plan = plans[0];
        pred = preds[0];
        AggProgram& P = plan.P;
        const JoinTableDev jt = a0.table->t;
        const long long build_rows = a0.build->rows;
        // The group key's sample (build side) and the Float64 inputs' largest
        // values over every request, in one round trip.
        unsigned long long h[3 + kMaxAccs] = {0, (unsigned long long)LLONG_MAX, (unsigned long long)LLONG_MIN};
        const long long samples = build_rows < 8192 ? build_rows : 8192;
        if (samples > 0) {
            const unsigned int tcap = 16384;
            Scratch<long long> t(s, tcap);
            Scratch<unsigned long long> outs(s, 3 + kMaxAccs);
            OXB_CUDA(cudaMemcpyAsync(outs.get(), h, sizeof h, cudaMemcpyHostToDevice, s->stream));
            note_launch(), fill_i64_kernel<<<16, 256, 0, s->stream>>>(t.get(), tcap, kEmptyKey);
            AggKey sk{gk->values, gk->validity, gk->type, 0};
            note_launch(), agg_sample_kernel<<<grid_for(b, samples, 256, 2), 256, 0, s->stream>>>(sk, build_rows, samples,
                                                                                                t.get(), tcap, outs.get());
            for (int r = 0; r < n; r++) {
                const long long nr = a[r].probe->rows, fs = nr < 8192 ? nr : 8192;
                for (int j = 0; j < P.nacc && fs > 0; j++)
                    if (plans[r].P.acc[j].kind == kAccSumF64 && plans[r].P.acc[j].in_type == kFloat64)
                        note_launch(), f64_absmax_sample_kernel<<<grid_for(b, fs, 256, 2), 256, 0, s->stream>>>(
                            (const double*)plans[r].P.acc[j].values, plans[r].P.acc[j].validity, nr, fs, outs.get() + 3 + j);
            }
            OXB_CUDA(cudaGetLastError());
            OXB_CUDA(cudaMemcpyAsync(h, outs.get(), sizeof h, cudaMemcpyDeviceToHost, s->stream));
            OXB_CUDA(cudaStreamSynchronize(s->stream));
        }
        const long long d = (long long)h[0];
        const unsigned long long span = d > 0 ? (unsigned long long)(long long)h[2] - (unsigned long long)(long long)h[1] : ~0ull;
        if (d == 0 || span >= 4096ull || fused_smem_bytes((int)span + 1, P.narrays) > 48 * 1024) {
            for (int r = 0; r < n; r++) alone(r);
            return finish();
        }
        const long long full = build_rows < 1 ? 1 : build_rows;
        const unsigned int cap = d * 8 <= samples ? next_pow2(std::min<long long>(2 * full, 64ll * d + 4096), 4096)
                                                  : next_pow2(2 * full, 4096);
        const int S = (int)span + 1;
        const long long direct_lo = (long long)h[1];
        // Fixed-point windows (the widest any request needs), as run_aggregate places them.
        int fix_lo[kMaxAccs];
        for (int j = 0; j < P.nacc; j++) {
            fix_lo[j] = INT_MIN;
            if (P.acc[j].kind != kAccSumF64 || P.acc[j].in_type != kFloat64 || h[3 + j] == 0) continue;
            int e = 0;
            std::frexp(as_f64_host(h[3 + j]), &e);
            const int lo = e + 1 - 63;
            if (lo >= -900 && lo <= 800) fix_lo[j] = lo;
        }
        P.smem_slots = S;
        P.wslots = 0;
        P.direct = 1;
        P.direct_lo = direct_lo;
        P.capacity = cap;
        P.probe_limit = kMaxInsertProbes;
        P.stride = (long long)cap + 2;
        for (int j = 0; j < P.nacc; j++) {
            P.acc[j].fix = fix_lo[j] != INT_MIN;
            P.acc[j].fix_lo = P.acc[j].fix ? fix_lo[j] : 0;
        }
        // The probe table, once for every request.
        AggKey k{gk->values, gk->validity, gk->type, 1};
        FusedTab ft{};
        AllocRef fs;
        const unsigned long long key_span = (unsigned long long)jt.key_hi - (unsigned long long)jt.key_lo;
        const bool dense = jt.key_lo <= jt.key_hi && key_span < (1ull << 26) && (long long)key_span < 4 * jt.ndistinct + 4096;
        const int fgrid = grid_for(b, jt.capacity, 256, 8);
        if (dense) {
            ft.dense_lo = jt.key_lo;
            ft.dense_n = key_span + 1;
            fs = dev_alloc(s, (size_t)ft.dense_n * 4, false);
            OXB_CUDA(cudaMemsetAsync(fs->ptr, 0xff, (size_t)ft.dense_n * 4, s->stream));
            ft.dense = (const int*)fs->ptr;
            note_launch(), fuse_dense_kernel<<<fgrid, 256, 0, s->stream>>>(jt, k, direct_lo, S, (int*)fs->ptr, ft.dense_lo);
        } else {
            fs = dev_alloc(s, (size_t)jt.capacity * sizeof(FusedSlot), false);
            ft.slots = (const FusedSlot*)fs->ptr;
            note_launch(), fuse_table_kernel<<<fgrid, 256, 0, s->stream>>>(jt, k, direct_lo, S, (FusedSlot*)fs->ptr);
        }
        // Each request's HBM table and its work.
        std::vector<AllocRef> keep;
        std::vector<LeanReq> hreq(n);
        std::vector<AggProgram> Pr(n, P);
        Scratch<unsigned int> status(s, n, true);
        long long ntiles = 0;
        for (int r = 0; r < n; r++) {
            AllocRef km = dev_alloc(s, (size_t)cap * 8, false);
            AllocRef am = dev_alloc(s, (size_t)P.narrays * P.stride * 8, false);
            keep.push_back(km);
            keep.push_back(am);
            Pr[r].keys = (long long*)km->ptr;
            Pr[r].arr = (unsigned long long*)am->ptr;
            Pr[r].status = status.get() + r;
            note_launch(), agg_init_kernel<<<grid_for(b, (long long)P.narrays * P.stride, 256, 8), 256, 0, s->stream>>>(Pr[r]);
            LeanReq& q = hreq[r];
            const oxb_join_aggregate_args& ar = a[r];
            q.cols.pk = ar.probe->cols[ar.probe_key].values;
            for (int l = 0; l < 2; l++) {
                q.cols.leaf[l] = l < ar.nleaves ? preds[r].leaves[l].values : nullptr;
                q.cols.lit[l] = l < ar.nleaves ? preds[r].leaves[l].lit : 0;
                q.cols.acc[l] = l < plans[r].P.nacc ? plans[r].P.acc[l].values : nullptr;
            }
            q.n = ar.probe->rows;
            q.tile0 = ntiles;
            ntiles += (q.n + kLeanTile - 1) / kLeanTile;
            q.keys = Pr[r].keys;
            q.arr = Pr[r].arr;
            q.status = Pr[r].status;
        }
        Scratch<LeanReq> dreq(s, n);
        Scratch<unsigned long long> queue(s, 1, true);
        OXB_CUDA(cudaMemcpyAsync(dreq.get(), hreq.data(), n * sizeof(LeanReq), cudaMemcpyHostToDevice, s->stream));
        LeanPlan L = lean_plan(P, pred);
        L.acc_leaf[0] = L.acc_leaf[1] = -1;  // the requests' columns differ
        LeanMultiKernel kern = lean_multi_kernel_for(la0, la1, dense);
        const size_t smem = fused_smem_bytes(S, P.narrays);
        set_smem(kern, smem);
        {
            KernelTimer timer(b, s, dense ? "agg_join_kernel<fused-dense,lean,many>" : "agg_join_kernel<fused,lean,many>");
            timer.begin();
            if (ntiles > 0)
                note_launch(), kern<<<(unsigned)resident_grid(b, kern, smem, ntiles * kFusedThreads), kFusedThreads, smem,
                                      s->stream>>>(P, pred, L, k, a0.probe->cols[a0.probe_key].type, jt, ft, dreq.get(), n,
                                                   ntiles, queue.get());
            timer.end();
        }
        OXB_CUDA(cudaGetLastError());
        for (int r = 0; r < n; r++) {
            out[r] = emit_groups(s, b, plans[r], Pr[r], cap, status.get() + r, true);
            if (!out[r]) alone(r);  // its table overflowed: alone, with its own retry
        }
        return finish();
        } catch (...) {
            for (oxb_batch* x : out) delete x;
            throw;
        }
    } catch (...) {
        for (oxb_batch* x : res) delete x;
        throw;
    }
}


}  // namespace oxb
