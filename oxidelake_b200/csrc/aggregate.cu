// Grouped SUM / COUNT / MIN / MAX / AVG / COUNT(*) over one integer key
// (GpuBackend::aggregate, crates/oxidelake-device/src/backend.rs:166;
// semantics cpu/kernels.rs:478-818), and the fused inner-join probe ->
// WHERE -> GROUP BY form that runs a whole join + aggregate query in one
// pass over the probe side.
//
// One open-addressing table in HBM holds the groups: a key array (empty =
// kEmptyKey, claimed by one 64-bit CAS, so no publication wait is needed)
// and structure-of-arrays accumulators beside it.  Each CTA first folds rows
// into a private table in shared memory (bounded probing, half-full cap)
// and merges it into the HBM table when its rows are done; rows whose key
// does not fit the private table go straight to HBM.  Low-cardinality
// queries therefore touch HBM only for their input columns.
//
// Float64 SUM/AVG: every atomicAdd returns the old sum, so the rounding
// error of that very addition is recovered exactly (TwoSum) and accumulated
// in a compensation array; the result is sum + compensation.  This keeps the
// error to O(eps) relative independently of the order atomics land in.
// Int64 SUM wraps (unsigned add), MIN/MAX over Float64 follow totalOrder via
// integer keys, exactly as the reference.
#include "internal.h"

namespace oxb {

namespace {

constexpr int kMaxOps = OXB_MAX_AGGREGATES;
constexpr int kMaxArrays = 1 + 3 * kMaxOps;
constexpr int kThreads = 256;
constexpr int kSmemProbes = 16;

enum : unsigned char { kInitZero = 0, kInitMax = 1, kInitMin = 2 };
enum : unsigned char { kMergeAddU64 = 0, kMergeAddF64Comp = 1, kMergeAddF64 = 2, kMergeMin = 3, kMergeMax = 4 };

struct DevAggOp {
    const void* values;
    const uint8_t* validity;
    int func;
    int in_type;
    int side;  // 0: the input (probe) row, 1: the build row
    int a0, a1, a2;
};

struct AggProgram {
    int nops;
    int narrays;
    DevAggOp ops[kMaxOps];
    unsigned char init[kMaxArrays];
    unsigned char merge[kMaxArrays];
    long long* keys;           // capacity entries
    unsigned long long* acc;   // narrays * stride entries
    long long stride;          // capacity + 2: [capacity] NULL group, [capacity+1] key == kEmptyKey
    unsigned int capacity;
    int smem_slots;            // power of two, 0 = no private table
    unsigned int* status;
    unsigned long long* fill;      // keys placed in the HBM table
    unsigned long long fill_limit; // 3/4 of capacity: no insert beyond it
};

struct AggKey {
    const void* values;
    const uint8_t* validity;
    int type;
    int side;
};

__device__ __forceinline__ void add_f64_comp(double* sum, double* comp, double x) {
    double old = atomicAdd(sum, x);
    double s = __dadd_rn(old, x);
    if (isfinite(s)) {
        double bp = __dsub_rn(s, old);
        double e = __dadd_rn(__dsub_rn(old, __dsub_rn(s, bp)), __dsub_rn(x, bp));
        if (e != 0.0) atomicAdd(comp, e);
    }
}

__device__ __forceinline__ long long load_int(const void* v, int type, long long row) {
    return type == kInt64 ? __ldg((const long long*)v + row) : (long long)__ldg((const int*)v + row);
}

// Folds one row into accumulators at `slot` (arrays `stride` entries apart).
__device__ __forceinline__ void agg_apply(const AggProgram& P, unsigned long long* acc, long long stride,
                                          long long slot, long long row_p, long long row_b) {
    atomicAdd(&acc[slot], 1ull);  // array 0: rows of the group
    for (int j = 0; j < P.nops; j++) {
        const DevAggOp& op = P.ops[j];
        if (op.func == OXB_AGG_COUNT_STAR) continue;
        const long long row = op.side ? row_b : row_p;
        if (!valid_at(op.validity, row)) continue;
        unsigned long long* a0 = acc + op.a0 * stride + slot;
        switch (op.func) {
            case OXB_AGG_COUNT:
                if (op.a0) atomicAdd(a0, 1ull);
                continue;
            case OXB_AGG_SUM:
                if (op.in_type == kFloat64) {
                    add_f64_comp((double*)a0, (double*)(acc + op.a1 * stride + slot),
                                 __ldg((const double*)op.values + row));
                    if (op.a2) atomicAdd(acc + op.a2 * stride + slot, 1ull);
                } else {
                    atomicAdd(a0, (unsigned long long)load_int(op.values, op.in_type, row));
                    if (op.a1) atomicAdd(acc + op.a1 * stride + slot, 1ull);
                }
                continue;
            case OXB_AGG_AVG: {
                double x = op.in_type == kFloat64 ? __ldg((const double*)op.values + row)
                                                  : (double)load_int(op.values, op.in_type, row);
                add_f64_comp((double*)a0, (double*)(acc + op.a1 * stride + slot), x);
                if (op.a2) atomicAdd(acc + op.a2 * stride + slot, 1ull);
                continue;
            }
            case OXB_AGG_MIN:
            case OXB_AGG_MAX: {
                long long k = op.in_type == kFloat64 ? total_order_key(__ldg((const double*)op.values + row))
                                                     : load_int(op.values, op.in_type, row);
                if (op.func == OXB_AGG_MIN) atomicMin((long long*)a0, k);
                else atomicMax((long long*)a0, k);
                if (op.a1) atomicAdd(acc + op.a1 * stride + slot, 1ull);
                continue;
            }
            default: continue;
        }
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
            // Past 3/4 load a new key is refused (the host retries with a
            // table sized for every row), which keeps every probe sequence short.
            if (__ldcg(P.fill) >= P.fill_limit) break;
            unsigned long long old = atomicCAS((unsigned long long*)&P.keys[h], (unsigned long long)kEmptyKey,
                                               (unsigned long long)key);
            if (old == (unsigned long long)kEmptyKey) {
                atomicAdd(P.fill, 1ull);
                return h;
            }
            if (old == (unsigned long long)key) return h;
        }
        h = (h + 1u) & (P.capacity - 1u);
    }
    atomicOr(P.status, kStatusTableFull);
    return -1;
}

// The private slot of a key, -1 when it is not there and cannot be added.
__device__ __forceinline__ int smem_slot(long long key, long long* s_keys, int S, int* s_fill) {
    unsigned int h = (unsigned int)(fmix64((unsigned long long)key) & (unsigned)(S - 1));
    for (int p = 0; p < kSmemProbes; p++) {
        long long k = ((volatile long long*)s_keys)[h];
        if (k == key) return (int)h;
        if (k == kEmptyKey) {
            if (*(volatile int*)s_fill >= S / 2) return -1;
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
    return -1;
}

__device__ __forceinline__ void fold_row(const AggProgram& P, long long* s_keys, unsigned long long* s_acc,
                                         int* s_fill, bool kvalid, long long key, long long row_p,
                                         long long row_b) {
    const int S = P.smem_slots;
    if (S > 0 && kvalid && key != kEmptyKey) {
        int ls = smem_slot(key, s_keys, S, s_fill);
        if (ls >= 0) {
            agg_apply(P, s_acc, S, ls, row_p, row_b);
            return;
        }
    }
    long long g = global_slot(P, kvalid, key);
    if (g >= 0) agg_apply(P, P.acc, P.stride, g, row_p, row_b);
}

__device__ __forceinline__ unsigned long long init_value(unsigned char tag) {
    return tag == kInitMax ? 0x7fffffffffffffffull : (tag == kInitMin ? 0x8000000000000000ull : 0ull);
}

__device__ void smem_init(const AggProgram& P, long long* s_keys, unsigned long long* s_acc, int* s_fill) {
    const int S = P.smem_slots;
    for (int i = threadIdx.x; i < S; i += blockDim.x) s_keys[i] = kEmptyKey;
    for (int i = threadIdx.x; i < S * P.narrays; i += blockDim.x) s_acc[i] = init_value(P.init[i / S]);
    if (threadIdx.x == 0) *s_fill = 0;
    __syncthreads();
}

// Merges the private table into HBM.
__device__ void smem_flush(const AggProgram& P, long long* s_keys, unsigned long long* s_acc) {
    __syncthreads();
    const int S = P.smem_slots;
    for (int i = threadIdx.x; i < S; i += blockDim.x) {
        long long key = s_keys[i];
        if (key == kEmptyKey) continue;
        long long g = global_slot(P, true, key);
        if (g < 0) continue;
        for (int a = 0; a < P.narrays; a++) {
            unsigned long long v = s_acc[a * S + i];
            unsigned long long* dst = P.acc + a * P.stride + g;
            switch (P.merge[a]) {
                case kMergeAddU64:
                    if (v) atomicAdd(dst, v);
                    break;
                case kMergeAddF64Comp:
                    add_f64_comp((double*)dst, (double*)(dst + P.stride), __longlong_as_double((long long)v));
                    break;
                case kMergeAddF64: {
                    double x = __longlong_as_double((long long)v);
                    if (x != 0.0) atomicAdd((double*)dst, x);
                    break;
                }
                case kMergeMin:
                    if ((long long)v != 0x7fffffffffffffffll) atomicMin((long long*)dst, (long long)v);
                    break;
                default:
                    if ((long long)v != (long long)0x8000000000000000ull) atomicMax((long long*)dst, (long long)v);
                    break;
            }
        }
    }
}

__global__ void __launch_bounds__(kThreads) agg_rows_kernel(AggProgram P, DevPredicate pred, AggKey key,
                                                            long long n) {
    extern __shared__ __align__(16) unsigned char smem[];
    long long* s_keys = (long long*)smem;
    unsigned long long* s_acc = (unsigned long long*)(s_keys + P.smem_slots);
    int* s_fill = (int*)(s_acc + (long long)P.smem_slots * P.narrays);
    if (P.smem_slots) smem_init(P, s_keys, s_acc, s_fill);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (pred.nleaves && !predicate_holds(pred, i)) continue;
        bool kv = valid_at(key.validity, i);
        long long k = kv ? load_int(key.values, key.type, i) : 0;
        fold_row(P, s_keys, s_acc, s_fill, kv, k, i, 0);
    }
    if (P.smem_slots) smem_flush(P, s_keys, s_acc);
}

__device__ __forceinline__ bool jt_lookup(const JoinTableDev& t, long long key, unsigned int* start,
                                          unsigned int* count) {
    if (key == kEmptyKey) {
        *start = t.special_start;
        *count = t.special_count;
        return *count > 0;
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

// probe JOIN build ON key WHERE <probe leaves> GROUP BY <key of either side>:
// one thread per probe row walks its key's run in build order.
__global__ void __launch_bounds__(kThreads) agg_join_kernel(AggProgram P, DevPredicate pred, AggKey gkey,
                                                            const void* __restrict__ pk, const uint8_t* __restrict__ pkv,
                                                            int pk_type, JoinTableDev jt, long long n) {
    extern __shared__ __align__(16) unsigned char smem[];
    long long* s_keys = (long long*)smem;
    unsigned long long* s_acc = (unsigned long long*)(s_keys + P.smem_slots);
    int* s_fill = (int*)(s_acc + (long long)P.smem_slots * P.narrays);
    if (P.smem_slots) smem_init(P, s_keys, s_acc, s_fill);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (pred.nleaves && !predicate_holds(pred, i)) continue;
        if (!valid_at(pkv, i)) continue;
        unsigned int start, count;
        if (!jt_lookup(jt, load_int(pk, pk_type, i), &start, &count)) continue;
        for (unsigned int m = 0; m < count; m++) {
            long long b = jt.rows[start + m];
            long long grow = gkey.side ? b : i;
            bool kv = valid_at(gkey.validity, grow);
            long long k = kv ? load_int(gkey.values, gkey.type, grow) : 0;
            fold_row(P, s_keys, s_acc, s_fill, kv, k, i, b);
        }
    }
    if (P.smem_slots) smem_flush(P, s_keys, s_acc);
}

__global__ void agg_init_kernel(AggProgram P) {
    const long long total = (long long)P.narrays * P.stride;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x)
        P.acc[i] = init_value(P.init[i / P.stride]);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P.capacity;
         i += (long long)gridDim.x * blockDim.x)
        P.keys[i] = kEmptyKey;
}

// Occupied slots (the NULL group aside) as 0/1 flags; also the key range.
__global__ void agg_flags_kernel(AggProgram P, unsigned int* __restrict__ flags,
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
            occ = P.acc[s] > 0;  // rows of the kEmptyKey group
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

__global__ void agg_compact_kernel(AggProgram P, const unsigned int* __restrict__ flags,
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
    OutCol cols[kMaxOps];
};

// One output row per thread: the group at sorted position r, the NULL group last.
__global__ void agg_emit_kernel(AggProgram P, AggOutput O, const unsigned long long* __restrict__ skeys,
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
        const unsigned long long* acc = P.acc;
        const long long st = P.stride;
        for (int j = 0; j < P.nops; j++) {
            const DevAggOp& op = P.ops[j];
            bool valid = true;
            if (live) {
                unsigned long long a0 = acc[op.a0 * st + slot];
                switch (op.func) {
                    case OXB_AGG_COUNT:
                    case OXB_AGG_COUNT_STAR:
                        ((unsigned long long*)O.cols[j].values)[r] = a0;
                        break;
                    case OXB_AGG_SUM:
                        if (op.in_type == kFloat64) {
                            double s = __longlong_as_double((long long)a0);
                            double c = __longlong_as_double((long long)acc[op.a1 * st + slot]);
                            ((double*)O.cols[j].values)[r] = isfinite(s) ? __dadd_rn(s, c) : s;
                            valid = acc[op.a2 * st + slot] > 0;
                        } else {
                            ((unsigned long long*)O.cols[j].values)[r] = a0;
                            valid = acc[op.a1 * st + slot] > 0;
                        }
                        break;
                    case OXB_AGG_AVG: {
                        double s = __longlong_as_double((long long)a0);
                        double c = __longlong_as_double((long long)acc[op.a1 * st + slot]);
                        unsigned long long cnt = acc[op.a2 * st + slot];
                        double t = isfinite(s) ? __dadd_rn(s, c) : s;
                        ((double*)O.cols[j].values)[r] = cnt ? __ddiv_rn(t, (double)cnt) : 0.0;
                        valid = cnt > 0;
                        break;
                    }
                    default: {
                        valid = acc[op.a1 * st + slot] > 0;
                        long long k = (long long)a0;
                        if (op.in_type == kFloat64)
                            ((double*)O.cols[j].values)[r] = valid ? from_total_order_key(k) : 0.0;
                        else if (op.in_type == kInt64)
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

// Distinct keys among a strided sample of rows (an estimate of the table size).
__global__ void agg_sample_kernel(AggKey key, long long n, long long samples, long long* __restrict__ table,
                                  unsigned int tcap, unsigned int* __restrict__ distinct) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < samples;
         i += (long long)gridDim.x * blockDim.x) {
        long long row = (long long)((double)i * (double)n / (double)samples);
        if (row >= n) row = n - 1;
        if (!valid_at(key.validity, row)) continue;
        long long k = load_int(key.values, key.type, row);
        if (k == kEmptyKey) continue;
        unsigned int h = (unsigned int)(fmix64((unsigned long long)k) & (tcap - 1u));
        for (unsigned int p = 0; p < tcap; p++) {
            unsigned long long old =
                atomicCAS((unsigned long long*)&table[h], (unsigned long long)kEmptyKey, (unsigned long long)k);
            if (old == (unsigned long long)kEmptyKey) {
                atomicAdd(distinct, 1u);
                break;
            }
            if ((long long)old == k) break;
            h = (h + 1u) & (tcap - 1u);
        }
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

// One aggregate as the kernels run it: a column or the build side.
struct AggInputCol {
    const Column* col;  // null for COUNT(*)
    int side;
};

struct AggPlan {
    AggProgram P{};
    std::vector<int> out_types;
    int key_type = kInt64;
};

AggPlan plan_aggregate(const std::vector<int>& funcs, const std::vector<AggInputCol>& inputs, int key_type) {
    AggPlan plan;
    AggProgram& P = plan.P;
    P.nops = (int)funcs.size();
    int na = 1;  // array 0: rows per group
    P.init[0] = kInitZero;
    P.merge[0] = kMergeAddU64;
    auto add_array = [&](unsigned char init, unsigned char merge) {
        P.init[na] = init;
        P.merge[na] = merge;
        return na++;
    };
    for (int j = 0; j < P.nops; j++) {
        DevAggOp& op = P.ops[j];
        op.func = funcs[j];
        const Column* c = inputs[j].col;
        op.side = inputs[j].side;
        op.values = c ? c->values : nullptr;
        op.validity = c ? c->validity : nullptr;
        op.in_type = c ? c->type : kInt64;
        const bool nullable = c && c->validity;
        auto nn = [&]() { return nullable ? add_array(kInitZero, kMergeAddU64) : 0; };
        int out_type = kInt64;
        switch (op.func) {
            case OXB_AGG_COUNT_STAR:
                op.a0 = 0;
                break;
            case OXB_AGG_COUNT:
                op.a0 = nn();
                break;
            case OXB_AGG_SUM:
                if (op.in_type == kFloat64) {
                    op.a0 = add_array(kInitZero, kMergeAddF64Comp);
                    op.a1 = add_array(kInitZero, kMergeAddF64);
                    op.a2 = nn();
                    out_type = kFloat64;
                } else {
                    op.a0 = add_array(kInitZero, kMergeAddU64);
                    op.a1 = nn();
                }
                break;
            case OXB_AGG_AVG:
                op.a0 = add_array(kInitZero, kMergeAddF64Comp);
                op.a1 = add_array(kInitZero, kMergeAddF64);
                op.a2 = nn();
                out_type = kFloat64;
                break;
            case OXB_AGG_MIN:
                op.a0 = add_array(kInitMax, kMergeMin);
                op.a1 = nn();
                out_type = op.in_type;
                break;
            case OXB_AGG_MAX:
                op.a0 = add_array(kInitMin, kMergeMax);
                op.a1 = nn();
                out_type = op.in_type;
                break;
            default:
                fail(OXB_PLAN, "unknown aggregate function " + std::to_string(op.func));
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

// Runs the planned aggregation kernel(s) and emits the sorted output batch.
template <typename Launch>
oxb_batch* run_aggregate(const StreamRef& s, const Backend& b, AggPlan& plan, const AggKey& key_for_sample,
                         long long sample_rows, long long max_groups, const char* kernel_name, Launch&& launch) {
    AggProgram& P = plan.P;
    // Size the table: a strided sample decides between a small table
    // (keys repeat) and one that holds every row's key.
    unsigned int cap;
    {
        long long samples = sample_rows < 8192 ? sample_rows : 8192;
        unsigned int d = 0;
        if (samples > 0) {
            const unsigned int tcap = 16384;
            Scratch<long long> t(s, tcap);
            Scratch<unsigned int> dist(s, 1, true);
            note_launch(), fill_i64_kernel<<<16, 256, 0, s->stream>>>(t.get(), tcap, kEmptyKey);
            note_launch(), agg_sample_kernel<<<grid_for(b, samples, 256, 2), 256, 0, s->stream>>>(key_for_sample, sample_rows,
                                                                                   samples, t.get(), tcap, dist.get());
            OXB_CUDA(cudaGetLastError());
            OXB_CUDA(cudaMemcpyAsync(&d, dist.get(), 4, cudaMemcpyDeviceToHost, s->stream));
            OXB_CUDA(cudaStreamSynchronize(s->stream));
        }
        long long full = max_groups < 1 ? 1 : max_groups;
        if ((long long)d * 8 <= samples) cap = next_pow2(std::min<long long>(2 * full, 64ll * d + 4096), 4096);
        else cap = next_pow2(2 * full, 4096);
    }
    // Private table size: as many slots as fit in 48 KB (power of two, <= 2048).
    const long long per_slot = 8ll * (1 + P.narrays);
    int S = 2048;
    while (S > 0 && S * per_slot + 16 > 48 * 1024) S >>= 1;
    if (S < 64) S = 0;
    P.smem_slots = S;
    const size_t smem = S ? (size_t)S * per_slot + 16 : 0;

    for (int attempt = 0; attempt < 2; attempt++) {
        P.capacity = cap;
        P.stride = (long long)cap + 2;
        AllocRef keys_mem = dev_alloc(s, (size_t)cap * 8, false);
        AllocRef acc_mem = dev_alloc(s, (size_t)P.narrays * P.stride * 8, false);
        Scratch<unsigned int> status(s, 1, true);
        Scratch<unsigned long long> fill(s, 1, true);
        P.keys = (long long*)keys_mem->ptr;
        P.acc = (unsigned long long*)acc_mem->ptr;
        P.status = status.get();
        P.fill = fill.get();
        P.fill_limit = (unsigned long long)cap / 4 * 3;
        note_launch(), agg_init_kernel<<<grid_for(b, (long long)P.narrays * P.stride, 256, 8), 256, 0, s->stream>>>(P);
        OXB_CUDA(cudaGetLastError());
        {
            KernelTimer timer(b, s, kernel_name);
            timer.begin();
            launch(P, smem);
            timer.end();
        }
        OXB_CUDA(cudaGetLastError());

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
        OXB_CUDA(cudaMemcpyAsync(&h.null_rows, P.acc + cap, 8, cudaMemcpyDeviceToHost, s->stream));
        OXB_CUDA(cudaMemcpyAsync(&h.status, status.get(), 4, cudaMemcpyDeviceToHost, s->stream));
        OXB_CUDA(cudaStreamSynchronize(s->stream));
        if ((h.status & kStatusTableFull) && attempt == 0) {
            cap = next_pow2(2 * (max_groups < 1 ? 1 : max_groups), 4096);
            continue;  // the small table overflowed: rerun with room for every row
        }
        check_status_word(h.status, "aggregate");

        const long long G = (long long)h.G;
        const bool has_null = h.null_rows > 0;
        const long long rows = G + (has_null ? 1 : 0);
        Scratch<unsigned long long> skeys(s, G + 1);
        Scratch<unsigned int> sslots(s, G + 1);
        unsigned long long lo = G > 0 ? h.lo : 0;
        if (G > 0) {
            note_launch(), agg_compact_kernel<<<grid_for(b, m, 256, 8), 256, 0, s->stream>>>(P, flags.get(), pos.get(), lo,
                                                                               skeys.get(), sslots.get());
            OXB_CUDA(cudaGetLastError());
            unsigned long long span = h.hi - h.lo;
            int bits = 0;
            while (bits < 64 && (span >> bits) != 0) bits++;
            radix_sort_pairs(s, b, skeys.get(), sslots.get(), G, bits);
        }

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
        for (int j = 0; j < P.nops; j++) {
            const int f = P.ops[j].func;
            const bool nullable = !(f == OXB_AGG_COUNT || f == OXB_AGG_COUNT_STAR);
            out->cols.push_back(make_col(plan.out_types[j], nullable));
            O.cols[j] = OutCol{out->cols.back().values, (unsigned int*)out->cols.back().validity};
        }
        if (rows > 0) {
            note_launch(), agg_emit_kernel<<<grid_for(b, rows, 256, 8), 256, 0, s->stream>>>(P, O, skeys.get(), sslots.get(), lo, G,
                                                                               rows);
            OXB_CUDA(cudaGetLastError());
            OXB_CUDA(cudaStreamSynchronize(s->stream));
        }
        return out.release();
    }
    fail(OXB_TABLE_FULL, "aggregate hash table full after a retry");
}

}  // namespace

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
    if (spec.naggregates < 0 || spec.naggregates > kMaxOps) fail(OXB_UNSUPPORTED, "too many aggregates");
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
    return run_aggregate(s, b, plan, k, n, n, "agg_rows_kernel", [&](AggProgram& P, size_t smem) {
        if (n == 0) return;
        if (smem > 48 * 1024)
            OXB_CUDA(cudaFuncSetAttribute(agg_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        note_launch(), agg_rows_kernel<<<grid_for(b, n, kThreads, 4), kThreads, smem, s->stream>>>(P, pred, k, n);
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
        const oxb_batch& bt = side ? build : probe;
        if (side != 0 && side != 1) fail(OXB_PLAN, "side must be 0 (probe) or 1 (build)");
        if (col < 0 || col >= (int)bt.cols.size()) fail(OXB_PLAN, "column index " + std::to_string(col) + " out of range");
        return &bt.cols[col];
    };
    const Column* gk = side_col(a.group_side, a.group_column);
    if (gk->type != kInt64 && gk->type != kInt32) fail(OXB_UNSUPPORTED, "group key must be Int64 or Int32");
    if (a.naggregates < 0 || a.naggregates > kMaxOps) fail(OXB_UNSUPPORTED, "too many aggregates");
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
    const long long max_groups = a.group_side ? build.rows : probe.rows;
    AggKey sample_key{gk->values, gk->validity, gk->type, 0};
    const JoinTableDev jt = a.table->t;
    return run_aggregate(s, b, plan, sample_key, group_rows, max_groups, "agg_join_kernel", [&](AggProgram& P, size_t smem) {
        if (n == 0) return;
        if (smem > 48 * 1024)
            OXB_CUDA(cudaFuncSetAttribute(agg_join_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        note_launch(), agg_join_kernel<<<grid_for(b, n, kThreads, 4), kThreads, smem, s->stream>>>(P, pred, k, pk.values, pk.validity,
                                                                                    pk.type, jt, n);
    });
}

}  // namespace oxb
