// Device-side helpers shared by every kernel of liboxb200.
//
// Layout of a column in HBM (crates/oxidelake-device/src/columns.rs:28-40):
// values packed from row 0; an optional LSB-first validity bitmap, bit 0 =
// row 0, a null pointer meaning every row is valid.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace oxb {

// Bits of the per-call device status word (read back by the host after the
// call's kernels; mapped to oxb_status).
constexpr uint32_t kStatusTableFull = 1u;  // a hash table had no free slot
constexpr uint32_t kStatusTimeout = 2u;    // a bounded wait gave up
constexpr uint32_t kStatusBounds = 4u;     // an index failed its bounds check

// Type tags, equal to oxb_type.
constexpr int kInt64 = 1;
constexpr int kFloat64 = 2;
constexpr int kInt32 = 3;
constexpr int kFloat32 = 4;
constexpr int kVectorF32 = 5;

// The slot key that marks an empty hash-table slot.  A real key equal to it
// is kept in a dedicated side slot instead (see hash tables below).
constexpr long long kEmptyKey = (long long)0x8000000000000000ULL;

__host__ __device__ __forceinline__ int type_width(int type, int dim) {
    return type == kInt32 || type == kFloat32 ? 4 : (type == kVectorF32 ? 4 * dim : 8);
}

__device__ __forceinline__ bool valid_at(const uint8_t* __restrict__ v, long long i) {
    return v == nullptr || ((__ldg(v + (i >> 3)) >> (i & 7)) & 1);
}

// IEEE 754 totalOrder as a signed integer: comparing two keys as int64 is
// f64::total_cmp (cpu/kernels.rs:825-830).  Its own inverse.
__device__ __forceinline__ long long total_order_key(double x) {
    long long b = __double_as_longlong(x);
    return b ^ (long long)(((unsigned long long)(b >> 63)) >> 1);
}
__device__ __forceinline__ double from_total_order_key(long long k) {
    return __longlong_as_double(k ^ (long long)(((unsigned long long)(k >> 63)) >> 1));
}
// The order a Float64 filter compares in: -0.0 read as +0.0, then totalOrder
// (cpu/kernels.rs:62-69, 99-141).
__device__ __forceinline__ long long filter_order_key(double x) {
    long long b = __double_as_longlong(x);
    if (b == kEmptyKey) b = 0;  // -0.0 has the bit pattern 0x8000...
    return b ^ (long long)(((unsigned long long)(b >> 63)) >> 1);
}

// 64-bit finalizer (murmur3 fmix64) used to place keys in every device hash
// table of this library.
__host__ __device__ __forceinline__ unsigned long long fmix64(unsigned long long h) {
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdULL;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ULL;
    h ^= h >> 33;
    return h;
}

// One predicate leaf as kernels read it (a flattened oxb_leaf with the
// column's device pointers resolved on the host).
struct DevLeaf {
    const void* values;
    const uint8_t* validity;
    long long lit;   // int literal, or the filter order key of a Float64 literal
    int type;
    int op;
};

constexpr int kMaxLeaves = 64;

struct DevPredicate {
    int nleaves;
    DevLeaf leaves[kMaxLeaves];
};

__device__ __forceinline__ bool cmp_holds(int op, long long a, long long b) {
    switch (op) {
        case 0: return a == b;
        case 1: return a < b;
        case 2: return a <= b;
        case 3: return a > b;
        default: return a >= b;
    }
}

// Every leaf true at `row` (a NULL operand makes its leaf, so the row, fail).
__device__ __forceinline__ bool predicate_holds(const DevPredicate& p, long long row) {
    for (int l = 0; l < p.nleaves; l++) {
        const DevLeaf& lf = p.leaves[l];
        if (!valid_at(lf.validity, row)) return false;
        long long a;
        if (lf.type == kFloat64) a = filter_order_key(__ldg((const double*)lf.values + row));
        else if (lf.type == kInt64) a = __ldg((const long long*)lf.values + row);
        else a = (long long)__ldg((const int*)lf.values + row);
        if (!cmp_holds(lf.op, a, lf.lit)) return false;
    }
    return true;
}

// The predicate over RPT rows at once: bit r of the result is set when row
// base + r * stride (bit r of `live`) satisfies every leaf.  A leaf's type
// and comparison are dispatched once for the RPT rows, whose loads are
// issued together.
template <int RPT>
__device__ __forceinline__ unsigned predicate_mask(const DevPredicate& p, long long base, long long stride,
                                                   unsigned live) {
    for (int l = 0; l < p.nleaves && live; l++) {
        const DevLeaf& lf = p.leaves[l];
        long long a[RPT];
        if (lf.type == kFloat64) {
#pragma unroll
            for (int r = 0; r < RPT; r++)
                a[r] = (live >> r) & 1u ? filter_order_key(__ldcs((const double*)lf.values + base + r * stride)) : 0;
        } else if (lf.type == kInt64) {
#pragma unroll
            for (int r = 0; r < RPT; r++)
                a[r] = (live >> r) & 1u ? __ldcs((const long long*)lf.values + base + r * stride) : 0;
        } else {
#pragma unroll
            for (int r = 0; r < RPT; r++)
                a[r] = (live >> r) & 1u ? (long long)__ldcs((const int*)lf.values + base + r * stride) : 0;
        }
        const long long lit = lf.lit;
        unsigned m = 0;
        switch (lf.op) {
            case 0:
#pragma unroll
                for (int r = 0; r < RPT; r++) m |= (unsigned)(a[r] == lit) << r;
                break;
            case 1:
#pragma unroll
                for (int r = 0; r < RPT; r++) m |= (unsigned)(a[r] < lit) << r;
                break;
            case 2:
#pragma unroll
                for (int r = 0; r < RPT; r++) m |= (unsigned)(a[r] <= lit) << r;
                break;
            case 3:
#pragma unroll
                for (int r = 0; r < RPT; r++) m |= (unsigned)(a[r] > lit) << r;
                break;
            default:
#pragma unroll
                for (int r = 0; r < RPT; r++) m |= (unsigned)(a[r] >= lit) << r;
                break;
        }
        live &= m;
        if (lf.validity) {
#pragma unroll
            for (int r = 0; r < RPT; r++)
                if (((live >> r) & 1u) && !valid_at(lf.validity, base + r * stride)) live &= ~(1u << r);
        }
    }
    return live;
}

__device__ __forceinline__ long long load_key(const void* values, int type, long long row) {
    return type == kInt64 ? __ldg((const long long*)values + row)
                          : (long long)__ldg((const int*)values + row);
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace oxb
