// L2 / cosine distance between one query and a FixedSizeList<Float32>
// column (GpuBackend::vector_distance, crates/oxidelake-device/src/backend.rs:173).
//
// Bit-exact with cpu/kernels.rs:909-927: each row's sums are folded in index
// order from -0.0 with one correctly rounded IEEE operation per Rust
// operator (no fused multiply-add: __fmul_rn / __fadd_rn), then sqrt and
// divide correctly rounded.  One thread owns one row; a block stages 128 rows
// x 32 dimensions at a time through shared memory with coalesced loads, so
// the sequential per-row fold still reads HBM at full width.  When every row
// starts on a 16-byte boundary (dim a multiple of 4), the stages are a ring
// of kStages filled by 16-byte asynchronous copies (cp.async) several
// stages ahead of the fold; otherwise (or for dim < 32) one stage is loaded
// and folded at a time.
#include "async_copy.cuh"
#include "internal.h"

namespace oxb {

namespace {

constexpr int kRowsPerBlock = 128;

__global__ void __launch_bounds__(kRowsPerBlock) vector_distance_kernel(
    const float* __restrict__ vecs, const uint8_t* __restrict__ validity, long long n, int dim,
    const float* __restrict__ q, int metric, float* __restrict__ out) {
    extern __shared__ float smem[];
    const int C = dim <= 64 ? dim : 32;  // dimensions staged per round
    float* tile = smem;                   // kRowsPerBlock x (C + 1)
    float* qs = smem + kRowsPerBlock * (C + 1);
    // The query's own squared norm, folded in index order (cosine only).
    __shared__ float q_norm;
    if (threadIdx.x == 0 && metric == 1) {
        float sb = -0.0f;
        for (int k = 0; k < dim; k++) sb = __fadd_rn(sb, __fmul_rn(q[k], q[k]));
        q_norm = __fsqrt_rn(sb);
    }
    for (long long base = (long long)blockIdx.x * kRowsPerBlock; base < n;
         base += (long long)gridDim.x * kRowsPerBlock) {
        const long long row = base + threadIdx.x;
        float s0 = -0.0f, s1 = -0.0f;
        for (int c0 = 0; c0 < dim; c0 += C) {
            const int w = dim - c0 < C ? dim - c0 : C;
            __syncthreads();
            for (int idx = threadIdx.x; idx < kRowsPerBlock * C; idx += kRowsPerBlock) {
                const int r = idx / C, c = idx - r * C;
                float v = 0.0f;
                if (base + r < n && c < w) v = __ldg(vecs + (base + r) * (long long)dim + c0 + c);
                tile[r * (C + 1) + c] = v;
            }
            for (int c = threadIdx.x; c < w; c += kRowsPerBlock) qs[c] = q[c0 + c];
            __syncthreads();
            const float* my = tile + threadIdx.x * (C + 1);
            if (metric == 0) {
                for (int k = 0; k < w; k++) {
                    float d = __fsub_rn(my[k], qs[k]);
                    s0 = __fadd_rn(s0, __fmul_rn(d, d));
                }
            } else {
                for (int k = 0; k < w; k++) {
                    float a = my[k];
                    s0 = __fadd_rn(s0, __fmul_rn(a, qs[k]));
                    s1 = __fadd_rn(s1, __fmul_rn(a, a));
                }
            }
        }
        if (row < n) {
            float r;
            if (!valid_at(validity, row)) r = 0.0f;
            else if (metric == 0) r = __fsqrt_rn(s0);
            else {
                float na = __fsqrt_rn(s1), nb = q_norm;
                r = (na == 0.0f || nb == 0.0f) ? __int_as_float(0x7fc00000)
                                               : __fsub_rn(1.0f, __fdiv_rn(s0, __fmul_rn(na, nb)));
            }
            out[row] = r;
        }
    }
}

// ---- the pipelined form: dim % 4 == 0, 16-byte aligned rows ----------------
constexpr int kDimChunk = 32;                // dimensions a stage holds per row
constexpr int kRowStride = kDimChunk + 4;    // floats per staged row: 16-byte aligned, and a quarter-warp's
                                             // 16-byte reads of 8 rows cover all 32 banks
constexpr int kStages = 4;
constexpr int kStageFloats = kRowsPerBlock * kRowStride;

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__global__ void __launch_bounds__(kRowsPerBlock) vector_distance_async_kernel(
    const float* __restrict__ vecs, const uint8_t* __restrict__ validity, long long n, int dim,
    const float* __restrict__ q, int metric, float* __restrict__ out) {
    extern __shared__ __align__(16) float smem[];
    float* ring = smem;                        // kStages x kStageFloats
    float* qs = smem + kStages * kStageFloats;  // the whole query
    __shared__ float q_norm;
    for (int k = threadIdx.x; k < dim; k += blockDim.x) qs[k] = q[k];
    if (threadIdx.x == 0 && metric == 1) {
        float sb = -0.0f;
        for (int k = 0; k < dim; k++) sb = __fadd_rn(sb, __fmul_rn(q[k], q[k]));
        q_norm = __fsqrt_rn(sb);
    }
    const int nchunks = (dim + kDimChunk - 1) / kDimChunk;
    for (long long base = (long long)blockIdx.x * kRowsPerBlock; base < n;
         base += (long long)gridDim.x * kRowsPerBlock) {
        const int rows = n - base < kRowsPerBlock ? (int)(n - base) : kRowsPerBlock;
        // Chunk c of every row into stage c % kStages: 16-byte pieces, a
        // warp's 32 covering 4 rows x 128 contiguous bytes.
        auto issue = [&](int c) {
            if (c < nchunks) {
                const int c0 = c * kDimChunk;
                const int pieces = (dim - c0 < kDimChunk ? dim - c0 : kDimChunk) / 4;
                float* st = ring + (c % kStages) * kStageFloats;
                for (int idx = threadIdx.x; idx < kRowsPerBlock * (kDimChunk / 4); idx += blockDim.x) {
                    const int r = idx / (kDimChunk / 4), pc = idx % (kDimChunk / 4);
                    if (r < rows && pc < pieces)
                        cp_async16(st + r * kRowStride + pc * 4, vecs + (base + r) * (long long)dim + c0 + pc * 4);
                }
            }
            cp_async_commit();  // one group per chunk index, empty past the last
        };
        __syncthreads();  // the previous rows' folds are done with the ring
#pragma unroll
        for (int c = 0; c < kStages - 1; c++) issue(c);
        float s0 = -0.0f, s1 = -0.0f;
        for (int c = 0; c < nchunks; c++) {
            issue(c + kStages - 1);
            cp_async_wait<kStages - 1>();  // this thread's pieces of chunk c have landed
            __syncthreads();               // ... and every thread's
            const int c0 = c * kDimChunk;
            const int w = dim - c0 < kDimChunk ? dim - c0 : kDimChunk;
            const float* my = ring + (c % kStages) * kStageFloats + threadIdx.x * kRowStride;
            const float* qc = qs + c0;
            if (metric == 0) {
                for (int k = 0; k < w; k += 4) {
                    const float4 a = *(const float4*)(my + k);
                    float d = __fsub_rn(a.x, qc[k]);
                    s0 = __fadd_rn(s0, __fmul_rn(d, d));
                    d = __fsub_rn(a.y, qc[k + 1]);
                    s0 = __fadd_rn(s0, __fmul_rn(d, d));
                    d = __fsub_rn(a.z, qc[k + 2]);
                    s0 = __fadd_rn(s0, __fmul_rn(d, d));
                    d = __fsub_rn(a.w, qc[k + 3]);
                    s0 = __fadd_rn(s0, __fmul_rn(d, d));
                }
            } else {
                for (int k = 0; k < w; k += 4) {
                    const float4 a = *(const float4*)(my + k);
                    s0 = __fadd_rn(s0, __fmul_rn(a.x, qc[k]));
                    s1 = __fadd_rn(s1, __fmul_rn(a.x, a.x));
                    s0 = __fadd_rn(s0, __fmul_rn(a.y, qc[k + 1]));
                    s1 = __fadd_rn(s1, __fmul_rn(a.y, a.y));
                    s0 = __fadd_rn(s0, __fmul_rn(a.z, qc[k + 2]));
                    s1 = __fadd_rn(s1, __fmul_rn(a.z, a.z));
                    s0 = __fadd_rn(s0, __fmul_rn(a.w, qc[k + 3]));
                    s1 = __fadd_rn(s1, __fmul_rn(a.w, a.w));
                }
            }
            __syncthreads();  // stage c % kStages is refilled by the next issue
        }
        cp_async_wait<0>();
        const long long row = base + threadIdx.x;
        if (row < n) {
            float r;
            if (!valid_at(validity, row)) r = 0.0f;
            else if (metric == 0) r = __fsqrt_rn(s0);
            else {
                const float na = __fsqrt_rn(s1), nb = q_norm;
                r = (na == 0.0f || nb == 0.0f) ? __int_as_float(0x7fc00000)
                                               : __fsub_rn(1.0f, __fdiv_rn(s0, __fmul_rn(na, nb)));
            }
            out[row] = r;
        }
    }
}

}  // namespace

// Launches the distance kernel for one query already in device memory.
void launch_vector_distance(const StreamRef& s, const Backend& b, const Column& vec, long long n,
                            const float* dquery, int metric, float* out) {
    if (n <= 0) return;
    const size_t async_smem = ((size_t)kStages * kStageFloats + vec.dim) * sizeof(float);
    if (vec.dim >= kDimChunk && vec.dim % 4 == 0 && ((uintptr_t)vec.values & 15) == 0 &&
        async_smem <= b.smem_optin) {
        const size_t smem = async_smem;
        allow_smem(vector_distance_async_kernel, smem);
        int per_sm = 0;
        OXB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vector_distance_async_kernel, kRowsPerBlock, smem));
        const long long blocks = (n + kRowsPerBlock - 1) / kRowsPerBlock;
        const long long cap = (long long)b.sms * (per_sm > 0 ? per_sm : 1);
        note_launch(), vector_distance_async_kernel<<<(unsigned)(blocks < cap ? blocks : cap), kRowsPerBlock, smem,
                                                      s->stream>>>((const float*)vec.values, vec.validity, n, vec.dim,
                                                                   dquery, metric, out);
        OXB_CUDA(cudaGetLastError());
        return;
    }
    const int C = vec.dim <= 64 ? vec.dim : 32;
    const size_t smem = (size_t)(kRowsPerBlock * (C + 1) + C) * sizeof(float);
    long long blocks = (n + kRowsPerBlock - 1) / kRowsPerBlock;
    long long cap = (long long)b.sms * 8;
    note_launch(), vector_distance_kernel<<<(unsigned)(blocks < cap ? blocks : cap), kRowsPerBlock, smem, s->stream>>>(
        (const float*)vec.values, vec.validity, n, vec.dim, dquery, metric, out);
    OXB_CUDA(cudaGetLastError());
}

oxb_batch* vector_distance(const StreamRef& s, const Backend& b, const oxb_vector_distance_args& a) {
    if (!a.input) fail(OXB_PLAN, "vector_distance: input batch is null");
    const oxb_batch& in = *a.input;
    if (a.column < 0 || a.column >= (int)in.cols.size())
        fail(OXB_PLAN, "column index " + std::to_string(a.column) + " out of range for a batch with " +
                           std::to_string(in.cols.size()) + " columns");
    const Column& vec = in.cols[a.column];
    if (vec.type != kVectorF32)
        fail(OXB_UNSUPPORTED, "column " + std::to_string(a.column) + " is not FixedSizeList<Float32>");
    if (a.dim != vec.dim)
        fail(OXB_PLAN, "query vector has " + std::to_string(a.dim) + " dimensions but the column has " +
                           std::to_string(vec.dim));
    if (a.metric != OXB_METRIC_L2 && a.metric != OXB_METRIC_COSINE) fail(OXB_PLAN, "unknown metric");
    if (a.dim > 0 && !a.query) fail(OXB_PLAN, "query pointer is null");
    const long long n = in.rows;
    auto out = std::make_unique<oxb_batch>(*a.input);  // input columns shared, not copied
    Column d;
    d.type = kFloat32;
    d.length = n;
    if (n > 0) {
        d.owner_values = dev_alloc(s, n * 4, false);
        d.values = d.owner_values->ptr;
        if (vec.validity) {
            d.owner_validity = dev_alloc(s, (n + 7) / 8, false);
            d.validity = (uint8_t*)d.owner_validity->ptr;
            OXB_CUDA(cudaMemcpyAsync(d.validity, vec.validity, (n + 7) / 8, cudaMemcpyDeviceToDevice, s->stream));
        }
        Scratch<float> q(s, a.dim > 0 ? a.dim : 1);
        OXB_CUDA(cudaMemcpyAsync(q.get(), a.query, a.dim * sizeof(float), cudaMemcpyHostToDevice, s->stream));
        KernelTimer timer(b, s, "vector_distance_kernel");
        timer.begin();
        launch_vector_distance(s, b, vec, n, q.get(), a.metric, (float*)d.values);
        timer.end();
        OXB_CUDA(cudaStreamSynchronize(s->stream));
    }
    out->cols.push_back(std::move(d));
    return out.release();
}

}  // namespace oxb
