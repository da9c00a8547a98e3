// L2 / cosine distance between one query and a FixedSizeList<Float32>
// column (GpuBackend::vector_distance, crates/oxidelake-device/src/backend.rs:173).
//
// Bit-exact with cpu/kernels.rs:909-927: each row's sums are folded in index
// order from -0.0 with one correctly rounded IEEE operation per Rust
// operator (no fused multiply-add: __fmul_rn / __fadd_rn), then sqrt and
// divide correctly rounded.  One thread owns one row; a block stages 128 rows
// x 32 (or all, when dim <= 64) dimensions through shared memory with
// coalesced loads, so the sequential per-row fold still reads HBM at full
// width.
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

}  // namespace

// Launches the distance kernel for one query already in device memory.
void launch_vector_distance(const StreamRef& s, const Backend& b, const Column& vec, long long n,
                            const float* dquery, int metric, float* out) {
    if (n <= 0) return;
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
