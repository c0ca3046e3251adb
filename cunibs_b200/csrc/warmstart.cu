// Learned warm start: the network's elementwise and reduction kernels (training and inference), the
// pose features, and the prolongation of predicted coefficients into a PCG initial guess with a
// per-column fallback to the zero guess.
//
// The network maps a coil pose (the coil origin / 100 mm and the handle axis, 6 numbers) through
// SiLU hidden layers to the coefficients of a reduced basis of the grounded potential built from
// solves the plain method generated. Every matrix product runs on the BF16 tcgen05 GEMM
// (gemm_tc.cu); what is here is the glue around it. A guess whose relative residual is not below 1
// (no better than the zero guess) is dropped for that column, so the plain zero-guess solve remains
// the fallback, and PCG still runs to the same tolerance either way.
#include <cuda_bf16.h>

#include <cmath>

#include "../../include/cunibs_b200.h"
#include <type_traits>

#include "internal.hpp"

namespace cunibs {
namespace {

constexpr int kReduceBlocks = 296;  // 2 x 148 SMs; fixed, so every reduction has one order
constexpr int kReduceThreads = 256;

// x16[i, j] = bf16((f_j - mean_j) / std_j) for the 6 pose features, zero up to ld.
__global__ void features_kernel(const double* __restrict__ T, int k, const float* __restrict__ mean,
                                const float* __restrict__ std, __nv_bfloat16* __restrict__ x16, int ld) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= k * ld) return;
    const int i = q / ld, j = q % ld;
    float v = 0.0f;
    if (j < 6) {
        const double* t = T + 16 * static_cast<std::int64_t>(i);
        // Coil origin (column 3) in units of 100 mm, handle axis (column 1).
        const double f = j < 3 ? t[4 * j + 3] * 0.01 : t[4 * (j - 3) + 1];
        v = (static_cast<float>(f) - mean[j]) / std[j];
    }
    x16[q] = __float2bfloat16_rn(v);
}

// out[j] = sum_i x[i, j], rows summed in order (bias gradients).
__global__ void colsum_kernel(const float* __restrict__ x, int rows, int cols, int ld, float* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= cols) return;
    float s = 0.0f;
    for (int i = 0; i < rows; ++i) s += x[static_cast<std::int64_t>(i) * ld + j];
    out[j] = s;
}

// d = 2 (pred - target) / (rows * cols) in FP32 and BF16 (row-major and transposed); per-block
// partial sums of the squared error.
__global__ void mse_kernel(const float* __restrict__ pred, const float* __restrict__ target, int rows, int cols, int ld,
                           float* __restrict__ d32, __nv_bfloat16* __restrict__ d16, __nv_bfloat16* __restrict__ d16t,
                           int ld_t, float* __restrict__ partial) {
    __shared__ float red[kReduceThreads];
    const std::int64_t total = static_cast<std::int64_t>(rows) * cols;
    const float scale = 2.0f / static_cast<float>(total);
    float acc = 0.0f;
    for (std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; q < total;
         q += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(q / cols), j = static_cast<int>(q % cols);
        const std::int64_t at = static_cast<std::int64_t>(i) * ld + j;
        const float e = pred[at] - target[at];
        acc += e * e;
        const float g = scale * e;
        if (d32) d32[at] = g;
        if (d16) d16[at] = __float2bfloat16_rn(g);
        if (d16t) d16t[static_cast<std::int64_t>(j) * ld_t + i] = __float2bfloat16_rn(g);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int off = kReduceThreads / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void mse_final_kernel(const float* __restrict__ partial, int n, std::int64_t total, float* __restrict__ loss) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float s = 0.0f;
    for (int i = 0; i < n; ++i) s += partial[i];
    *loss = s / static_cast<float>(total);
}

// Adam with bias correction (and decoupled weight decay); refreshes the BF16 copies the GEMMs read:
// w16 [rows, cols] and its transpose w16t [cols, rows].
__global__ void adam_kernel(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ g, std::int64_t n, float lr, float b1, float b2, float eps,
                            float c1, float c2, float wd, int rows, int cols, __nv_bfloat16* __restrict__ w16,
                            __nv_bfloat16* __restrict__ w16t) {
    const std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.0f - b1) * gq;
    const float vq = b2 * v[q] + (1.0f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    float pq = p[q];
    pq -= lr * ((mq / c1) / (sqrtf(vq / c2) + eps) + wd * pq);
    p[q] = pq;
    if (w16) w16[q] = __float2bfloat16_rn(pq);
    if (w16t) {
        const int i = static_cast<int>(q / cols), j = static_cast<int>(q % cols);
        w16t[static_cast<std::int64_t>(j) * rows + i] = __float2bfloat16_rn(pq);
    }
}

// Predicted (standardised) coefficients c -> the B operand of the split-BF16 prolongation. The basis
// is stored [V_hi | V_lo] (K = 2 r); row i of the operand is [c_hi | c_hi] and row 16 + i is
// [c_lo | 0], so output columns i and 16 + i sum to V_hi c_hi + V_lo c_hi + V_hi c_lo, which is V c
// to about 16 significant bits (a BF16 basis alone would leave rounding noise that the residual
// amplifies).
__global__ void denorm_kernel(const float* __restrict__ pred, int k, int n_out, int ld, const float* __restrict__ mean,
                              const float* __restrict__ std, __nv_bfloat16* __restrict__ c16) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= 16 * ld) return;
    const int i = q / ld, j = q % ld;
    float v = 0.0f;
    if (i < k && j < n_out) v = pred[static_cast<std::int64_t>(i) * ld + j] * std[j] + mean[j];
    const __nv_bfloat16 hi = __float2bfloat16_rn(v);
    const __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
    const std::int64_t w = 2 * static_cast<std::int64_t>(ld);
    c16[i * w + j] = hi;
    c16[i * w + ld + j] = hi;
    c16[(16 + i) * w + j] = lo;
    c16[(16 + i) * w + ld + j] = __float2bfloat16_rn(0.0f);
}

// Galerkin coefficients of the right-hand sides in the A-orthonormal basis, c[j][a] = sum_n
// W[n][a] b[n][j] with W = V_hi + V_lo (the stored split basis). Block g takes the contiguous row
// range [g * rows_per, (g + 1) * rows_per) in order, kProjUnroll rows per step with their basis loads
// issued together; thread t owns basis column t (the basis is at most kProjThreads wide per pass,
// wider bases loop). The block's right-hand-side rows are staged in shared memory. The partial sums
// are FP32 (FP64 accumulation measured 174 us per block of 8 at the 1M-tet head, FP64-FMA bound):
// the coefficients are rounded to a split BF16 pair (about 16 bits) before use, and the block
// partials are summed in FP64.
constexpr int kProjThreads = 256;
constexpr int kProjBlocks = 592;
constexpr int kProjUnroll = 8;
constexpr int kProjStage = 64;  // right-hand-side rows staged per step (kProjStage x kMaxK floats)
template <int kMaxK>
__global__ void __launch_bounds__(kProjThreads) project_kernel(const __nv_bfloat16* __restrict__ basis, int n, int ld,
                                                               int n_out, const double* __restrict__ B, int K, int k,
                                                               int rows_per, double* __restrict__ part) {
    __shared__ float sb[kProjStage][kMaxK];
    const int r0 = blockIdx.x * rows_per;
    const int r1 = min(n, r0 + rows_per);
    for (int a0 = 0; a0 < n_out; a0 += kProjThreads) {
        const int a = a0 + threadIdx.x;
        float acc[kMaxK];
#pragma unroll
        for (int j = 0; j < kMaxK; ++j) acc[j] = 0.0f;
        for (int s0 = r0; s0 < r1; s0 += kProjStage) {
            const int ns = min(kProjStage, r1 - s0);
            __syncthreads();
            for (int q = threadIdx.x; q < kProjStage * kMaxK; q += kProjThreads) {
                const int rr = q / kMaxK, j = q % kMaxK;
                sb[rr][j] = (rr < ns && j < k) ? static_cast<float>(B[static_cast<std::int64_t>(s0 + rr) * K + j]) : 0.0f;
            }
            __syncthreads();
            if (a < n_out) {
                // Full steps without guards, so the step's basis loads issue together; then the tail.
                int u0 = 0;
                for (; u0 + kProjUnroll <= ns; u0 += kProjUnroll) {
                    const __nv_bfloat16* w0 = basis + static_cast<std::int64_t>(s0 + u0) * 2 * ld + a;
                    float hi[kProjUnroll], lo[kProjUnroll];
#pragma unroll
                    for (int u = 0; u < kProjUnroll; ++u) {
                        hi[u] = __bfloat162float(w0[static_cast<std::int64_t>(u) * 2 * ld]);
                        lo[u] = __bfloat162float(w0[static_cast<std::int64_t>(u) * 2 * ld + ld]);
                    }
#pragma unroll
                    for (int u = 0; u < kProjUnroll; ++u) {
                        const float wv = hi[u] + lo[u];
#pragma unroll
                        for (int j = 0; j < kMaxK; ++j) acc[j] = fmaf(wv, sb[u0 + u][j], acc[j]);
                    }
                }
                for (; u0 < ns; ++u0) {
                    const __nv_bfloat16* w = basis + static_cast<std::int64_t>(s0 + u0) * 2 * ld + a;
                    const float wv = __bfloat162float(w[0]) + __bfloat162float(w[ld]);
#pragma unroll
                    for (int j = 0; j < kMaxK; ++j) acc[j] = fmaf(wv, sb[u0][j], acc[j]);
                }
            }
        }
        if (a < n_out)
#pragma unroll
            for (int j = 0; j < kMaxK; ++j)
                if (j < k) part[(static_cast<std::int64_t>(blockIdx.x) * k + j) * n_out + a] = acc[j];
    }
}

// One warp per coefficient: the per-block partials summed in a fixed order (lane l takes blocks
// l, l + 32, ..., then a fixed shuffle tree), then split into the prolongation operand (rows
// [c_hi | c_hi] and [c_lo | 0], as denorm_kernel writes them).
__global__ void project_final_kernel(const double* __restrict__ part, int blocks, int k, int n_out, int ld,
                                     __nv_bfloat16* __restrict__ c16) {
    const int warp = static_cast<int>((static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / kWarp);
    const int lane = threadIdx.x % kWarp;
    if (warp >= 16 * ld) return;
    const int i = warp / ld, j = warp % ld;
    double v = 0.0;
    if (i < k && j < n_out)
        for (int g = lane; g < blocks; g += kWarp) v += part[(static_cast<std::int64_t>(g) * k + i) * n_out + j];
    for (int off = kWarp / 2; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane != 0) return;
    const float vf = static_cast<float>(v);
    const __nv_bfloat16 hi = __float2bfloat16_rn(vf);
    const __nv_bfloat16 lo = __float2bfloat16_rn(vf - __bfloat162float(hi));
    const std::int64_t w = 2 * static_cast<std::int64_t>(ld);
    c16[i * w + j] = hi;
    c16[i * w + ld + j] = hi;
    c16[(16 + i) * w + j] = lo;
    c16[(16 + i) * w + ld + j] = __float2bfloat16_rn(0.0f);
}

// X0[row, c] (FP64, width K) = x0f[row, c] + x0f[row, 16 + c] for the k predicted columns.
__global__ void widen_kernel(const float* __restrict__ x0f, int n, int ldf, int k, int K, double* __restrict__ X0) {
    const std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<std::int64_t>(n) * K) return;
    const int row = static_cast<int>(q / K), c = static_cast<int>(q % K);
    const float* r = x0f + static_cast<std::int64_t>(row) * ldf;
    X0[q] = c < k ? static_cast<double>(r[c]) + static_cast<double>(r[16 + c]) : 0.0;
}

}  // namespace

void pose_features(const double* T_dev, int k, const float* mean, const float* std, __nv_bfloat16* x16, int ld,
                   cudaStream_t s) {
    features_kernel<<<grid_for(static_cast<std::int64_t>(k) * ld), kBlock, 0, s>>>(T_dev, k, mean, std, x16, ld);
    count_launch();
    CUNIBS_LAUNCH_CHECK("pose features");
}

void warm_start_guess(WarmStart& ws, const double* T_dev, const double* B, int k, int K, double* X0, int mode,
                      cudaStream_t s) {
    constexpr int kRowsPad = 16;  // the network's batch (k <= 16), one BN = 16 GEMM tile wide
    const int depth = ws.depth;
    if (mode == kGuessProjection) {
        // The Galerkin projection onto the basis: the A-norm-best guess it spans, from the
        // right-hand sides themselves (no network).
        ws.c16.reserve(static_cast<std::size_t>(2 * kRowsPad) * 2 * ws.n_out_pad);
        ws.x0f.reserve(static_cast<std::size_t>(ws.n_red) * 2 * kRowsPad);
        ws.error.reserve(1);
        const int rows_per = (ws.n_red + kProjBlocks - 1) / kProjBlocks;
        const int blocks = (ws.n_red + rows_per - 1) / rows_per;
        ws.partials.reserve(static_cast<std::size_t>(blocks) * k * ws.n_out);
        // Accumulators for the block's own width only (K in {1, 2, 4, 8, 16}).
        auto go = [&](auto kc) {
            constexpr int KK = decltype(kc)::value;
            project_kernel<KK><<<blocks, kProjThreads, 0, s>>>(ws.basis.get(), ws.n_red, ws.n_out_pad, ws.n_out, B, K,
                                                               k, rows_per, ws.partials.get());
        };
        if (K <= 1) go(std::integral_constant<int, 1>{});
        else if (K <= 2) go(std::integral_constant<int, 2>{});
        else if (K <= 4) go(std::integral_constant<int, 4>{});
        else if (K <= 8) go(std::integral_constant<int, 8>{});
        else go(std::integral_constant<int, 16>{});
        count_launch();
        project_final_kernel<<<grid_for(static_cast<std::int64_t>(16) * ws.n_out_pad * kWarp), kBlock, 0, s>>>(
            ws.partials.get(), blocks, k, ws.n_out, ws.n_out_pad, ws.c16.get());
        count_launch();
    } else {
        ws.x16.reserve(kRowsPad * kWarmInPad);
        ws.h16a.reserve(kRowsPad * ws.hidden);
        ws.h16b.reserve(kRowsPad * ws.hidden);
        ws.pred.reserve(static_cast<std::size_t>(kRowsPad) * ws.n_out_pad);
        ws.c16.reserve(static_cast<std::size_t>(2 * kRowsPad) * 2 * ws.n_out_pad);
        ws.x0f.reserve(static_cast<std::size_t>(ws.n_red) * 2 * kRowsPad);
        ws.partials.reserve(1);
        ws.norms.reserve(16);
        ws.error.reserve(1);
        CUNIBS_CHECK(cudaMemsetAsync(ws.x16.get(), 0, sizeof(__nv_bfloat16) * kRowsPad * kWarmInPad, s));
        pose_features(T_dev, k, ws.in_mean.get(), ws.in_std.get(), ws.x16.get(), kWarmInPad, s);
        // Hidden layers: h = silu(x W^T + b).
        const __nv_bfloat16* in = ws.x16.get();
        int in_dim = kWarmInPad;
        for (int l = 0; l < depth; ++l) {
            __nv_bfloat16* out = (l % 2 == 0) ? ws.h16a.get() : ws.h16b.get();
            GemmProblem g;
            g.a = in;
            g.lda = in_dim;
            g.b = ws.w16[l].get();
            g.ldb = in_dim;
            g.M = kRowsPad;
            g.N = ws.hidden;
            g.K = in_dim;
            g.ep.bias = ws.bias[l].get();
            g.ep.act = 1;
            g.ep.out16 = out;
            g.ep.ld_out = ws.hidden;
            g.ep.error = ws.error.get();
            gemm_bf16(g, s);
            in = out;
            in_dim = ws.hidden;
        }
        GemmProblem g;
        g.a = in;
        g.lda = in_dim;
        g.b = ws.w16[depth].get();
        g.ldb = in_dim;
        g.M = kRowsPad;
        g.N = ws.n_out_pad;
        g.K = in_dim;
        g.ep.bias = ws.bias[depth].get();
        g.ep.out32 = ws.pred.get();
        g.ep.ld_out = ws.n_out_pad;
        g.ep.error = ws.error.get();
        gemm_bf16(g, s);
        denorm_kernel<<<grid_for(kRowsPad * ws.n_out_pad), kBlock, 0, s>>>(ws.pred.get(), k, ws.n_out, ws.n_out_pad,
                                                                            ws.out_mean.get(), ws.out_std.get(),
                                                                            ws.c16.get());
        count_launch();
    }
    // Prolongation through the basis: [n_red, 32] = [V_hi | V_lo] [n_red, 2r] . c16 [32, 2r]^T.
    GemmProblem p;
    p.a = ws.basis.get();
    p.lda = 2 * ws.n_out_pad;
    p.b = ws.c16.get();
    p.ldb = 2 * ws.n_out_pad;
    p.M = ws.n_red;
    p.N = 2 * kRowsPad;
    p.K = 2 * ws.n_out_pad;
    p.ep.out32 = ws.x0f.get();
    p.ep.ld_out = 2 * kRowsPad;
    p.ep.error = ws.error.get();
    gemm_bf16(p, s);
    const std::int64_t nk = static_cast<std::int64_t>(ws.n_red) * K;
    widen_kernel<<<grid_for(nk), kBlock, 0, s>>>(ws.x0f.get(), ws.n_red, 2 * kRowsPad, k, K, X0);
    count_launch();
    CUNIBS_LAUNCH_CHECK("warm start");
}

void warm_start_check(WarmStart& ws, cudaStream_t s) {
    int h_err = 0;
    CUNIBS_CHECK(cudaMemcpyAsync(&h_err, ws.error.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    CUNIBS_CHECK(cudaStreamSynchronize(s));
    if (h_err) fail(kETimeout, "a tensor-core GEMM of the warm start timed out waiting on its pipeline");
}

}  // namespace cunibs

using namespace cunibs;

namespace {
template <typename F>
int guarded_call(F&& f) {
    try {
        f();
        return CUNIBS_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return CUNIBS_EINTERNAL;
    }
}
}  // namespace

extern "C" {

int cunibs_gemm_bf16(const void* A, int lda, const void* B, int ldb, int M, int N, int K, const float* bias,
                     const float* gate, int ld_gate, int act, float* out32, void* out16, int ld_out, void* out16t,
                     int ld_t, void* stream) {
    return guarded_call([&] {
        if (!A || !B) fail(kEInval, "A and B must not be NULL");
        if (!out32 && !out16 && !out16t) fail(kEInval, "no output");
        if (act != 0 && act != 1) fail(kEInval, "act must be 0 (none) or 1 (SiLU)");
        GemmProblem g;
        g.a = static_cast<const __nv_bfloat16*>(A);
        g.lda = lda;
        g.b = static_cast<const __nv_bfloat16*>(B);
        g.ldb = ldb;
        g.M = M;
        g.N = N;
        g.K = K;
        g.ep.bias = bias;
        g.ep.gate = gate;
        g.ep.ld_gate = ld_gate;
        g.ep.act = act;
        g.ep.out32 = out32;
        g.ep.out16 = static_cast<__nv_bfloat16*>(out16);
        g.ep.ld_out = ld_out;
        g.ep.out16t = static_cast<__nv_bfloat16*>(out16t);
        g.ep.ld_t = ld_t;
        if (lda < K || ldb < K || (out32 || out16 ? ld_out < N : false)) fail(kEInval, "leading dimension below the size");
        gemm_bf16(g, static_cast<cudaStream_t>(stream));
    });
}

int cunibs_gemm_status(void* stream, int* expired) {
    return guarded_call([&] {
        const bool e = gemm_status(static_cast<cudaStream_t>(stream));
        if (expired) *expired = e ? 1 : 0;
        if (e) fail(kETimeout, "a bounded mbarrier wait of a tensor-core GEMM expired; its outputs are invalid");
    });
}

int cunibs_debug_gemm_waits(long long max_polls, long long max_ns, int withhold_loads) {
    return guarded_call([&] {
        gemm_set_waits(max_polls, max_ns > 0 ? static_cast<unsigned long long>(max_ns) : 0ULL, withhold_loads);
    });
}

int cunibs_mlp_colsum(const float* x, int rows, int cols, int ld, float* out, void* stream) {
    return guarded_call([&] {
        if (!x || !out || rows < 1 || cols < 1 || ld < cols) fail(kEInval, "bad colsum arguments");
        colsum_kernel<<<grid_for(cols), kBlock, 0, static_cast<cudaStream_t>(stream)>>>(x, rows, cols, ld, out);
        count_launch();
        CUNIBS_LAUNCH_CHECK("colsum");
    });
}

int cunibs_mlp_mse(const float* pred, const float* target, int rows, int cols, int ld, float* loss, float* d32,
                   void* d16, void* d16t, int ld_t, float* scratch, void* stream) {
    return guarded_call([&] {
        if (!pred || !target || !loss || !scratch || rows < 1 || cols < 1 || ld < cols)
            fail(kEInval, "bad mse arguments");
        if (d16t && ld_t < rows) fail(kEInval, "transposed gradient leading dimension below rows");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        mse_kernel<<<kReduceBlocks, kReduceThreads, 0, s>>>(pred, target, rows, cols, ld, d32,
                                                            static_cast<__nv_bfloat16*>(d16),
                                                            static_cast<__nv_bfloat16*>(d16t), ld_t, scratch);
        mse_final_kernel<<<1, 32, 0, s>>>(scratch, kReduceBlocks, static_cast<std::int64_t>(rows) * cols, loss);
        count_launch(2);
        CUNIBS_LAUNCH_CHECK("mse");
    });
}

int cunibs_mlp_adam(float* param, float* m, float* v, const float* grad, long long n, float lr, float beta1,
                    float beta2, float eps, int step, float weight_decay, int rows, int cols, void* w16, void* w16t,
                    void* stream) {
    return guarded_call([&] {
        if (!param || !m || !v || !grad || n < 1 || step < 1) fail(kEInval, "bad adam arguments");
        if ((w16 || w16t) && static_cast<long long>(rows) * cols != n) fail(kEInval, "rows * cols must equal n");
        const float c1 = 1.0f - std::pow(beta1, static_cast<float>(step));
        const float c2 = 1.0f - std::pow(beta2, static_cast<float>(step));
        adam_kernel<<<grid_for(n), kBlock, 0, static_cast<cudaStream_t>(stream)>>>(
            param, m, v, grad, n, lr, beta1, beta2, eps, c1, c2, weight_decay, rows, cols,
            static_cast<__nv_bfloat16*>(w16), static_cast<__nv_bfloat16*>(w16t));
        count_launch();
        CUNIBS_LAUNCH_CHECK("adam");
    });
}

int cunibs_mlp_features(const double* transforms, int k, const float* mean, const float* std, void* x16, int ld,
                        void* stream) {
    return guarded_call([&] {
        if (!transforms || !mean || !std || !x16 || k < 1 || ld < 6) fail(kEInval, "bad feature arguments");
        pose_features(transforms, k, mean, std, static_cast<__nv_bfloat16*>(x16), ld,
                      static_cast<cudaStream_t>(stream));
    });
}

}  // extern "C"
