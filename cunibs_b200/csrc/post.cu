// Post-processing of a solved block: E = -grad v - dA/dt per tetrahedron, the potential on the full
// node set, and the gray-matter summary metrics.
//
// Reference behaviour restated: reconstruct.cu:36-76 (FP64 accumulation of grad v, FP32 output),
// fem/solve.py:939-941 (grounded node carries v = 0), metrics.py:58-243 (volume-weighted
// peak/location, centre of gravity, mean/std, p50/p95/p99/p99.9 at midpoint positions with linear
// interpolation, focality at 0.5 and 0.75 of p99.9). The percentiles come from a stable segmented
// radix sort of each placement's gray-matter |E| (keys = |E|, values = element slot) and a
// fixed-order tiled prefix sum of the sorted volumes, so the ranks are integer-exact and the
// cumulative weights reproduce run to run.
#include <cub/cub.cuh>

#include "internal.hpp"

namespace cunibs {
namespace {

// One thread per (tet, column): E = -sum_i v[n_i] g_i - dadt_elm (FP64 accumulation).
__global__ void reconstruct_kernel(const double* __restrict__ x_red, int K, int ground, const int* __restrict__ tets,
                                   const float* __restrict__ g32, const float* __restrict__ elm, int n_tets, int k,
                                   float* __restrict__ E, float* __restrict__ magn) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<long>(n_tets) * k) return;
    const int c = static_cast<int>(q / n_tets);
    const int e = static_cast<int>(q % n_tets);
    const int4 tn = reinterpret_cast<const int4*>(tets)[e];
    const int nd[4] = {tn.x, tn.y, tn.z, tn.w};
    const float* ge = g32 + 12 * static_cast<long>(e);
    double gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int node = nd[i];
        const double vi = (node == ground) ? 0.0 : x_red[static_cast<long>(node - (node > ground ? 1 : 0)) * K + c];
        gx += vi * static_cast<double>(ge[3 * i]);
        gy += vi * static_cast<double>(ge[3 * i + 1]);
        gz += vi * static_cast<double>(ge[3 * i + 2]);
    }
    const float* el = elm + static_cast<long>(c) * n_tets * 3 + 3 * static_cast<long>(e);
    const double ex = -gx - static_cast<double>(el[0]);
    const double ey = -gy - static_cast<double>(el[1]);
    const double ez = -gz - static_cast<double>(el[2]);
    if (E != nullptr) {
        float* o = E + static_cast<long>(c) * n_tets * 3 + 3 * static_cast<long>(e);
        o[0] = static_cast<float>(ex);
        o[1] = static_cast<float>(ey);
        o[2] = static_cast<float>(ez);
    }
    magn[static_cast<long>(c) * n_tets + e] = static_cast<float>(sqrt(ex * ex + ey * ey + ez * ez));
}

__global__ void scatter_kernel(const double* __restrict__ x_red, int K, int ground, int n_nodes, int k,
                               double* __restrict__ v) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<long>(n_nodes) * k) return;
    const int c = static_cast<int>(q / n_nodes);
    const int i = static_cast<int>(q % n_nodes);
    v[q] = (i == ground) ? 0.0 : x_red[static_cast<long>(i - (i > ground ? 1 : 0)) * K + c];
}

// Sort keys of every placement's gray-matter |E|: (placement << 32) | bits(|E|). |E| >= 0, so its
// IEEE bit pattern orders like its value, and one stable radix sort of all k segments together
// orders each placement's values with ties kept in element order.
__global__ void gm_gather_kernel(const float* __restrict__ magn, const int* __restrict__ gm, int n_gm, int n_tets, int k,
                                 std::uint64_t* __restrict__ keys, int* __restrict__ vals) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<long>(n_gm) * k) return;
    const int c = static_cast<int>(q / n_gm);
    const int i = static_cast<int>(q % n_gm);
    const float v = magn[static_cast<long>(c) * n_tets + gm[i]];
    keys[q] = (static_cast<std::uint64_t>(c) << 32) | __float_as_uint(v);
    vals[q] = i;
}

constexpr int kScanTile = 1024;

// Inclusive scan of the sorted FP64 volumes within each tile of each placement's segment: a
// sequential walk per 8-element thread strip, then a fixed tree over the strips.
__global__ void tile_scan_kernel(const int* __restrict__ sorted_idx, const std::uint64_t* __restrict__ sorted_keys,
                                 const int* __restrict__ gm, const float* __restrict__ vols32, int n_gm,
                                 float* __restrict__ values, double* __restrict__ w_sorted, double* __restrict__ cw,
                                 double* __restrict__ tile_tot) {
    constexpr int kPer = kScanTile / 128;
    __shared__ double strip[128];
    const int c = blockIdx.y;
    const int tile = blockIdx.x;
    const long base = static_cast<long>(c) * n_gm;
    const int start = tile * kScanTile + threadIdx.x * kPer;
    double local[kPer];
    double run = 0.0;
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
        const int i = start + u;
        double w = 0.0;
        if (i < n_gm) {
            w = static_cast<double>(vols32[gm[sorted_idx[base + i]]]);
            w_sorted[base + i] = w;
            values[base + i] = __uint_as_float(static_cast<unsigned>(sorted_keys[base + i] & 0xffffffffu));
        }
        run += w;
        local[u] = run;
    }
    strip[threadIdx.x] = run;
    __syncthreads();
    // Exclusive prefix of the strip totals, Hillis-Steele over 128 entries (fixed order).
    for (int off = 1; off < 128; off <<= 1) {
        const double add = (threadIdx.x >= off) ? strip[threadIdx.x - off] : 0.0;
        __syncthreads();
        strip[threadIdx.x] += add;
        __syncthreads();
    }
    const double before = (threadIdx.x > 0) ? strip[threadIdx.x - 1] : 0.0;
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
        const int i = start + u;
        if (i < n_gm) cw[base + i] = before + local[u];
    }
    if (threadIdx.x == 127) tile_tot[static_cast<long>(c) * gridDim.x + tile] = strip[127];
}

// Adds the (sequentially scanned) totals of earlier tiles.
__global__ void tile_offset_kernel(double* __restrict__ cw, const double* __restrict__ tile_tot, int n_gm, int tiles) {
    __shared__ double off;
    const int c = blockIdx.y;
    const int tile = blockIdx.x;
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int t = 0; t < tile; ++t) s += tile_tot[static_cast<long>(c) * tiles + t];
        off = s;
    }
    __syncthreads();
    if (tile == 0) return;
    const long base = static_cast<long>(c) * n_gm;
    for (int i = tile * kScanTile + threadIdx.x; i < min(n_gm, (tile + 1) * kScanTile); i += blockDim.x)
        cw[base + i] += off;
}

// Gray-matter summary of each placement (metrics.py:209-243) in three launches, so the element
// passes spread over the GPU: kSumBlocks blocks per placement reduce fixed strided shares of the
// elements in a fixed tree, and the partials are combined in a fixed sequential order (results
// reproducible and independent of k). The peak is the largest |E|, the first in gray-matter order
// among equals.
constexpr int kSumBlocks = 64;
constexpr int kSumT = 256;
constexpr int kSumFields = 6;  // peak value, w, w*|E|, and the three w*|E|*barycentre sums

__global__ void __launch_bounds__(kSumT) summary_stats_kernel(const float* __restrict__ magn, const int* __restrict__ gm,
                                                             int n_gm, int n_tets, const float* __restrict__ vols32,
                                                             const double* __restrict__ bary, double* __restrict__ part,
                                                             int* __restrict__ part_i) {
    __shared__ double sv[kSumT], sw[kSumT], swm[kSumT], sx[kSumT], sy[kSumT], sz[kSumT];
    __shared__ int si[kSumT];
    const int c = blockIdx.y;
    const float* m = magn + static_cast<long>(c) * n_tets;
    double best = -1.0;
    int bi = 0x7fffffff;
    double w_s = 0.0, wm_s = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
    for (int i = blockIdx.x * kSumT + threadIdx.x; i < n_gm; i += kSumBlocks * kSumT) {
        const int e = gm[i];
        const double mv = m[e];
        const double w = vols32[e];
        if (mv > best) {
            best = mv;
            bi = i;
        }
        w_s += w;
        const double ww = w * mv;
        wm_s += ww;
        cx += ww * bary[3 * static_cast<long>(e)];
        cy += ww * bary[3 * static_cast<long>(e) + 1];
        cz += ww * bary[3 * static_cast<long>(e) + 2];
    }
    const int t = threadIdx.x;
    sv[t] = best;
    si[t] = bi;
    sw[t] = w_s;
    swm[t] = wm_s;
    sx[t] = cx;
    sy[t] = cy;
    sz[t] = cz;
    __syncthreads();
    for (int off = kSumT / 2; off > 0; off >>= 1) {
        if (t < off) {
            const int o = t + off;
            if (sv[o] > sv[t] || (sv[o] == sv[t] && si[o] < si[t])) {
                sv[t] = sv[o];
                si[t] = si[o];
            }
            sw[t] += sw[o];
            swm[t] += swm[o];
            sx[t] += sx[o];
            sy[t] += sy[o];
            sz[t] += sz[o];
        }
        __syncthreads();
    }
    if (t == 0) {
        const long q = static_cast<long>(c) * kSumBlocks + blockIdx.x;
        double* o = part + q * kSumFields;
        o[0] = sv[0];
        o[1] = sw[0];
        o[2] = swm[0];
        o[3] = sx[0];
        o[4] = sy[0];
        o[5] = sz[0];
        part_i[q] = si[0];
    }
}

// Sum of field f over a placement's partials, in block order.
__device__ __forceinline__ double part_sum(const double* part, int c, int f) {
    double v = 0.0;
    for (int b = 0; b < kSumBlocks; ++b) v += part[(static_cast<long>(c) * kSumBlocks + b) * kSumFields + f];
    return v;
}

__global__ void __launch_bounds__(kSumT) summary_var_kernel(const float* __restrict__ magn, const int* __restrict__ gm,
                                                           int n_gm, int n_tets, const float* __restrict__ vols32,
                                                           const double* __restrict__ part,
                                                           double* __restrict__ var_part) {
    __shared__ double sv[kSumT];
    __shared__ double mean_sh;
    const int c = blockIdx.y;
    if (threadIdx.x == 0) mean_sh = part_sum(part, c, 2) / part_sum(part, c, 1);
    __syncthreads();
    const double mean = mean_sh;
    const float* m = magn + static_cast<long>(c) * n_tets;
    double var = 0.0;
    for (int i = blockIdx.x * kSumT + threadIdx.x; i < n_gm; i += kSumBlocks * kSumT) {
        const int e = gm[i];
        const double d = static_cast<double>(m[e]) - mean;
        var += static_cast<double>(vols32[e]) * d * d;
    }
    sv[threadIdx.x] = var;
    __syncthreads();
    for (int off = kSumT / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) sv[threadIdx.x] += sv[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) var_part[static_cast<long>(c) * kSumBlocks + blockIdx.x] = sv[0];
}

// Largest i in [lo, hi) with pred(i) true, for a predicate true on a prefix of [lo, hi) and
// pred(lo) true: 32 probes per step across the warp (about log32 n dependent loads instead of
// log2 n). Every lane returns the same index, the one a binary search finds.
template <typename Pred>
__device__ __forceinline__ int warp_last_true(int lo, int hi, Pred pred) {
    const int lane = threadIdx.x % kWarp;
    while (hi - lo > 1) {
        const long span = hi - lo;
        const int probe = lo + static_cast<int>((span * (lane + 1)) / (kWarp + 1));
        const bool ok = probe > lo && probe < hi && pred(probe);
        const unsigned mask = __ballot_sync(0xffffffffu, ok || probe <= lo);
        const int cnt = __popc(mask);  // probes are non-decreasing, so the true ones are a prefix
        const int new_lo = cnt > 0 ? __shfl_sync(0xffffffffu, probe, cnt - 1) : lo;
        const int new_hi = cnt < kWarp ? __shfl_sync(0xffffffffu, probe, cnt) : hi;
        lo = max(lo, new_lo);
        hi = (new_hi > lo) ? new_hi : lo + 1;
    }
    return lo;
}

// Weighted quantile of the sorted values v with weights w (cw: their cumulative sum):
// interp(q, pos, v) with pos_i = (cw_i - w_i/2) / cw_last (metrics.py:82-95, numpy.interp), the
// search spread over a warp.
__device__ double warp_quantile(double q, const float* __restrict__ v, const double* __restrict__ w,
                                const double* __restrict__ cw, int n) {
    const double total = cw[n - 1];
    auto pos = [&](int i) { return (cw[i] - 0.5 * w[i]) / total; };
    if (q <= pos(0)) return v[0];
    if (q >= pos(n - 1)) return v[n - 1];
    const int lo = warp_last_true(0, n - 1, [&](int i) { return pos(i) <= q; });
    const double x0 = pos(lo), x1 = pos(lo + 1);
    const double slope = (static_cast<double>(v[lo + 1]) - static_cast<double>(v[lo])) / (x1 - x0);
    return slope * (q - x0) + static_cast<double>(v[lo]);
}

// One warp per placement: partials combined in a fixed order (lane l takes blocks l and l + 32,
// then a butterfly), the weighted quantiles and focality from the sorted |E| and its cumulative
// volume with warp-wide searches.
__global__ void __launch_bounds__(kWarp) summary_final_kernel(
    int k, const int* __restrict__ gm, int n_gm, const double* __restrict__ bary, const double* __restrict__ part,
    const int* __restrict__ part_i, const double* __restrict__ var_part, const float* __restrict__ sorted_keys,
    const double* __restrict__ w_sorted, const double* __restrict__ cw, double* __restrict__ out) {
    static_assert(kSumBlocks == 2 * kWarp, "two partials per lane");
    const int c = blockIdx.x;
    const int lane = threadIdx.x;
    double best = -1.0;
    int bi = 0x7fffffff;
    double f[kSumFields] = {};
    double var = 0.0;
    for (int h = 0; h < 2; ++h) {
        const long q = static_cast<long>(c) * kSumBlocks + lane + h * kWarp;
        const double v = part[q * kSumFields];
        const int i = part_i[q];
        if (v > best || (v == best && i < bi)) {
            best = v;
            bi = i;
        }
#pragma unroll
        for (int j = 1; j < kSumFields; ++j) f[j] += part[q * kSumFields + j];
        var += var_part[q];
    }
#pragma unroll
    for (int off = kWarp / 2; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, best, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        if (ov > best || (ov == best && oi < bi)) {
            best = ov;
            bi = oi;
        }
#pragma unroll
        for (int j = 1; j < kSumFields; ++j) f[j] += __shfl_xor_sync(0xffffffffu, f[j], off);
        var += __shfl_xor_sync(0xffffffffu, var, off);
    }
    double* o = out + static_cast<long>(c) * kSummaryLen;
    const double w_s = f[1], wm_s = f[2];
    if (lane == 0) {
        const int e = gm[bi];
        o[0] = best;
        o[1] = bary[3 * static_cast<long>(e)];
        o[2] = bary[3 * static_cast<long>(e) + 1];
        o[3] = bary[3 * static_cast<long>(e) + 2];
        o[4] = f[3] / wm_s;
        o[5] = f[4] / wm_s;
        o[6] = f[5] / wm_s;
        o[7] = w_s;
        o[8] = wm_s / w_s;
        o[9] = sqrt(var / w_s);
    }
    const long base = static_cast<long>(c) * n_gm;
    const float* v = sorted_keys + base;
    const double* w = w_sorted + base;
    const double* cwp = cw + base;
    const double qs[4] = {static_cast<double>(0.5f), static_cast<double>(0.95f), static_cast<double>(0.99f),
                          static_cast<double>(0.999f)};
    double p999 = 0.0;
    for (int j = 0; j < 4; ++j) {
        const double qv = warp_quantile(qs[j], v, w, cwp, n_gm);
        if (lane == 0) o[10 + j] = qv;
        p999 = qv;
    }
    const double fr[2] = {0.5, 0.75};
    for (int g = 0; g < 2; ++g) {
        const double thr = fr[g] * p999;
        // First sorted slot with |E| >= thr; everything from there on is stimulated.
        int lo;
        if (static_cast<double>(v[0]) >= thr) lo = 0;
        else if (!(static_cast<double>(v[n_gm - 1]) >= thr)) lo = n_gm;
        else lo = warp_last_true(0, n_gm - 1, [&](int i) { return !(static_cast<double>(v[i]) >= thr); }) + 1;
        if (lane == 0) o[14 + g] = (lo == 0) ? cwp[n_gm - 1] : (cwp[n_gm - 1] - cwp[lo - 1]);
    }
}

__global__ void nan_fill_kernel(double* out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = NAN;
}

}  // namespace

void reconstruct_block(const Mesh& m, const double* x_red, int k, int K, const float* elm, float* E, float* magnE,
                       cudaStream_t s) {
    const long total = static_cast<long>(m.n_tets) * k;
    reconstruct_kernel<<<grid_for(total), kBlock, 0, s>>>(x_red, K, m.ground, m.tets.get(), m.g32.get(), elm, m.n_tets,
                                                          k, E, magnE); count_launch();
    CUNIBS_LAUNCH_CHECK("reconstruct");
}

void scatter_potential(const Mesh& m, const double* x_red, int k, int K, double* v, cudaStream_t s) {
    const long total = static_cast<long>(m.n_nodes) * k;
    scatter_kernel<<<grid_for(total), kBlock, 0, s>>>(x_red, K, m.ground, m.n_nodes, k, v); count_launch();
    CUNIBS_LAUNCH_CHECK("scatter potential");
}

void gm_summary_impl(const Mesh& m, const float* magnE, int k, double* out, SummaryWork& w, cudaStream_t s) {
    const int n = m.n_gm;
    if (n == 0) {
        nan_fill_kernel<<<grid_for(k * kSummaryLen), kBlock, 0, s>>>(out, k * kSummaryLen); count_launch();
        return;
    }
    const long total = static_cast<long>(n) * k;
    w.keys.reserve(total);
    w.keys_s.reserve(total);
    w.vals.reserve(total);
    w.vals_s.reserve(total);
    w.offsets.reserve(k + 1);
    w.w_sorted.reserve(total);
    w.cw.reserve(total);
    const int tiles = (n + kScanTile - 1) / kScanTile;
    w.tile_tot.reserve(static_cast<std::size_t>(tiles) * k);
    w.k64.reserve(total);
    w.k64_s.reserve(total);
    gm_gather_kernel<<<grid_for(total), kBlock, 0, s>>>(magnE, m.gm_index.get(), n, m.n_tets, k, w.k64.get(),
                                                        w.vals.get()); count_launch();
    int seg_bits = 0;
    while ((1 << seg_bits) < k) ++seg_bits;
    std::size_t bytes = 0;
    CUNIBS_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, w.k64.get(), w.k64_s.get(), w.vals.get(),
                                                 w.vals_s.get(), static_cast<int>(total), 0, 32 + seg_bits, s));
    w.temp.reserve(bytes ? bytes : 1);
    CUNIBS_CHECK(cub::DeviceRadixSort::SortPairs(w.temp.get(), bytes, w.k64.get(), w.k64_s.get(), w.vals.get(),
                                                 w.vals_s.get(), static_cast<int>(total), 0, 32 + seg_bits, s));
    tile_scan_kernel<<<dim3(tiles, k), 128, 0, s>>>(w.vals_s.get(), w.k64_s.get(), m.gm_index.get(), m.vols32.get(), n,
                                                   w.keys_s.get(), w.w_sorted.get(), w.cw.get(), w.tile_tot.get()); count_launch();
    tile_offset_kernel<<<dim3(tiles, k), 256, 0, s>>>(w.cw.get(), w.tile_tot.get(), n, tiles); count_launch();
    w.part.reserve(static_cast<std::size_t>(k) * kSumBlocks * (kSumFields + 1));
    w.part_i.reserve(static_cast<std::size_t>(k) * kSumBlocks);
    double* part = w.part.get();
    double* var_part = part + static_cast<std::size_t>(k) * kSumBlocks * kSumFields;
    summary_stats_kernel<<<dim3(kSumBlocks, k), kSumT, 0, s>>>(magnE, m.gm_index.get(), n, m.n_tets, m.vols32.get(),
                                                               m.bary.get(), part, w.part_i.get());
    summary_var_kernel<<<dim3(kSumBlocks, k), kSumT, 0, s>>>(magnE, m.gm_index.get(), n, m.n_tets, m.vols32.get(),
                                                             part, var_part);
    summary_final_kernel<<<k, kWarp, 0, s>>>(k, m.gm_index.get(), n, m.bary.get(), part, w.part_i.get(), var_part,
                                          w.keys_s.get(), w.w_sorted.get(), w.cw.get(), out);
    count_launch(3);
    CUNIBS_LAUNCH_CHECK("gm summary");
}

void gm_summary(const Mesh& m, const float* magnE, int k, double* summary_dev, SummaryWork& w, cudaStream_t s) {
    gm_summary_impl(m, magnE, k, summary_dev, w, s);
}

}  // namespace cunibs
