// Coil field table: the coil's dipole sum sampled once per coil in its own frame and interpolated
// at the nodes away from the coil, so that a block's dA/dt costs a table read per node instead of
// a sum over every dipole.
//
// dA/dt(r) = didt * mu0/4pi * sum_j m_j x (r - s_j) / |r - s_j|^3 (fem/placement.py:279-317) depends
// on r only through the coil-frame position r' = R^T (r - c), so the bare sum A'(r') is one smooth
// field per coil, shared by every placement: A(r) = didt * 1e-7 * R A'(r'). Below the coil (depth
// zr = z' - z_top > 0, the coil frame's z pointing into the head) it is harmonic and varies on the
// scale of the depth, so its samples sit in layers at depths z_j = z0 (1 + step)^(j - 1), each a
// square grid of spacing step * z_j: a fixed number of points per depth scale, from z0 to the far
// side of the head. A node takes the tricubic Lagrange interpolant of the 4 x 4 x 4 samples around
// it, with the depth coordinate zeta = ln(zr / z0) / ln(1 + step) (uniform across layers). Its error
// falls as step^4: at step 0.035 about 1e-7 of the field in relative L2, the rounding level of the
// FP32 direct sum. Nodes shallower than z0, or outside the sampled box, take the direct sum; they are
// listed per placement and summed by blocks that split the dipoles over eight warps.
//
// Every table is checked when it is built: at 4096 points in the middle of grid cells (where the
// interpolant is least accurate) it is compared with the direct sum, and a table whose relative L2
// error exceeds kCheckTolerance is not used.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "coil_packed.cuh"
#include "internal.hpp"

namespace cunibs {
namespace {

constexpr int kTableThreads = 256;
constexpr int kNearWarps = 8;
constexpr int kCheckPoints = 4096;
constexpr double kCheckTolerance = 2e-6;

struct TableArgs {
    const CoilTableLayer* layers;
    const void* data;
    int n_layers;
    float z_top, inv_z0, inv_log_step;
};

template <int NC>
struct TableVec;
template <>
struct TableVec<2> {
    using T = float2;
};
template <>
struct TableVec<3> {
    using T = float4;
};

// Cubic Lagrange weights at the nodes -1, 0, 1, 2 for the position t (t in [0, 1) up to rounding).
__device__ __forceinline__ void lagrange4(float t, float w[4]) {
    const float tp1 = t + 1.f, tm1 = t - 1.f, tm2 = t - 2.f;
    w[0] = -t * tm1 * tm2 * (1.f / 6.f);
    w[1] = tp1 * tm1 * tm2 * 0.5f;
    w[2] = -tp1 * t * tm2 * 0.5f;
    w[3] = tp1 * t * tm1 * (1.f / 6.f);
}

// The interpolant at coil-frame (x, y) and depth zr; false when the point lies outside the sampled
// box (shallower than z0, deeper than the last layers, or beyond a layer's edge).
template <int NC>
__device__ __forceinline__ bool table_lookup(const CoilTableLayer* lay, const TableArgs& tb, float x, float y, float zr,
                                             float acc[NC]) {
    using V = typename TableVec<NC>::T;
    const V* data = static_cast<const V*>(tb.data);
    if (!(zr > 0.f)) return false;
    const float zeta = logf(zr * tb.inv_z0) * tb.inv_log_step;  // 0 at layer 1
    if (!(zeta >= 0.f && zeta < static_cast<float>(tb.n_layers - 3))) return false;
    const int k0 = static_cast<int>(zeta) + 1;  // layers k0 - 1 .. k0 + 2 exist
    // The position between layers k0 and k0 + 1, from the depth relative to layer k0 (small, so the
    // logarithm keeps its digits); rounding may put it a hair outside [0, 1), which the polynomial
    // weights tolerate.
    const float zk = lay[k0].z;
    const float t = log1pf((zr - zk) / zk) * tb.inv_log_step;
    float wz[4];
    lagrange4(t, wz);
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[c] = 0.f;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const CoilTableLayer Ly = lay[k0 - 1 + a];
        const float fu = floorf(x * Ly.inv_h), fv = floorf(y * Ly.inv_h);
        const float lo = static_cast<float>(1 - Ly.half), hi = static_cast<float>(Ly.n - 3 - Ly.half);
        if (!(fu >= lo && fu <= hi && fv >= lo && fv <= hi)) return false;
        const float s = fmaf(x, Ly.inv_h, -fu), r = fmaf(y, Ly.inv_h, -fv);
        const int i0 = static_cast<int>(fu) + Ly.half, j0 = static_cast<int>(fv) + Ly.half;
        float wx[4], wy[4];
        lagrange4(s, wx);
        lagrange4(r, wy);
        const V* base = data + Ly.offset + static_cast<long long>(j0 - 1) * Ly.n + (i0 - 1);
        float la[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) la[c] = 0.f;
#pragma unroll
        for (int row = 0; row < 4; ++row) {
            const V* rp = base + static_cast<long long>(row) * Ly.n;
            float ra[NC];
#pragma unroll
            for (int c = 0; c < NC; ++c) ra[c] = 0.f;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const V v = __ldg(rp + b);
                ra[0] = fmaf(wx[b], v.x, ra[0]);
                ra[1] = fmaf(wx[b], v.y, ra[1]);
                if constexpr (NC == 3) ra[2] = fmaf(wx[b], v.z, ra[2]);
            }
#pragma unroll
            for (int c = 0; c < NC; ++c) la[c] = fmaf(wy[row], ra[c], la[c]);
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[c] = fmaf(wz[a], la[c], acc[c]);
    }
    return true;
}

// Coil-frame position of node i under transform Tp (rotation columns = coil axes, translation in
// mm), formed in FP64 and rounded once; R receives the rotation.
__device__ __forceinline__ void coil_frame(const double* __restrict__ nodes_mm, int i, const double* __restrict__ Tp,
                                           double R[3][3], float& px, float& py, float& pz) {
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) R[a][b] = Tp[4 * a + b];
    double d[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) d[a] = nodes_mm[3 * static_cast<long>(i) + a] * 1e-3 - Tp[4 * a + 3] * 1e-3;
    px = static_cast<float>(R[0][0] * d[0] + R[1][0] * d[1] + R[2][0] * d[2]);
    py = static_cast<float>(R[0][1] * d[0] + R[1][1] * d[1] + R[2][1] * d[2]);
    pz = static_cast<float>(R[0][2] * d[0] + R[1][2] * d[1] + R[2][2] * d[2]);
}

// One thread per (node, placement), q = p * N + i, walked by a grid of any size in warp-uniform
// strides. Nodes the table covers get A = scale * R A'; the rest are appended to their placement's
// list, one atomic per placement per warp.
template <int NC>
__global__ void __launch_bounds__(kTableThreads) dadt_table_kernel(const double* __restrict__ nodes_mm, int n_nodes,
                                                                   const double* __restrict__ T, int k, TableArgs tb,
                                                                   float scale, float* __restrict__ out,
                                                                   int* __restrict__ near_list,
                                                                   int* __restrict__ near_cnt) {
    __shared__ CoilTableLayer lay[kCoilTableMaxLayers];
    for (int j = threadIdx.x; j < tb.n_layers; j += blockDim.x) lay[j] = tb.layers[j];
    __syncthreads();
    const long long total = static_cast<long long>(n_nodes) * k;
    const int lane = threadIdx.x & 31;
    for (long long base = static_cast<long long>(blockIdx.x) * blockDim.x; base < total;
         base += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long q = base + threadIdx.x;
        const bool valid = q < total;
        int p = 0, i = 0;
        bool near = false;
        if (valid) {
            p = static_cast<int>(q / n_nodes);
            i = static_cast<int>(q - static_cast<long long>(p) * n_nodes);
            double R[3][3];
            float px, py, pz;
            coil_frame(nodes_mm, i, T + 16 * static_cast<long>(p), R, px, py, pz);
            float acc[NC];
            if (table_lookup<NC>(lay, tb, px, py, pz - tb.z_top, acc)) {
                float* o = out + (static_cast<long long>(p) * n_nodes + i) * 3;
                if constexpr (NC == 2) {
                    const float a0 = scale * acc[0], a1 = scale * acc[1];
                    o[0] = static_cast<float>(R[0][0]) * a0 + static_cast<float>(R[0][1]) * a1;
                    o[1] = static_cast<float>(R[1][0]) * a0 + static_cast<float>(R[1][1]) * a1;
                    o[2] = static_cast<float>(R[2][0]) * a0 + static_cast<float>(R[2][1]) * a1;
                } else {
                    const float a0 = scale * acc[0], a1 = scale * acc[1], a2 = scale * acc[2];
#pragma unroll
                    for (int r = 0; r < 3; ++r)
                        o[r] = static_cast<float>(R[r][0]) * a0 + static_cast<float>(R[r][1]) * a1 +
                               static_cast<float>(R[r][2]) * a2;
                }
            } else {
                near = true;
            }
        }
        const unsigned want = __ballot_sync(0xffffffffu, near);
        if (want) {
            const unsigned same = __match_any_sync(0xffffffffu, p);
            if (near) {
                const unsigned grp = same & want;
                const int leader = __ffs(grp) - 1;
                int at = 0;
                if (lane == leader) at = atomicAdd(near_cnt + p, __popc(grp));
                at = __shfl_sync(grp, at, leader);
                near_list[static_cast<long long>(p) * n_nodes + at + __popc(grp & ((1u << lane) - 1u))] = i;
            }
        }
    }
}

__device__ __forceinline__ float2 f2sub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }

// Items (tile of 64 listed nodes, placement), tile-major so that the occupied tiles of every
// placement come first; a tile past its placement's count is skipped (uniformly per block). Lane l of
// every warp carries the tile's nodes l and l + 32 as one float2 pair (packed FP32 arithmetic); warp
// w sums dipoles [w * chunk, (w + 1) * chunk) through a 32-dipole shared-memory stage, and a stage
// whose dipoles share their plane and moment (a figure-8 wing) takes the 8-operation form of
// dadt_zcoil_kernel; warp 0 adds the eight partial sums in warp order.
__global__ void __launch_bounds__(32 * kNearWarps) dadt_near_zcoil_kernel(
    const double* __restrict__ nodes_mm, int n_nodes, const ZDipolePacked* __restrict__ dip, int n_dip,
    const double* __restrict__ T, int k, float scale, float* __restrict__ out, const int* __restrict__ near_list,
    const int* __restrict__ near_cnt) {
    __shared__ ZDipolePacked stage[kNearWarps][32];
    __shared__ float part[kNearWarps][2][64];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int chunk = (n_dip + kNearWarps - 1) / kNearWarps;
    const int j_lo = min(n_dip, w * chunk), j_hi = min(n_dip, j_lo + chunk);
    const int tiles = (n_nodes + 63) / 64;
    for (int item = blockIdx.x; item < tiles * k; item += gridDim.x) {
        const int tile = item / k, p = item - tile * k;
        const int cnt = near_cnt[p];
        if (tile * 64 >= cnt) continue;
        const int e0 = tile * 64 + lane, e1 = e0 + 32;
        const int* lp = near_list + static_cast<long long>(p) * n_nodes;
        const int i0 = lp[e0 < cnt ? e0 : tile * 64], i1 = lp[e1 < cnt ? e1 : tile * 64];
        const double* Tp = T + 16 * static_cast<long>(p);
        float2 rx, ry, rz;
        {
            double R[3][3];
            float px0, py0, pz0, px1, py1, pz1;
            coil_frame(nodes_mm, i0, Tp, R, px0, py0, pz0);
            coil_frame(nodes_mm, i1, Tp, R, px1, py1, pz1);
            rx = make_float2(px0, px1);
            ry = make_float2(py0, py1);
            rz = make_float2(pz0, pz1);
        }
        float2 ax = make_float2(0.f, 0.f), ay = ax;
        for (int t0 = j_lo; t0 < j_hi; t0 += 32) {
            const int nt = min(32, j_hi - t0);
            __syncwarp();
            if (lane < nt) stage[w][lane] = dip[t0 + lane];
            __syncwarp();
            const float z_first = stage[w][0].sz.x, m_first = stage[w][0].m.x;
            const bool same = lane >= nt || (stage[w][lane].sz.x == z_first && stage[w][lane].m.x == m_first);
            if (__all_sync(0xffffffffu, same)) {
                const float2 dz = f2sub(rz, stage[w][0].sz);
                const float2 zz = __fmul2_rn(dz, dz);
                float2 tx = make_float2(0.f, 0.f), ty = tx;
                for (int j = 0; j < nt; ++j) {
                    const ZDipolePacked d = stage[w][j];
                    const float2 dx = f2sub(rx, d.sx), dy = f2sub(ry, d.sy);
                    const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, zz));
                    const float2 inv = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
                    const float2 w3 = __fmul2_rn(inv, __fmul2_rn(inv, inv));
                    tx = __ffma2_rn(w3, dy, tx);
                    ty = __ffma2_rn(w3, dx, ty);
                }
                const float2 mt = stage[w][0].m;
                ax = __ffma2_rn(mt, tx, ax);
                ay = __ffma2_rn(mt, ty, ay);
            } else {
                for (int j = 0; j < nt; ++j) {
                    const ZDipolePacked d = stage[w][j];
                    const float2 dx = f2sub(rx, d.sx), dy = f2sub(ry, d.sy), dz = f2sub(rz, d.sz);
                    const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
                    const float2 inv = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
                    const float2 wm = __fmul2_rn(__fmul2_rn(inv, d.m), __fmul2_rn(inv, inv));
                    ax = __ffma2_rn(wm, dy, ax);
                    ay = __ffma2_rn(wm, dx, ay);
                }
            }
        }
        part[w][0][lane] = ax.x;
        part[w][0][lane + 32] = ax.y;
        part[w][1][lane] = ay.x;
        part[w][1][lane + 32] = ay.y;
        __syncthreads();
        if (w == 0) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int e = h == 0 ? e0 : e1;
                if (e >= cnt) continue;
                const int slot = lane + 32 * h;
                float sx = 0.f, sy = 0.f;
#pragma unroll
                for (int u = 0; u < kNearWarps; ++u) {
                    sx += part[u][0][slot];
                    sy += part[u][1][slot];
                }
                // A' = (-sum wm dy, sum wm dx, 0); A = R A' (rotation columns = coil axes, Tp[4a + b]).
                const float a0 = -scale * sx, a1 = scale * sy;
                float* o = out + (static_cast<long long>(p) * n_nodes + (h == 0 ? i0 : i1)) * 3;
#pragma unroll
                for (int r = 0; r < 3; ++r)
                    o[r] = static_cast<float>(Tp[4 * r]) * a0 + static_cast<float>(Tp[4 * r + 1]) * a1;
            }
        }
        __syncthreads();
    }
}

// The general-moment form: dipoles already rotated into the head frame per placement
// (prep_dipoles), the node taken relative to the coil origin; same items and warp split.
__global__ void __launch_bounds__(32 * kNearWarps) dadt_near_general_kernel(
    const double* __restrict__ nodes_mm, int n_nodes, const DipolePacked* __restrict__ dip, int n_dip,
    const double* __restrict__ T, int k, float scale, float* __restrict__ out, const int* __restrict__ near_list,
    const int* __restrict__ near_cnt) {
    __shared__ float part[kNearWarps][3][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int chunk = (n_dip + kNearWarps - 1) / kNearWarps;
    const int j_lo = min(n_dip, w * chunk), j_hi = min(n_dip, j_lo + chunk);
    const int tiles = (n_nodes + 31) / 32;
    for (int item = blockIdx.x; item < tiles * k; item += gridDim.x) {
        const int tile = item / k, p = item - tile * k;
        const int cnt = near_cnt[p];
        if (tile * 32 >= cnt) continue;
        const int e = tile * 32 + lane;
        const bool valid = e < cnt;
        const int* lp = near_list + static_cast<long long>(p) * n_nodes;
        const int i = lp[valid ? e : tile * 32];
        const double* Tp = T + 16 * static_cast<long>(p);
        const float rx = static_cast<float>(nodes_mm[3 * static_cast<long>(i)] * 1e-3 - Tp[3] * 1e-3);
        const float ry = static_cast<float>(nodes_mm[3 * static_cast<long>(i) + 1] * 1e-3 - Tp[7] * 1e-3);
        const float rz = static_cast<float>(nodes_mm[3 * static_cast<long>(i) + 2] * 1e-3 - Tp[11] * 1e-3);
        float ax = 0.f, ay = 0.f, az = 0.f;
        const float4* d4 = reinterpret_cast<const float4*>(dip + static_cast<long long>(p) * n_dip);
        for (int j = j_lo; j < j_hi; ++j) {
            const float4 f0 = __ldg(d4 + 3 * j);      // sx.x sx.y sy.x sy.y
            const float4 f1 = __ldg(d4 + 3 * j + 1);  // sz.x sz.y mx.x mx.y
            const float4 f2 = __ldg(d4 + 3 * j + 2);  // my.x my.y mz.x mz.y
            const float dx = rx - f0.x, dy = ry - f0.z, dz = rz - f1.x;
            const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const float inv = rsqrtf(d2);
            const float wgt = (inv * inv) * inv;
            const float mx = f1.z, my = f2.x, mz = f2.z;
            ax = fmaf(wgt, fmaf(my, dz, -mz * dy), ax);
            ay = fmaf(wgt, fmaf(mz, dx, -mx * dz), ay);
            az = fmaf(wgt, fmaf(mx, dy, -my * dx), az);
        }
        part[w][0][lane] = ax;
        part[w][1][lane] = ay;
        part[w][2][lane] = az;
        __syncthreads();
        if (w == 0 && valid) {
            float s[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int u = 0; u < kNearWarps; ++u)
#pragma unroll
                for (int c = 0; c < 3; ++c) s[c] += part[u][c][lane];
            float* o = out + (static_cast<long long>(p) * n_nodes + i) * 3;
#pragma unroll
            for (int c = 0; c < 3; ++c) o[c] = scale * s[c];
        }
        __syncthreads();
    }
}

// Sample positions (mm, coil frame) of every table point: layer found by bisection of the offsets.
__global__ void table_points_kernel(const CoilTableLayer* __restrict__ lay, int n_layers, long long points,
                                    double z_top, double* __restrict__ out_mm) {
    const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= points) return;
    int lo = 0, hi = n_layers - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (lay[mid].offset <= q) lo = mid;
        else hi = mid - 1;
    }
    const CoilTableLayer L = lay[lo];
    const long long loc = q - L.offset;
    const int iy = static_cast<int>(loc / L.n), ix = static_cast<int>(loc - static_cast<long long>(iy) * L.n);
    const double ih = static_cast<double>(L.inv_h);
    out_mm[3 * q] = static_cast<double>(ix - L.half) / ih * 1e3;
    out_mm[3 * q + 1] = static_cast<double>(iy - L.half) / ih * 1e3;
    out_mm[3 * q + 2] = (z_top + static_cast<double>(L.z)) * 1e3;
}

__global__ void table_pack_kernel(const float* __restrict__ a3, long long points, int nc, float* __restrict__ data) {
    const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= points) return;
    if (nc == 2) {
        data[2 * q] = a3[3 * q];
        data[2 * q + 1] = a3[3 * q + 1];
    } else {
        data[4 * q] = a3[3 * q];
        data[4 * q + 1] = a3[3 * q + 1];
        data[4 * q + 2] = a3[3 * q + 2];
        data[4 * q + 3] = 0.f;
    }
}

// The interpolant at coil-frame points (mm); NaN where the table does not cover the point.
template <int NC>
__global__ void table_probe_kernel(TableArgs tb, const double* __restrict__ pts_mm, int n, float* __restrict__ out3) {
    __shared__ CoilTableLayer lay[kCoilTableMaxLayers];
    for (int j = threadIdx.x; j < tb.n_layers; j += blockDim.x) lay[j] = tb.layers[j];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float px = static_cast<float>(pts_mm[3 * i] * 1e-3), py = static_cast<float>(pts_mm[3 * i + 1] * 1e-3);
    const float pz = static_cast<float>(pts_mm[3 * i + 2] * 1e-3);
    float acc[NC];
    const bool ok = table_lookup<NC>(lay, tb, px, py, pz - tb.z_top, acc);
    const float nan = __int_as_float(0x7fffffff);
    out3[3 * i] = ok ? acc[0] : nan;
    out3[3 * i + 1] = ok ? acc[1] : nan;
    if constexpr (NC == 3) out3[3 * i + 2] = ok ? acc[2] : nan;
    else out3[3 * i + 2] = 0.f;
}

__global__ void coil_compare_kernel(const double* __restrict__ pos, const double* __restrict__ mom,
                                    const double* __restrict__ tpos, const double* __restrict__ tmom, int n,
                                    int* __restrict__ flag) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const bool diff = q < n && (pos[q] != tpos[q] || mom[q] != tmom[q]);
    if (__syncthreads_or(diff) && threadIdx.x == 0) atomicOr(flag, 2);
}

TableArgs table_args(const CoilTable& tb) {
    TableArgs a;
    a.layers = tb.layers.get();
    a.data = tb.data.get();
    a.n_layers = tb.n_layers;
    a.z_top = tb.z_top;
    a.inv_z0 = tb.inv_z0;
    a.inv_log_step = tb.inv_log_step;
    return a;
}

int bounded(long long items, int max_blocks, int cap) {
    const long long b = max_blocks > 0 ? std::min<long long>(items, max_blocks) : std::min<long long>(items, cap);
    return static_cast<int>(std::max<long long>(b, 1));
}

// The bare dipole sum (scale 1, identity transform) at n points given in mm.
void direct_at(const double* pts_mm, long long n, const double* pos, const double* mom, int n_dip, bool zcoil,
               const void* zpacked, float* out3, cudaStream_t s) {
    DevArray<double> ident(16);
    const double I[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    CUNIBS_CHECK(cudaMemcpyAsync(ident.get(), I, sizeof I, cudaMemcpyHostToDevice, s));
    if (zcoil) {
        dadt_zcoil_raw(pts_mm, static_cast<int>(n), zpacked, n_dip, ident.get(), 1, 1.0f, out3, s);
    } else {
        DevArray<unsigned char> packed(packed_dipole_bytes() * static_cast<std::size_t>(n_dip));
        prep_dipoles(pos, mom, n_dip, ident.get(), 1, packed.get(), s);
        dadt_general_raw(pts_mm, static_cast<int>(n), reinterpret_cast<const float*>(packed.get()), n_dip, ident.get(),
                         1, 1.0f, out3, s);
        CUNIBS_CHECK(cudaStreamSynchronize(s));  // before the packed records are freed
    }
    CUNIBS_CHECK(cudaStreamSynchronize(s));      // before the transform is freed
}

}  // namespace

void coil_compare(const double* pos, const double* mom, int n_dip, const CoilTable& tb, int* flag, cudaStream_t s) {
    const int n = 3 * n_dip;
    coil_compare_kernel<<<grid_for(n), kBlock, 0, s>>>(pos, mom, tb.pos.get(), tb.mom.get(), n, flag);
    count_launch();
    CUNIBS_LAUNCH_CHECK("coil compare");
}

void build_coil_table(CoilTable& tb, const double* pos, const double* mom, int n_dip, bool zcoil, const void* zpacked,
                      double near_m, double step, double lateral_m, double depth_m, long long max_points,
                      cudaStream_t s) {
    if (n_dip <= 0) fail(kEInval, "a coil needs dipoles");
    if (!(near_m > 0.0 && step > 0.0 && step <= 0.5)) fail(kEInval, "coil table: near depth > 0 and 0 < step <= 0.5");
    tb.built = tb.valid = false;
    ++tb.builds;
    tb.nc = zcoil ? 2 : 3;
    tb.n_dip = n_dip;
    tb.near_m = near_m;
    tb.step = step;
    tb.lateral_m = lateral_m;
    tb.check_rel = 0.0;
    tb.pos.resize(3 * static_cast<std::size_t>(n_dip));
    tb.mom.resize(3 * static_cast<std::size_t>(n_dip));
    CUNIBS_CHECK(cudaMemcpyAsync(tb.pos.get(), pos, sizeof(double) * 3 * n_dip, cudaMemcpyDeviceToDevice, s));
    CUNIBS_CHECK(cudaMemcpyAsync(tb.mom.get(), mom, sizeof(double) * 3 * n_dip, cudaMemcpyDeviceToDevice, s));
    std::vector<double> hp(3 * static_cast<std::size_t>(n_dip));
    CUNIBS_CHECK(cudaMemcpyAsync(hp.data(), pos, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, s));
    CUNIBS_CHECK(cudaStreamSynchronize(s));
    double zt = hp[2];
    for (int j = 1; j < n_dip; ++j) zt = std::max(zt, hp[3 * static_cast<std::size_t>(j) + 2]);
    tb.z_top = static_cast<float>(zt);
    tb.z0 = static_cast<float>(near_m);
    tb.inv_z0 = 1.0f / tb.z0;
    tb.inv_log_step = static_cast<float>(1.0 / std::log1p(step));

    // Layers: one above z0 for the stencil, then enough to reach depth_m with two to spare.
    const int want = static_cast<int>(std::ceil(std::log(std::max(depth_m, 2.0 * near_m) / near_m) / std::log1p(step))) + 4;
    const int L = std::min(kCoilTableMaxLayers, want);
    std::vector<CoilTableLayer> lay(L);
    long long off = 0;
    for (int j = 0; j < L; ++j) {
        const double zj = near_m * std::pow(1.0 + step, j - 1);
        CoilTableLayer& y = lay[j];
        y.z = static_cast<float>(zj);
        y.inv_h = static_cast<float>(1.0 / (step * static_cast<double>(y.z)));
        y.half = static_cast<int>(std::ceil(lateral_m * static_cast<double>(y.inv_h))) + 2;
        y.n = 2 * y.half + 1;
        y.offset = off;
        off += static_cast<long long>(y.n) * y.n;
    }
    tb.n_layers = L;
    tb.points = off;
    tb.built = true;
    if (off > max_points || L < 5) return;  // too large (or too shallow) to be worth it: direct sums
    tb.layers.upload(lay.data(), lay.size(), s);
    tb.data.resize(static_cast<std::size_t>(off) * (tb.nc == 2 ? 2 : 4));

    {
        DevArray<double> pts(3 * static_cast<std::size_t>(off));
        DevArray<float> a3(3 * static_cast<std::size_t>(off));
        table_points_kernel<<<grid_for(off), kBlock, 0, s>>>(tb.layers.get(), L, off, static_cast<double>(tb.z_top),
                                                             pts.get());
        count_launch();
        CUNIBS_LAUNCH_CHECK("coil table points");
        direct_at(pts.get(), off, pos, mom, n_dip, zcoil, zpacked, a3.get(), s);
        table_pack_kernel<<<grid_for(off), kBlock, 0, s>>>(a3.get(), off, tb.nc, tb.data.get());
        count_launch();
        CUNIBS_LAUNCH_CHECK("coil table pack");
        CUNIBS_CHECK(cudaStreamSynchronize(s));
    }

    // Check points: the middle of a grid cell of layer j in all three coordinates, j over the
    // layers whose stencils exist, laterally anywhere within the sampled half-width.
    std::vector<double> cp(3 * kCheckPoints);
    std::uint64_t st = 0x9e3779b97f4a7c15ull;
    auto next = [&st]() {
        st ^= st << 13;
        st ^= st >> 7;
        st ^= st << 17;
        return static_cast<double>(st >> 11) * (1.0 / 9007199254740992.0);
    };
    for (int c = 0; c < kCheckPoints; ++c) {
        const int j = 1 + c % (L - 4);
        const CoilTableLayer& y = lay[j];
        const double ih = static_cast<double>(y.inv_h);
        const double lim = std::floor(lateral_m * ih) - 1.0;
        const double u = std::floor((2.0 * next() - 1.0) * lim), v = std::floor((2.0 * next() - 1.0) * lim);
        const double zr = near_m * std::pow(1.0 + step, (j - 1) + 0.5);
        cp[3 * c] = (u + 0.5) / ih * 1e3;
        cp[3 * c + 1] = (v + 0.5) / ih * 1e3;
        cp[3 * c + 2] = (static_cast<double>(tb.z_top) + zr) * 1e3;
    }
    DevArray<double> cpd;
    cpd.upload(cp.data(), cp.size(), s);
    DevArray<float> ref(3 * kCheckPoints), est(3 * kCheckPoints);
    direct_at(cpd.get(), kCheckPoints, pos, mom, n_dip, zcoil, zpacked, ref.get(), s);
    const TableArgs ta = table_args(tb);
    if (tb.nc == 2) table_probe_kernel<2><<<grid_for(kCheckPoints), kBlock, 0, s>>>(ta, cpd.get(), kCheckPoints, est.get());
    else table_probe_kernel<3><<<grid_for(kCheckPoints), kBlock, 0, s>>>(ta, cpd.get(), kCheckPoints, est.get());
    count_launch();
    CUNIBS_LAUNCH_CHECK("coil table probe");
    std::vector<float> hr(3 * kCheckPoints), he(3 * kCheckPoints);
    ref.download(hr.data(), hr.size(), s);
    est.download(he.data(), he.size(), s);
    CUNIBS_CHECK(cudaStreamSynchronize(s));
    double num = 0.0, den = 0.0;
    for (std::size_t q = 0; q < hr.size(); ++q) {
        const double d = static_cast<double>(he[q]) - static_cast<double>(hr[q]);
        num += d * d;
        den += static_cast<double>(hr[q]) * hr[q];
    }
    tb.check_rel = den > 0.0 ? std::sqrt(num / den) : (num == 0.0 ? 0.0 : INFINITY);
    tb.valid = std::isfinite(tb.check_rel) && tb.check_rel <= kCheckTolerance;
}

void dadt_table(const Mesh& m, const CoilTable& tb, const double* transforms_dev, int k, double didt, float* out,
                int* near_list, int* near_cnt, cudaStream_t s, int max_blocks) {
    if (!tb.valid) fail(kEInval, "the coil table is not usable");
    CUNIBS_CHECK(cudaMemsetAsync(near_cnt, 0, sizeof(int) * k, s));
    const long long total = static_cast<long long>(m.n_nodes) * k;
    const int blocks = bounded((total + kTableThreads - 1) / kTableThreads, max_blocks, 8192);
    const float scale = static_cast<float>(didt * 1e-7);
    const TableArgs ta = table_args(tb);
    if (tb.nc == 2)
        dadt_table_kernel<2><<<blocks, kTableThreads, 0, s>>>(m.nodes.get(), m.n_nodes, transforms_dev, k, ta, scale, out,
                                                              near_list, near_cnt);
    else
        dadt_table_kernel<3><<<blocks, kTableThreads, 0, s>>>(m.nodes.get(), m.n_nodes, transforms_dev, k, ta, scale, out,
                                                              near_list, near_cnt);
    count_launch();
    CUNIBS_LAUNCH_CHECK("dadt table");
}

void dadt_near_zcoil(const Mesh& m, const void* zpacked, int n_dip, const double* transforms_dev, int k, double didt,
                     float* out, const int* near_list, const int* near_cnt, cudaStream_t s, int max_blocks) {
    const long long items = static_cast<long long>((m.n_nodes + 63) / 64) * k;
    dadt_near_zcoil_kernel<<<bounded(items, max_blocks, 1184), 32 * kNearWarps, 0, s>>>(
        m.nodes.get(), m.n_nodes, static_cast<const ZDipolePacked*>(zpacked), n_dip, transforms_dev, k,
        static_cast<float>(didt * 1e-7), out, near_list, near_cnt);
    count_launch();
    CUNIBS_LAUNCH_CHECK("dadt near z-coil");
}

void dadt_near_general(const Mesh& m, const float* dip_packed, int n_dip, const double* transforms_dev, int k,
                       double didt, float* out, const int* near_list, const int* near_cnt, cudaStream_t s,
                       int max_blocks) {
    const long long items = static_cast<long long>((m.n_nodes + 31) / 32) * k;
    dadt_near_general_kernel<<<bounded(items, max_blocks, 4096), 32 * kNearWarps, 0, s>>>(
        m.nodes.get(), m.n_nodes, reinterpret_cast<const DipolePacked*>(dip_packed), n_dip, transforms_dev, k,
        static_cast<float>(didt * 1e-7), out, near_list, near_cnt);
    count_launch();
    CUNIBS_LAUNCH_CHECK("dadt near");
}

}  // namespace cunibs
