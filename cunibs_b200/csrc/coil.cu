// Coil dA/dt at the mesh nodes, its element average, and the k-wide FEM right-hand side.
//
// dA/dt(r) = didt * mu0/4pi * sum_j m_j x (r - s_j) / |r - s_j|^3   (fem/placement.py:279-317).
//
// The N-body sum is the hot part: N nodes x D dipoles x k placements pair evaluations. Each block
// stages a tile of one placement's dipoles in shared memory (positions and moments already rotated
// into the head frame and centred on the coil origin in FP64, then rounded to FP32, as the reference
// does to keep |r - s|^2 free of cancellation), and every thread carries four nodes as two float2
// pairs so the arithmetic issues as sm_100 packed FP32 instructions (FFMA2/FADD2/FMUL2): two node
// evaluations per instruction. The difference r - s is formed directly rather than through
// |r|^2 + |s|^2 - 2 r.s, which costs no more here and loses nothing to cancellation.
#include <algorithm>
#include <cstdint>

#include "coil_packed.cuh"
#include "internal.hpp"

namespace cunibs {
namespace {

constexpr int kDadtThreads = 128;
constexpr int kDipTile = 256;

// Per (placement, dipole): s' = R pos (metres), m' = R mom, where R is the transform's rotation.
// The translation cancels against the centring at the coil origin.
__global__ void prep_dipoles_kernel(const double* __restrict__ pos, const double* __restrict__ mom, int n_dip,
                                    const double* __restrict__ T, int k, DipolePacked* __restrict__ out) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<long>(n_dip) * k) return;
    const int p = static_cast<int>(q / n_dip);
    const int j = static_cast<int>(q % n_dip);
    const double* R = T + 16 * static_cast<long>(p);
    double s[3], m[3];
    for (int a = 0; a < 3; ++a) {
        s[a] = R[4 * a] * pos[3 * j] + R[4 * a + 1] * pos[3 * j + 1] + R[4 * a + 2] * pos[3 * j + 2];
        m[a] = R[4 * a] * mom[3 * j] + R[4 * a + 1] * mom[3 * j + 1] + R[4 * a + 2] * mom[3 * j + 2];
    }
    DipolePacked d;
    d.sx = make_float2(static_cast<float>(s[0]), static_cast<float>(s[0]));
    d.sy = make_float2(static_cast<float>(s[1]), static_cast<float>(s[1]));
    d.sz = make_float2(static_cast<float>(s[2]), static_cast<float>(s[2]));
    d.mx = make_float2(static_cast<float>(m[0]), static_cast<float>(m[0]));
    d.my = make_float2(static_cast<float>(m[1]), static_cast<float>(m[1]));
    d.mz = make_float2(static_cast<float>(m[2]), static_cast<float>(m[2]));
    out[q] = d;
}

__device__ __forceinline__ float2 f2neg(float2 a) { return make_float2(-a.x, -a.y); }

// Work items are (node tile, placement) pairs, item = p * n_tiles + tile, walked by a grid of any
// size (a bounded grid leaves room on every SM for kernels of other streams). Node i of this thread
// in a tile: tile * threads + threadIdx + {0, 1, 2, 3} * n_tiles * threads, paired as (0, 1) and
// (2, 3) into float2 lanes; the per-node arithmetic does not depend on the grid.
__global__ void __launch_bounds__(kDadtThreads) dadt_kernel(const double* __restrict__ nodes_mm, int n_nodes,
                                                            const DipolePacked* __restrict__ dip, int n_dip,
                                                            const double* __restrict__ T, float scale,
                                                            float* __restrict__ out, int n_tiles, int n_items) {
    __shared__ DipolePacked tile[kDipTile];
    for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int p = item / n_tiles;
    const double* Tp = T + 16 * static_cast<long>(p);
    const double ox = Tp[3] * 1e-3, oy = Tp[7] * 1e-3, oz = Tp[11] * 1e-3;
    const int stride = n_tiles * blockDim.x;
    const int base = (item - p * n_tiles) * blockDim.x + threadIdx.x;
    int node[4];
    float rxs[4], rys[4], rzs[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        node[u] = base + u * stride;
        const int i = node[u] < n_nodes ? node[u] : n_nodes - 1;
        rxs[u] = static_cast<float>(nodes_mm[3 * static_cast<long>(i)] * 1e-3 - ox);
        rys[u] = static_cast<float>(nodes_mm[3 * static_cast<long>(i) + 1] * 1e-3 - oy);
        rzs[u] = static_cast<float>(nodes_mm[3 * static_cast<long>(i) + 2] * 1e-3 - oz);
    }
    const float2 rx0 = make_float2(rxs[0], rxs[1]), ry0 = make_float2(rys[0], rys[1]), rz0 = make_float2(rzs[0], rzs[1]);
    const float2 rx1 = make_float2(rxs[2], rxs[3]), ry1 = make_float2(rys[2], rys[3]), rz1 = make_float2(rzs[2], rzs[3]);
    float2 ax0 = make_float2(0.f, 0.f), ay0 = ax0, az0 = ax0, ax1 = ax0, ay1 = ax0, az1 = ax0;
    const DipolePacked* dp = dip + static_cast<long>(p) * n_dip;
    for (int t0 = 0; t0 < n_dip; t0 += kDipTile) {
        const int nt = min(kDipTile, n_dip - t0);
        __syncthreads();
        for (int j = threadIdx.x; j < nt; j += blockDim.x) tile[j] = dp[t0 + j];
        __syncthreads();
#pragma unroll 2
        for (int j = 0; j < nt; ++j) {
            const DipolePacked d = tile[j];
            // pair 0
            {
                const float2 dx = __fadd2_rn(rx0, f2neg(d.sx));
                const float2 dy = __fadd2_rn(ry0, f2neg(d.sy));
                const float2 dz = __fadd2_rn(rz0, f2neg(d.sz));
                float2 d2 = __fmul2_rn(dx, dx);
                d2 = __ffma2_rn(dy, dy, d2);
                d2 = __ffma2_rn(dz, dz, d2);
                const float2 inv = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
                const float2 w = __fmul2_rn(__fmul2_rn(inv, inv), inv);
                const float2 cx = __ffma2_rn(d.my, dz, __fmul2_rn(f2neg(d.mz), dy));
                const float2 cy = __ffma2_rn(d.mz, dx, __fmul2_rn(f2neg(d.mx), dz));
                const float2 cz = __ffma2_rn(d.mx, dy, __fmul2_rn(f2neg(d.my), dx));
                ax0 = __ffma2_rn(w, cx, ax0);
                ay0 = __ffma2_rn(w, cy, ay0);
                az0 = __ffma2_rn(w, cz, az0);
            }
            // pair 1
            {
                const float2 dx = __fadd2_rn(rx1, f2neg(d.sx));
                const float2 dy = __fadd2_rn(ry1, f2neg(d.sy));
                const float2 dz = __fadd2_rn(rz1, f2neg(d.sz));
                float2 d2 = __fmul2_rn(dx, dx);
                d2 = __ffma2_rn(dy, dy, d2);
                d2 = __ffma2_rn(dz, dz, d2);
                const float2 inv = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
                const float2 w = __fmul2_rn(__fmul2_rn(inv, inv), inv);
                const float2 cx = __ffma2_rn(d.my, dz, __fmul2_rn(f2neg(d.mz), dy));
                const float2 cy = __ffma2_rn(d.mz, dx, __fmul2_rn(f2neg(d.mx), dz));
                const float2 cz = __ffma2_rn(d.mx, dy, __fmul2_rn(f2neg(d.my), dx));
                ax1 = __ffma2_rn(w, cx, ax1);
                ay1 = __ffma2_rn(w, cy, ay1);
                az1 = __ffma2_rn(w, cz, az1);
            }
        }
    }
    const float ax[4] = {ax0.x, ax0.y, ax1.x, ax1.y};
    const float ay[4] = {ay0.x, ay0.y, ay1.x, ay1.y};
    const float az[4] = {az0.x, az0.y, az1.x, az1.y};
    float* o = out + static_cast<long>(p) * n_nodes * 3;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        if (node[u] < n_nodes) {
            o[3 * static_cast<long>(node[u])] = scale * ax[u];
            o[3 * static_cast<long>(node[u]) + 1] = scale * ay[u];
            o[3 * static_cast<long>(node[u]) + 2] = scale * az[u];
        }
    }
    }
}

// ND source sets that share their positions and differ only in their moments (the mesh nodes as
// the sources of an adjoint's ND directions). One shared-memory record per source holds the
// position once and every set's moment.
template <int ND>
struct __align__(16) SharedSource {
    float2 sx, sy, sz;
    float2 m[ND][3];
};

// The field of ND source sets at common positions (records d * n_dip + j of prep_dipoles, all
// prepared with the one transform T): per (target, source) pair the difference and 1/|d|^3 are
// formed once and used for every set, with dadt_kernel's per-set arithmetic. Work items are
// (node tile, source chunk) pairs, item = chunk * n_tiles + tile, so that few targets (a grid of a
// few hundred thousand points) still fill the GPU: with one chunk a thread sums every source in
// order and writes the scaled field (dadt_kernel's order, bitwise its result for one set); with
// several it writes the chunk's unscaled partial to part[chunk][set][node][3], and
// shared_sum_kernel adds the chunks in order. The chunks depend on the sizes only, never on ND.
// Node order within a tile as dadt_kernel's.
template <int ND>
__global__ void __launch_bounds__(kDadtThreads) dadt_shared_kernel(const double* __restrict__ nodes_mm, int n_nodes,
                                                                   const DipolePacked* __restrict__ dip, int n_dip,
                                                                   const double* __restrict__ T, float scale,
                                                                   float* __restrict__ out, int n_tiles, int chunk,
                                                                   int n_items, float* __restrict__ part) {
    __shared__ SharedSource<ND> tile[kDipTile];
    const double ox = T[3] * 1e-3, oy = T[7] * 1e-3, oz = T[11] * 1e-3;
    const int stride = n_tiles * blockDim.x;
    for (int work = blockIdx.x; work < n_items; work += gridDim.x) {
    const int item = work % n_tiles, ch = work / n_tiles;
    const int j_begin = ch * chunk, j_end = min(n_dip, j_begin + chunk);
    const int base = item * blockDim.x + threadIdx.x;
    int node[4];
    float rxs[4], rys[4], rzs[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        node[u] = base + u * stride;
        const int i = node[u] < n_nodes ? node[u] : n_nodes - 1;
        rxs[u] = static_cast<float>(nodes_mm[3 * static_cast<long>(i)] * 1e-3 - ox);
        rys[u] = static_cast<float>(nodes_mm[3 * static_cast<long>(i) + 1] * 1e-3 - oy);
        rzs[u] = static_cast<float>(nodes_mm[3 * static_cast<long>(i) + 2] * 1e-3 - oz);
    }
    const float2 rx[2] = {make_float2(rxs[0], rxs[1]), make_float2(rxs[2], rxs[3])};
    const float2 ry[2] = {make_float2(rys[0], rys[1]), make_float2(rys[2], rys[3])};
    const float2 rz[2] = {make_float2(rzs[0], rzs[1]), make_float2(rzs[2], rzs[3])};
    float2 ax[ND][2], ay[ND][2], az[ND][2];
#pragma unroll
    for (int d = 0; d < ND; ++d)
#pragma unroll
        for (int q = 0; q < 2; ++q) ax[d][q] = ay[d][q] = az[d][q] = make_float2(0.f, 0.f);
    for (int t0 = j_begin; t0 < j_end; t0 += kDipTile) {
        const int nt = min(kDipTile, j_end - t0);
        __syncthreads();
        for (int j = threadIdx.x; j < nt; j += blockDim.x) {
            const DipolePacked p0 = dip[t0 + j];
            SharedSource<ND> r;
            r.sx = p0.sx;
            r.sy = p0.sy;
            r.sz = p0.sz;
#pragma unroll
            for (int d = 0; d < ND; ++d) {
                const DipolePacked pd = dip[static_cast<long>(d) * n_dip + t0 + j];
                r.m[d][0] = pd.mx;
                r.m[d][1] = pd.my;
                r.m[d][2] = pd.mz;
            }
            tile[j] = r;
        }
        __syncthreads();
        for (int j = 0; j < nt; ++j) {
            const float2 sx = tile[j].sx, sy = tile[j].sy, sz = tile[j].sz;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const float2 dx = __fadd2_rn(rx[q], f2neg(sx));
                const float2 dy = __fadd2_rn(ry[q], f2neg(sy));
                const float2 dz = __fadd2_rn(rz[q], f2neg(sz));
                float2 d2 = __fmul2_rn(dx, dx);
                d2 = __ffma2_rn(dy, dy, d2);
                d2 = __ffma2_rn(dz, dz, d2);
                const float2 inv = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
                const float2 w = __fmul2_rn(__fmul2_rn(inv, inv), inv);
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    const float2 mx = tile[j].m[d][0], my = tile[j].m[d][1], mz = tile[j].m[d][2];
                    const float2 cx = __ffma2_rn(my, dz, __fmul2_rn(f2neg(mz), dy));
                    const float2 cy = __ffma2_rn(mz, dx, __fmul2_rn(f2neg(mx), dz));
                    const float2 cz = __ffma2_rn(mx, dy, __fmul2_rn(f2neg(my), dx));
                    ax[d][q] = __ffma2_rn(w, cx, ax[d][q]);
                    ay[d][q] = __ffma2_rn(w, cy, ay[d][q]);
                    az[d][q] = __ffma2_rn(w, cz, az[d][q]);
                }
            }
        }
    }
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        const float vx[4] = {ax[d][0].x, ax[d][0].y, ax[d][1].x, ax[d][1].y};
        const float vy[4] = {ay[d][0].x, ay[d][0].y, ay[d][1].x, ay[d][1].y};
        const float vz[4] = {az[d][0].x, az[d][0].y, az[d][1].x, az[d][1].y};
        float* o = part ? part + (static_cast<long>(ch) * ND + d) * n_nodes * 3 : out + static_cast<long>(d) * n_nodes * 3;
        const float sc = part ? 1.0f : scale;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (node[u] < n_nodes) {
                o[3 * static_cast<long>(node[u])] = sc * vx[u];
                o[3 * static_cast<long>(node[u]) + 1] = sc * vy[u];
                o[3 * static_cast<long>(node[u]) + 2] = sc * vz[u];
            }
        }
    }
    }
}

// out = scale * (the chunks' partials added in chunk order).
__global__ void shared_sum_kernel(long count, int chunks, const float* __restrict__ part, float scale,
                                  float* __restrict__ out) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= count) return;
    float v = part[q];
    for (int c = 1; c < chunks; ++c) v += part[c * count + q];
    out[q] = scale * v;
}

// dadt_elm[p][e] = 1/4 sum of the four nodal values (dadt_element.cu:6-31).
__global__ void element_average_kernel(const float* __restrict__ nodal, const int* __restrict__ tets, int n_nodes,
                                       int n_tets, int k, float* __restrict__ elm) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<long>(n_tets) * k) return;
    const int p = static_cast<int>(q / n_tets);
    const int e = static_cast<int>(q % n_tets);
    const int4 tn = reinterpret_cast<const int4*>(tets)[e];
    const float* v = nodal + static_cast<long>(p) * n_nodes * 3;
    float* o = elm + static_cast<long>(p) * n_tets * 3;
#pragma unroll
    for (int a = 0; a < 3; ++a)
        o[3 * static_cast<long>(e) + a] =
            0.25f * (v[3 * static_cast<long>(tn.x) + a] + v[3 * static_cast<long>(tn.y) + a] +
                     v[3 * static_cast<long>(tn.z) + a] + v[3 * static_cast<long>(tn.w) + a]);
}

// b_red[r][c] = sum over the corners of node i of neg_vc[e] * (dadt_elm[c][e] . g[corner]),
// accumulated in FP64 in node2corner order; node i = r, skipping the grounded node. Columns past
// k repeat column k-1 (the padding of a partial block).
template <int K>
__global__ void __launch_bounds__(64 * K) rhs_kernel(const float* __restrict__ elm, const float* __restrict__ g32,
                                                     const float* __restrict__ neg_vc, const int* __restrict__ ptr,
                                                     const int* __restrict__ idx, int n_nodes, int n_tets, int k,
                                                     int ground, double* __restrict__ b_red) {
    const int r = blockIdx.x * 64 + threadIdx.x / K;
    const int c = threadIdx.x % K;
    if (r >= n_nodes - 1) return;
    const int i = r + (r >= ground ? 1 : 0);
    const int src = c < k ? c : k - 1;
    const float* el = elm + static_cast<long>(src) * n_tets * 3;
    double acc = 0.0;
    for (int q = ptr[i]; q < ptr[i + 1]; ++q) {
        const int corner = idx[q];
        const int e = corner >> 2;
        const float* gc = g32 + 3 * static_cast<long>(corner);
        const double d = static_cast<double>(el[3 * static_cast<long>(e)]) * gc[0] +
                         static_cast<double>(el[3 * static_cast<long>(e) + 1]) * gc[1] +
                         static_cast<double>(el[3 * static_cast<long>(e) + 2]) * gc[2];
        acc += static_cast<double>(neg_vc[e]) * d;
    }
    b_red[static_cast<long>(r) * K + c] = acc;
}

// w_ij = sum over entry (i, j)'s element contributions (ascending element) of 1/4 neg_vc[e] g[e, i]:
// b_i = sum_{corners of i} neg_vc[e] (1/4 sum_{n in e} A_n) . g[e, i] = sum_j w_ij . A_j.
__global__ void rhs_weights_kernel(const float* __restrict__ g32, const float* __restrict__ neg_vc,
                                   const int* __restrict__ contrib_ptr, const int* __restrict__ contrib_idx, long nnz,
                                   float* __restrict__ w) {
    const long p = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= nnz) return;
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int q = contrib_ptr[p], end = contrib_ptr[p + 1]; q < end; ++q) {
        const int idx = contrib_idx[q];
        const long e = idx >> 4;
        const float* gi = g32 + 12 * e + 3 * ((idx >> 2) & 3);
        const double sv = 0.25 * static_cast<double>(neg_vc[e]);
        ax += sv * static_cast<double>(gi[0]);
        ay += sv * static_cast<double>(gi[1]);
        az += sv * static_cast<double>(gi[2]);
    }
    w[3 * p] = static_cast<float>(ax);
    w[3 * p + 1] = static_cast<float>(ay);
    w[3 * p + 2] = static_cast<float>(az);
}

// b_red[r][c] = sum over row i's stiffness entries of w_ij . dadt_nodes[c][j] in FP64 (entry
// order), i = r skipping the grounded node; columns past k repeat column k-1.
template <int K>
__global__ void __launch_bounds__(64 * K) rhs_nodes_kernel(const float* __restrict__ nodal, const float* __restrict__ w,
                                                           const int* __restrict__ ptr, const int* __restrict__ col,
                                                           int n_nodes, int k, int ground, double* __restrict__ b_red) {
    const int r = blockIdx.x * 64 + threadIdx.x / K;
    const int c = threadIdx.x % K;
    if (r >= n_nodes - 1) return;
    const int i = r + (r >= ground ? 1 : 0);
    const int src = c < k ? c : k - 1;
    const float* a = nodal + static_cast<long>(src) * n_nodes * 3;
    double acc = 0.0;
    for (int q = ptr[i]; q < ptr[i + 1]; ++q) {
        const long j = col[q];
        const float* wq = w + 3 * static_cast<long>(q);
        acc += static_cast<double>(wq[0]) * a[3 * j] + static_cast<double>(wq[1]) * a[3 * j + 1] +
               static_cast<double>(wq[2]) * a[3 * j + 2];
    }
    b_red[static_cast<long>(r) * K + c] = acc;
}

}  // namespace

void prep_dipoles(const double* pos, const double* mom, int n_dip, const double* transforms_dev, int k, void* out,
                  cudaStream_t s) {
    const long total = static_cast<long>(n_dip) * k;
    prep_dipoles_kernel<<<grid_for(total), kBlock, 0, s>>>(pos, mom, n_dip, transforms_dev, k,
                                                           static_cast<DipolePacked*>(out)); count_launch();
    CUNIBS_LAUNCH_CHECK("prep dipoles");
}

std::size_t packed_dipole_bytes() { return sizeof(DipolePacked); }

namespace {

// Tiles of 4 * threads nodes; the grid is one block per (tile, placement) item, or max_blocks
// blocks walking the items when max_blocks > 0.
struct DadtGrid {
    int n_tiles, n_items, blocks;
};

DadtGrid dadt_grid(int n_nodes, int k, int max_blocks) {
    const int per_block = 4 * kDadtThreads;
    DadtGrid g;
    g.n_tiles = (n_nodes + per_block - 1) / per_block;
    g.n_items = g.n_tiles * k;
    g.blocks = max_blocks > 0 ? std::min(g.n_items, max_blocks) : g.n_items;
    return g;
}

}  // namespace

void dadt_nodes(const Mesh& m, const float* dip_packed, int n_dip, const double* transforms_dev, int k, double didt,
                float* out, cudaStream_t s, int max_blocks) {
    const DadtGrid g = dadt_grid(m.n_nodes, k, max_blocks);
    dadt_kernel<<<g.blocks, kDadtThreads, 0, s>>>(m.nodes.get(), m.n_nodes,
                                                 reinterpret_cast<const DipolePacked*>(dip_packed), n_dip,
                                                 transforms_dev, static_cast<float>(didt * 1e-7), out, g.n_tiles,
                                                 g.n_items);
    count_launch();
    CUNIBS_LAUNCH_CHECK("dadt");
}

void dadt_nodes_raw(const double* nodes_mm, int n_nodes, const float* dip_packed, int n_dip,
                    const double* transforms_dev, int k, double didt, float* out, cudaStream_t s) {
    const DadtGrid g = dadt_grid(n_nodes, k, 0);
    dadt_kernel<<<g.blocks, kDadtThreads, 0, s>>>(nodes_mm, n_nodes, reinterpret_cast<const DipolePacked*>(dip_packed),
                                                 n_dip, transforms_dev, static_cast<float>(didt * 1e-7), out,
                                                 g.n_tiles, g.n_items);
    count_launch();
}

void dadt_nodes_shared(const double* nodes_mm, int n_nodes, const float* dip_packed, int n_dip,
                       const double* transform_dev, int n_sets, double didt, float* out, cudaStream_t s,
                       DevArray<float>& scratch) {
    const DadtGrid g = dadt_grid(n_nodes, 1, 0);
    const float scale = static_cast<float>(didt * 1e-7);
    const auto* dp = reinterpret_cast<const DipolePacked*>(dip_packed);
    if (n_sets < 1 || n_sets > 3) fail(kEInval, "between 1 and 3 source sets");
    // Source chunks: about two waves of resident blocks when the targets alone leave the GPU short
    // of them (kDipTile-multiples of sources, at least one tile each); one chunk otherwise.
    int dev = 0, sms = 0;
    CUNIBS_CHECK(cudaGetDevice(&dev));
    CUNIBS_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int resident = sms * (2048 / kDadtThreads);
    int chunks = 1;
    if (g.n_tiles < resident) chunks = std::min((2 * resident + g.n_tiles - 1) / g.n_tiles, (n_dip + kDipTile - 1) / kDipTile);
    chunks = std::max(chunks, 1);
    const int chunk = ((n_dip + chunks - 1) / chunks + kDipTile - 1) / kDipTile * kDipTile;
    chunks = (n_dip + chunk - 1) / chunk;
    const int n_items = g.n_tiles * chunks;
    if (chunks > 1) scratch.reserve(static_cast<std::size_t>(chunks) * n_sets * n_nodes * 3);
    float* pp = chunks > 1 ? scratch.get() : nullptr;
    switch (n_sets) {
        case 1: dadt_shared_kernel<1><<<n_items, kDadtThreads, 0, s>>>(nodes_mm, n_nodes, dp, n_dip, transform_dev, scale, out, g.n_tiles, chunk, n_items, pp); break;
        case 2: dadt_shared_kernel<2><<<n_items, kDadtThreads, 0, s>>>(nodes_mm, n_nodes, dp, n_dip, transform_dev, scale, out, g.n_tiles, chunk, n_items, pp); break;
        default: dadt_shared_kernel<3><<<n_items, kDadtThreads, 0, s>>>(nodes_mm, n_nodes, dp, n_dip, transform_dev, scale, out, g.n_tiles, chunk, n_items, pp); break;
    }
    count_launch();
    if (chunks > 1) {
        const long count = static_cast<long>(n_sets) * n_nodes * 3;
        shared_sum_kernel<<<grid_for(count), kBlock, 0, s>>>(count, chunks, pp, scale, out);
        count_launch();
    }
}

void dadt_elements(const Mesh& m, const float* nodal, int k, float* elm, cudaStream_t s) {
    const long total = static_cast<long>(m.n_tets) * k;
    element_average_kernel<<<grid_for(total), kBlock, 0, s>>>(nodal, m.tets.get(), m.n_nodes, m.n_tets, k, elm); count_launch();
    CUNIBS_LAUNCH_CHECK("dadt element average");
}

void rhs_block_nodes(Mesh& m, const float* nodal, int k, int K, double* b_red, cudaStream_t s) {
    if (!m.rhs_w_ok) {
        m.rhs_w.resize(3 * static_cast<std::size_t>(m.k_nnz));
        rhs_weights_kernel<<<grid_for(m.k_nnz), kBlock, 0, s>>>(m.g32.get(), m.neg_vc32.get(), m.contrib_ptr.get(),
                                                                m.contrib_idx.get(), m.k_nnz, m.rhs_w.get());
        count_launch();
        CUNIBS_LAUNCH_CHECK("rhs weights");
        m.rhs_w_ok = true;
    }
    const unsigned g = (m.n_nodes - 1 + 63) / 64;
    auto go = [&](auto kc) {
        constexpr int KK = decltype(kc)::value;
        rhs_nodes_kernel<KK><<<g, 64 * KK, 0, s>>>(nodal, m.rhs_w.get(), m.k_ptr.get(), m.k_col.get(), m.n_nodes, k,
                                                   m.ground, b_red);
        count_launch();
    };
    switch (K) {
        case 1: go(std::integral_constant<int, 1>{}); break;
        case 2: go(std::integral_constant<int, 2>{}); break;
        case 4: go(std::integral_constant<int, 4>{}); break;
        case 8: go(std::integral_constant<int, 8>{}); break;
        case 16: go(std::integral_constant<int, 16>{}); break;
        default: fail(kEInval, "block width must be one of {1, 2, 4, 8, 16}");
    }
    CUNIBS_LAUNCH_CHECK("rhs from nodes");
}

void rhs_block(const Mesh& m, const float* elm, int k, int K, double* b_red, cudaStream_t s, const float* neg_vc) {
    const unsigned g = (m.n_nodes - 1 + 63) / 64;
    const float* w = neg_vc ? neg_vc : m.neg_vc32.get();
    auto go = [&](auto kc) {
        constexpr int KK = decltype(kc)::value;
        rhs_kernel<KK><<<g, 64 * KK, 0, s>>>(elm, m.g32.get(), w, m.n2c_ptr.get(), m.n2c_idx.get(),
                                             m.n_nodes, m.n_tets, k, m.ground, b_red); count_launch();
    };
    switch (K) {
        case 1: go(std::integral_constant<int, 1>{}); break;
        case 2: go(std::integral_constant<int, 2>{}); break;
        case 4: go(std::integral_constant<int, 4>{}); break;
        case 8: go(std::integral_constant<int, 8>{}); break;
        case 16: go(std::integral_constant<int, 16>{}); break;
        default: fail(kEInval, "block width must be one of {1, 2, 4, 8, 16}");
    }
    CUNIBS_LAUNCH_CHECK("rhs");
}

}  // namespace cunibs

// --- coils with moments along their own z axis ------------------------------------------------
//
// In the coil frame (r' = R^T (r - c)) such a coil's dipoles are m_j z_hat at s_j, shared by every
// placement, and m z_hat x d = m (-d_y, d_x, 0). Per pair: the difference (3), |d|^2 (3), one rsqrt,
// w*m = (inv*m)*(inv*inv) (3) and two accumulations (2): 11 FP32 operations against 17 for a
// general moment, with the same direct-difference accuracy; 9 where a tile of dipoles lies in one
// plane of the coil frame. The result is rotated back, A = R A'.

namespace cunibs {
namespace {

__global__ void prep_zdipoles_kernel(const double* __restrict__ pos, const double* __restrict__ mom, int n_dip,
                                     ZDipolePacked* __restrict__ out, int* __restrict__ flag) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    int general = 0;
    if (j < n_dip) {
        ZDipolePacked d;
        const float sx = static_cast<float>(pos[3 * j]), sy = static_cast<float>(pos[3 * j + 1]);
        const float sz = static_cast<float>(pos[3 * j + 2]), m = static_cast<float>(mom[3 * j + 2]);
        d.sx = make_float2(sx, sx);
        d.sy = make_float2(sy, sy);
        d.sz = make_float2(sz, sz);
        d.m = make_float2(m, m);
        out[j] = d;
        general = (mom[3 * j] != 0.0) || (mom[3 * j + 1] != 0.0);
    }
    const int any = __syncthreads_or(general);
    if (threadIdx.x == 0 && any) atomicOr(flag, 1);
}

// Work items and node order as dadt_kernel's.
__global__ void __launch_bounds__(kDadtThreads) dadt_zcoil_kernel(const double* __restrict__ nodes_mm, int n_nodes,
                                                                  const ZDipolePacked* __restrict__ dip, int n_dip,
                                                                  const double* __restrict__ T, float scale,
                                                                  float* __restrict__ out, int n_tiles, int n_items) {
    __shared__ ZDipolePacked tile[kDipTile];
    for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int p = item / n_tiles;
    const double* Tp = T + 16 * static_cast<long>(p);
    // Columns of the rotation are the coil axes in head coordinates: R[a][b] = Tp[4a + b].
    double R[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) R[a][b] = Tp[4 * a + b];
    const double o[3] = {Tp[3] * 1e-3, Tp[7] * 1e-3, Tp[11] * 1e-3};
    const int stride = n_tiles * blockDim.x;
    const int base = (item - p * n_tiles) * blockDim.x + threadIdx.x;
    int node[4];
    float px[4], py[4], pz[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        node[u] = base + u * stride;
        const int i = node[u] < n_nodes ? node[u] : n_nodes - 1;
        double d[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) d[a] = nodes_mm[3 * static_cast<long>(i) + a] * 1e-3 - o[a];
        px[u] = static_cast<float>(R[0][0] * d[0] + R[1][0] * d[1] + R[2][0] * d[2]);
        py[u] = static_cast<float>(R[0][1] * d[0] + R[1][1] * d[1] + R[2][1] * d[2]);
        pz[u] = static_cast<float>(R[0][2] * d[0] + R[1][2] * d[1] + R[2][2] * d[2]);
    }
    const float2 rx0 = make_float2(px[0], px[1]), ry0 = make_float2(py[0], py[1]), rz0 = make_float2(pz[0], pz[1]);
    const float2 rx1 = make_float2(px[2], px[3]), ry1 = make_float2(py[2], py[3]), rz1 = make_float2(pz[2], pz[3]);
    float2 ax0 = make_float2(0.f, 0.f), ay0 = ax0, ax1 = ax0, ay1 = ax0;
    for (int t0 = 0; t0 < n_dip; t0 += kDipTile) {
        const int nt = min(kDipTile, n_dip - t0);
        __syncthreads();
        bool same_z = true, same_m = true;
        const float z_first = dip[t0].sz.x, m_first = dip[t0].m.x;
        for (int j = threadIdx.x; j < nt; j += blockDim.x) {
            tile[j] = dip[t0 + j];
            same_z = same_z && tile[j].sz.x == z_first;
            same_m = same_m && tile[j].m.x == m_first;
        }
        const int flat = __syncthreads_and(same_z);
        // A flat tile whose dipoles all carry one moment (a figure-8 wing, a uniformly wound disc):
        // sum inv^3 (dy, dx) over the tile and scale by the moment once, 8 FP32 operations per pair.
        if (flat && __syncthreads_and(same_m)) {
            const float2 sz = tile[0].sz, mt = tile[0].m;
            const float2 dz0 = __fadd2_rn(rz0, f2neg(sz)), dz1 = __fadd2_rn(rz1, f2neg(sz));
            const float2 zz0 = __fmul2_rn(dz0, dz0), zz1 = __fmul2_rn(dz1, dz1);
            float2 tx0 = make_float2(0.f, 0.f), ty0 = tx0, tx1 = tx0, ty1 = tx0;
#pragma unroll 4
            for (int j = 0; j < nt; ++j) {
                const ZDipolePacked d = tile[j];
                {
                    const float2 dx = __fadd2_rn(rx0, f2neg(d.sx));
                    const float2 dy = __fadd2_rn(ry0, f2neg(d.sy));
                    const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, zz0));
                    const float2 inv = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
                    const float2 w3 = __fmul2_rn(inv, __fmul2_rn(inv, inv));
                    tx0 = __ffma2_rn(w3, dy, tx0);
                    ty0 = __ffma2_rn(w3, dx, ty0);
                }
                {
                    const float2 dx = __fadd2_rn(rx1, f2neg(d.sx));
                    const float2 dy = __fadd2_rn(ry1, f2neg(d.sy));
                    const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, zz1));
                    const float2 inv = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
                    const float2 w3 = __fmul2_rn(inv, __fmul2_rn(inv, inv));
                    tx1 = __ffma2_rn(w3, dy, tx1);
                    ty1 = __ffma2_rn(w3, dx, ty1);
                }
            }
            ax0 = __ffma2_rn(mt, tx0, ax0);
            ay0 = __ffma2_rn(mt, ty0, ay0);
            ax1 = __ffma2_rn(mt, tx1, ax1);
            ay1 = __ffma2_rn(mt, ty1, ay1);
            continue;
        }
        // A tile of dipoles in one plane of the coil frame (every dipole of a flat winding) shares
        // d_z, so d_z and d_z^2 are formed once per node: 9 FP32 operations per pair instead of 11.
        if (flat) {
            const float2 sz = tile[0].sz;
            const float2 dz0 = __fadd2_rn(rz0, f2neg(sz)), dz1 = __fadd2_rn(rz1, f2neg(sz));
            const float2 zz0 = __fmul2_rn(dz0, dz0), zz1 = __fmul2_rn(dz1, dz1);
#pragma unroll 4
            for (int j = 0; j < nt; ++j) {
                const ZDipolePacked d = tile[j];
                {
                    const float2 dx = __fadd2_rn(rx0, f2neg(d.sx));
                    const float2 dy = __fadd2_rn(ry0, f2neg(d.sy));
                    const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, zz0));
                    const float2 inv = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
                    const float2 wm = __fmul2_rn(__fmul2_rn(inv, d.m), __fmul2_rn(inv, inv));
                    ax0 = __ffma2_rn(wm, dy, ax0);
                    ay0 = __ffma2_rn(wm, dx, ay0);
                }
                {
                    const float2 dx = __fadd2_rn(rx1, f2neg(d.sx));
                    const float2 dy = __fadd2_rn(ry1, f2neg(d.sy));
                    const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, zz1));
                    const float2 inv = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
                    const float2 wm = __fmul2_rn(__fmul2_rn(inv, d.m), __fmul2_rn(inv, inv));
                    ax1 = __ffma2_rn(wm, dy, ax1);
                    ay1 = __ffma2_rn(wm, dx, ay1);
                }
            }
            continue;
        }
#pragma unroll 4
        for (int j = 0; j < nt; ++j) {
            const ZDipolePacked d = tile[j];
            {
                const float2 dx = __fadd2_rn(rx0, f2neg(d.sx));
                const float2 dy = __fadd2_rn(ry0, f2neg(d.sy));
                const float2 dz = __fadd2_rn(rz0, f2neg(d.sz));
                float2 d2 = __fmul2_rn(dx, dx);
                d2 = __ffma2_rn(dy, dy, d2);
                d2 = __ffma2_rn(dz, dz, d2);
                const float2 inv = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
                const float2 wm = __fmul2_rn(__fmul2_rn(inv, d.m), __fmul2_rn(inv, inv));
                ax0 = __ffma2_rn(wm, dy, ax0);
                ay0 = __ffma2_rn(wm, dx, ay0);
            }
            {
                const float2 dx = __fadd2_rn(rx1, f2neg(d.sx));
                const float2 dy = __fadd2_rn(ry1, f2neg(d.sy));
                const float2 dz = __fadd2_rn(rz1, f2neg(d.sz));
                float2 d2 = __fmul2_rn(dx, dx);
                d2 = __ffma2_rn(dy, dy, d2);
                d2 = __ffma2_rn(dz, dz, d2);
                const float2 inv = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
                const float2 wm = __fmul2_rn(__fmul2_rn(inv, d.m), __fmul2_rn(inv, inv));
                ax1 = __ffma2_rn(wm, dy, ax1);
                ay1 = __ffma2_rn(wm, dx, ay1);
            }
        }
    }
    // A' = (-sum wm dy, sum wm dx, 0); A = R A'.
    const float axs[4] = {ax0.x, ax0.y, ax1.x, ax1.y};
    const float ays[4] = {ay0.x, ay0.y, ay1.x, ay1.y};
    float* o_p = out + static_cast<long>(p) * n_nodes * 3;
    const float R00 = static_cast<float>(R[0][0]), R01 = static_cast<float>(R[0][1]);
    const float R10 = static_cast<float>(R[1][0]), R11 = static_cast<float>(R[1][1]);
    const float R20 = static_cast<float>(R[2][0]), R21 = static_cast<float>(R[2][1]);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        if (node[u] < n_nodes) {
            const float a0 = -scale * axs[u];
            const float a1 = scale * ays[u];
            o_p[3 * static_cast<long>(node[u])] = R00 * a0 + R01 * a1;
            o_p[3 * static_cast<long>(node[u]) + 1] = R10 * a0 + R11 * a1;
            o_p[3 * static_cast<long>(node[u]) + 2] = R20 * a0 + R21 * a1;
        }
    }
    }
}

}  // namespace

std::size_t packed_zdipole_bytes() { return sizeof(ZDipolePacked); }

void prep_zdipoles(const double* pos, const double* mom, int n_dip, void* zpacked, int* general_flag_dev,
                   cudaStream_t s) {
    CUNIBS_CHECK(cudaMemsetAsync(general_flag_dev, 0, sizeof(int), s));
    prep_zdipoles_kernel<<<grid_for(n_dip), kBlock, 0, s>>>(pos, mom, n_dip, static_cast<ZDipolePacked*>(zpacked),
                                                            general_flag_dev);
    count_launch();
    CUNIBS_LAUNCH_CHECK("prep z-dipoles");
}

void dadt_zcoil_raw(const double* nodes_mm, int n_nodes, const void* zpacked, int n_dip, const double* transforms_dev,
                    int k, float scale, float* out, cudaStream_t s, int max_blocks) {
    const DadtGrid g = dadt_grid(n_nodes, k, max_blocks);
    dadt_zcoil_kernel<<<g.blocks, kDadtThreads, 0, s>>>(nodes_mm, n_nodes, static_cast<const ZDipolePacked*>(zpacked),
                                                       n_dip, transforms_dev, scale, out, g.n_tiles, g.n_items);
    count_launch();
    CUNIBS_LAUNCH_CHECK("dadt z-coil");
}

void dadt_nodes_zcoil(const Mesh& m, const void* zpacked, int n_dip, const double* transforms_dev, int k, double didt,
                      float* out, cudaStream_t s, int max_blocks) {
    dadt_zcoil_raw(m.nodes.get(), m.n_nodes, zpacked, n_dip, transforms_dev, k, static_cast<float>(didt * 1e-7), out, s,
                   max_blocks);
}

void dadt_general_raw(const double* nodes_mm, int n_nodes, const float* dip_packed, int n_dip,
                      const double* transforms_dev, int k, float scale, float* out, cudaStream_t s) {
    const DadtGrid g = dadt_grid(n_nodes, k, 0);
    dadt_kernel<<<g.blocks, kDadtThreads, 0, s>>>(nodes_mm, n_nodes, reinterpret_cast<const DipolePacked*>(dip_packed),
                                                 n_dip, transforms_dev, scale, out, g.n_tiles, g.n_items);
    count_launch();
    CUNIBS_LAUNCH_CHECK("dadt");
}

}  // namespace cunibs
