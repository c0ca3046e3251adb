// Per-subject mesh setup: Morton layout, P1 operator, node->corner map, stiffness pattern and
// sigma-weighted assembly, grounding, skin normals, gray-matter slice.
//
// Compiled with -fmad=false: every product and sum here is rounded on its own, so the integer
// results that depend on floating-point comparisons (Morton keys; later the aggregation) are
// reproducible by a CPU restatement bit for bit.
//
// Reference behaviour restated: fem/solve.py:302-348 (Morton order), gradient.cu:29-66 (P1
// gradients), fem/assembly.py:15-42,142-162 (conductivity, node2corner), pattern.cu:145-299 and
// stiffness.cu:32-65 (CSR pattern and values), fem/solve.py:287-298,361-365 (grounding),
// skin.cu:46-150 (smoothed skin normals), metrics.py:246-259 (region slice).
#include <cub/cub.cuh>

#include <cmath>

#include "internal.hpp"

namespace cunibs {
namespace {

// Temporary storage for one CUB call, grown on demand.
struct CubTemp {
    DevArray<unsigned char> buf;
    void* get(std::size_t bytes) {
        buf.reserve(bytes ? bytes : 1);
        return buf.get();
    }
};

template <typename K, typename V>
void sort_pairs(const K* kin, K* kout, const V* vin, V* vout, std::size_t n, int end_bit, cudaStream_t s) {
    std::size_t bytes = 0;
    CUNIBS_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, n, 0, end_bit, s));
    CubTemp t;
    CUNIBS_CHECK(cub::DeviceRadixSort::SortPairs(t.get(bytes), bytes, kin, kout, vin, vout, n, 0, end_bit, s));
}

template <typename T>
void exclusive_scan(const T* in, T* out, std::size_t n, cudaStream_t s) {
    std::size_t bytes = 0;
    CUNIBS_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, s));
    CubTemp t;
    CUNIBS_CHECK(cub::DeviceScan::ExclusiveSum(t.get(bytes), bytes, in, out, n, s));
}

int bits_for(std::int64_t max_value) {
    int b = 1;
    while (b < 63 && (std::int64_t{1} << b) <= max_value) ++b;
    return b;
}

__global__ void iota_kernel(int* out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = i;
}

// Bounding box per axis: one block per axis. min/max are order independent.
__global__ void bbox_kernel(const double* __restrict__ pts, int n, double* __restrict__ lo_span) {
    __shared__ double smin[1024], smax[1024];
    const int a = blockIdx.x;
    double mn = INFINITY, mx = -INFINITY;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = pts[3 * static_cast<std::int64_t>(i) + a];
        mn = fmin(mn, v);
        mx = fmax(mx, v);
    }
    smin[threadIdx.x] = mn;
    smax[threadIdx.x] = mx;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + off]);
            smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + off]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        lo_span[a] = smin[0];
        lo_span[3 + a] = fmax(smax[0] - smin[0], 1e-12);
    }
}

__device__ __forceinline__ std::uint64_t spread3(std::uint64_t v) {
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__global__ void morton_key_kernel(const double* __restrict__ pts, int n, const double* __restrict__ lo_span,
                                  std::uint64_t* __restrict__ key) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    std::uint64_t k = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double t = (pts[3 * static_cast<std::int64_t>(i) + a] - lo_span[a]) / lo_span[3 + a] * 2097151.0;
        k |= spread3(static_cast<std::uint64_t>(t)) << a;
    }
    key[i] = k;
}

__global__ void invert_perm_kernel(const int* __restrict__ perm, int* __restrict__ inv, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) inv[perm[i]] = i;
}

__global__ void tet_lowest_kernel(const int* __restrict__ inverse, const int* __restrict__ tets, int m,
                                  int* __restrict__ lowest) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
    const int4 t = reinterpret_cast<const int4*>(tets)[e];
    lowest[e] = min(min(inverse[t.x], inverse[t.y]), min(inverse[t.z], inverse[t.w]));
}

__global__ void gather_nodes_kernel(const double* __restrict__ src, const int* __restrict__ perm, int n,
                                    double* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const std::int64_t p = perm[i];
#pragma unroll
    for (int a = 0; a < 3; ++a) dst[3 * static_cast<std::int64_t>(i) + a] = src[3 * p + a];
}

__global__ void gather_tets_kernel(const int* __restrict__ tets_in, const int* __restrict__ tags_in,
                                   const int* __restrict__ perm, const int* __restrict__ inverse, int m,
                                   int* __restrict__ tets_out, int* __restrict__ tags_out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
    const int src = perm[e];
    const int4 t = reinterpret_cast<const int4*>(tets_in)[src];
    reinterpret_cast<int4*>(tets_out)[e] = make_int4(inverse[t.x], inverse[t.y], inverse[t.z], inverse[t.w]);
    tags_out[e] = tags_in[src];
}

__global__ void renumber_kernel(const int* __restrict__ in, const int* __restrict__ inverse, std::int64_t n,
                                int* __restrict__ out) {
    const std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = inverse[in[i]];
}

// Count of indices outside [0, n) (validation before any gather).
__global__ void count_out_of_range_kernel(const int* __restrict__ v, std::int64_t len, int n, int* __restrict__ bad) {
    const std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int pred = (i < len) && (static_cast<unsigned>(v[i]) >= static_cast<unsigned>(n));
    const int c = __syncthreads_count(pred);
    if (threadIdx.x == 0 && c) atomicAdd(bad, c);
}

// P1 gradients (G = (T^-1 A)^T by adjugate over determinant) and volumes, one thread per tet.
__global__ void p1_gradients_kernel(const double* __restrict__ nodes, const int* __restrict__ tets, int m,
                                    double* __restrict__ g, double* __restrict__ vols, int* __restrict__ bad) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    int invalid = 0;
    if (e < m) {
        const int4 tn = reinterpret_cast<const int4*>(tets)[e];
        const int ni[3] = {tn.y, tn.z, tn.w};
        double t[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                t[i][c] = nodes[3 * static_cast<std::int64_t>(ni[i]) + c] - nodes[3 * static_cast<std::int64_t>(tn.x) + c];
        double adj[3][3];
        adj[0][0] = t[1][1] * t[2][2] - t[1][2] * t[2][1];
        adj[0][1] = t[1][2] * t[2][0] - t[1][0] * t[2][2];
        adj[0][2] = t[1][0] * t[2][1] - t[1][1] * t[2][0];
        adj[1][0] = t[2][1] * t[0][2] - t[2][2] * t[0][1];
        adj[1][1] = t[2][2] * t[0][0] - t[2][0] * t[0][2];
        adj[1][2] = t[2][0] * t[0][1] - t[2][1] * t[0][0];
        adj[2][0] = t[0][1] * t[1][2] - t[0][2] * t[1][1];
        adj[2][1] = t[0][2] * t[1][0] - t[0][0] * t[1][2];
        adj[2][2] = t[0][0] * t[1][1] - t[0][1] * t[1][0];
        const double det = t[0][0] * adj[0][0] + t[0][1] * adj[0][1] + t[0][2] * adj[0][2];
        const double inv = 1e3 / det;
        double* ge = g + 12 * static_cast<std::int64_t>(e);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double g1 = adj[0][c] * inv;
            const double g2 = adj[1][c] * inv;
            const double g3 = adj[2][c] * inv;
            ge[0 + c] = -(g1 + g2 + g3);
            ge[3 + c] = g1;
            ge[6 + c] = g2;
            ge[9 + c] = g3;
        }
        const double v = fabs(det) * (1e-9 / 6.0);
        vols[e] = v;
        invalid = !(v > 0.0) || !isfinite(v);
    }
    const int c = __syncthreads_count(invalid);
    if (threadIdx.x == 0 && c) atomicAdd(bad, c);
}

// Tissue conductivity table (fem/assembly.py:15-26); NaN marks an unknown tag.
// A conductivity table (index = tissue tag) passed by value: contexts driven from several host
// threads each launch with their own.
struct SigmaTable {
    double s[11];
};

SigmaTable sigma_table(const double* sigma_by_tag) {
    SigmaTable t;
    for (int i = 0; i < 11; ++i) t.s[i] = sigma_by_tag[i];
    return t;
}

__global__ void conductivity_kernel(const int* __restrict__ tags, int m, SigmaTable table, double* __restrict__ cond,
                                    int* __restrict__ bad) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    int invalid = 0;
    if (e < m) {
        const int t = tags[e];
        const double s = (t >= 0 && t <= 10) ? table.s[t] : NAN;
        cond[e] = s;
        invalid = isnan(s);
    }
    const int c = __syncthreads_count(invalid);
    if (threadIdx.x == 0 && c) atomicAdd(bad, c);
}

// -(vol * sigma) in FP32, the right-hand side's per-element weight (fem/solve.py:714).
__global__ void neg_vc_kernel(const float* __restrict__ vols32, const double* __restrict__ cond, int m,
                              float* __restrict__ neg_vc32) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < m) neg_vc32[e] = -(vols32[e] * static_cast<float>(cond[e]));
}

__global__ void resident_kernel(const double* __restrict__ g, const double* __restrict__ vols,
                                const double* __restrict__ cond, const double* __restrict__ nodes,
                                const int* __restrict__ tets, int m, float* __restrict__ g32,
                                float* __restrict__ vols32, float* __restrict__ neg_vc32,
                                double* __restrict__ bary) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
#pragma unroll
    for (int q = 0; q < 12; ++q) g32[12 * static_cast<std::int64_t>(e) + q] = static_cast<float>(g[12 * static_cast<std::int64_t>(e) + q]);
    const float v32 = static_cast<float>(vols[e]);
    vols32[e] = v32;
    // The reference forms -(vols.f32 * cond.f32) in FP32 (fem/solve.py:714).
    neg_vc32[e] = -(v32 * static_cast<float>(cond[e]));
    const int4 tn = reinterpret_cast<const int4*>(tets)[e];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        bary[3 * static_cast<std::int64_t>(e) + a] =
            (nodes[3 * static_cast<std::int64_t>(tn.x) + a] + nodes[3 * static_cast<std::int64_t>(tn.y) + a] +
             nodes[3 * static_cast<std::int64_t>(tn.z) + a] + nodes[3 * static_cast<std::int64_t>(tn.w) + a]) /
            4.0;
    }
}

// ptr[i] = first position in the sorted key list whose key is >= i (keys sorted ascending).
__global__ void segment_starts_kernel(const int* __restrict__ sorted_keys, std::int64_t len, int n_segments,
                                      int* __restrict__ ptr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n_segments) return;
    std::int64_t lo = 0, hi = len;
    while (lo < hi) {
        const std::int64_t mid = (lo + hi) >> 1;
        if (sorted_keys[mid] < i) lo = mid + 1;
        else hi = mid;
    }
    ptr[i] = static_cast<int>(lo);
}

// Element-pair keys for the stiffness pattern: (row node << 32) | col node, with the value
// e*16 + i*4 + j naming the element entry. A stable sort by key groups each CSR entry's
// contributions in ascending element order.
__global__ void pair_keys_kernel(const int* __restrict__ tets, int m, std::uint64_t* __restrict__ keys,
                                 int* __restrict__ vals) {
    const std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= 16 * static_cast<std::int64_t>(m)) return;
    const int e = static_cast<int>(q >> 4);
    const int i = static_cast<int>((q >> 2) & 3);
    const int j = static_cast<int>(q & 3);
    const std::uint64_t r = static_cast<std::uint32_t>(tets[4 * static_cast<std::int64_t>(e) + i]);
    const std::uint64_t c = static_cast<std::uint32_t>(tets[4 * static_cast<std::int64_t>(e) + j]);
    keys[q] = (r << 32) | c;
    vals[q] = static_cast<int>(q);
}

__global__ void head_flags_kernel(const std::uint64_t* __restrict__ keys, std::int64_t len, int* __restrict__ flags) {
    const std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q < len) flags[q] = (q == 0 || keys[q] != keys[q - 1]) ? 1 : 0;
}

// For every run head: its entry index, column, and where its contributions start.
__global__ void pattern_fill_kernel(const std::uint64_t* __restrict__ keys, const int* __restrict__ flags,
                                    const int* __restrict__ pos, std::int64_t len, int* __restrict__ col,
                                    int* __restrict__ row_of, int* __restrict__ contrib_ptr) {
    const std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= len || !flags[q]) return;
    const int p = pos[q];
    col[p] = static_cast<int>(keys[q] & 0xffffffffu);
    row_of[p] = static_cast<int>(keys[q] >> 32);
    contrib_ptr[p] = static_cast<int>(q);
}

// Element matrices, a half-warp per element: lane l owns entry (l/4, l%4) and writes
// vol*sigma*(g_i . g_j), products rounded one at a time, summed left to right.
// Stiffness values, deterministically: each CSR entry sums its element contributions
// vol_e sigma_e (g_ei . g_ej) in the order of contrib_idx (ascending element), with every product
// and sum rounded on its own; nothing is staged per contribution.
__global__ void assemble_entries_kernel(const double* __restrict__ g, const double* __restrict__ vols,
                                        const double* __restrict__ cond, const int* __restrict__ contrib_ptr,
                                        const int* __restrict__ contrib_idx, long nnz, double* __restrict__ out) {
    const long p = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= nnz) return;
    double acc = 0.0;
    const int end = contrib_ptr[p + 1];
    for (int q = contrib_ptr[p]; q < end; ++q) {
        const int idx = contrib_idx[q];
        const std::int64_t e = idx >> 4;
        const double* gi = g + 12 * e + 3 * ((idx >> 2) & 3);
        const double* gj = g + 12 * e + 3 * (idx & 3);
        const double dot = gi[0] * gj[0] + gi[1] * gj[1] + gi[2] * gj[2];
        const double sv = vols[e] * cond[e];
        acc = acc + sv * dot;
    }
    out[p] = acc;
}

// Grounded values on a known grounded pattern: row r of the reduced operator is row
// i = r + (r >= ground) of the full one without the ground column, entries in order.
__global__ void reduced_values_kernel(const int* __restrict__ ptr, const int* __restrict__ col,
                                     const double* __restrict__ val, int n, int ground, const int* __restrict__ rptr,
                                     double* __restrict__ rval) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n - 1) return;
    const int i = r + (r >= ground ? 1 : 0);
    int q = rptr[r];
    for (int p = ptr[i]; p < ptr[i + 1]; ++p) {
        if (col[p] == ground) continue;
        rval[q] = val[p];
        ++q;
    }
}

// Lowest-z node, lowest index on ties: a min over the total order (z, index).
__global__ void ground_kernel(const double* __restrict__ nodes, int n, int* __restrict__ out) {
    __shared__ double sz[1024];
    __shared__ int si[1024];
    double bz = INFINITY;
    int bi = 0x7fffffff;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double z = nodes[3 * static_cast<std::int64_t>(i) + 2];
        if (z < bz || (z == bz && i < bi)) {
            bz = z;
            bi = i;
        }
    }
    sz[threadIdx.x] = bz;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            const double z = sz[threadIdx.x + off];
            const int i = si[threadIdx.x + off];
            if (z < sz[threadIdx.x] || (z == sz[threadIdx.x] && i < si[threadIdx.x])) {
                sz[threadIdx.x] = z;
                si[threadIdx.x] = i;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = si[0];
}

__global__ void reduced_count_kernel(const int* __restrict__ ptr, const int* __restrict__ col, int n, int ground,
                                     int* __restrict__ cnt) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n - 1) return;
    const int i = r + (r >= ground ? 1 : 0);
    int c = 0;
    for (int p = ptr[i]; p < ptr[i + 1]; ++p) c += (col[p] != ground);
    cnt[r] = c;
}

__global__ void reduced_fill_kernel(const int* __restrict__ ptr, const int* __restrict__ col,
                                    const double* __restrict__ val, int n, int ground, const int* __restrict__ rptr,
                                    int* __restrict__ rcol, double* __restrict__ rval) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n - 1) return;
    const int i = r + (r >= ground ? 1 : 0);
    int q = rptr[r];
    for (int p = ptr[i]; p < ptr[i + 1]; ++p) {
        const int c = col[p];
        if (c == ground) continue;
        rcol[q] = c - (c > ground ? 1 : 0);
        rval[q] = val[p];
        ++q;
    }
}

// --- skin normals -----------------------------------------------------------------------

__global__ void face_normals_kernel(const double* __restrict__ nodes, const int* __restrict__ tris, int s,
                                    double* __restrict__ face) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= s) return;
    const double* a = nodes + 3 * static_cast<std::int64_t>(tris[3 * t]);
    const double* b = nodes + 3 * static_cast<std::int64_t>(tris[3 * t + 1]);
    const double* c = nodes + 3 * static_cast<std::int64_t>(tris[3 * t + 2]);
    double u[3], v[3];
    for (int i = 0; i < 3; ++i) {
        u[i] = b[i] - a[i];
        v[i] = c[i] - a[i];
    }
    face[3 * t] = u[1] * v[2] - u[2] * v[1];
    face[3 * t + 1] = u[2] * v[0] - u[0] * v[2];
    face[3 * t + 2] = u[0] * v[1] - u[1] * v[0];
}

__global__ void spread_kernel(const double* __restrict__ face, const int* __restrict__ ptr,
                              const int* __restrict__ idx, int n, double* __restrict__ node) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int p = ptr[i]; p < ptr[i + 1]; ++p) {
        const int t = idx[p] / 3;
        for (int a = 0; a < 3; ++a) acc[a] = acc[a] + face[3 * t + a];
    }
    for (int a = 0; a < 3; ++a) node[3 * static_cast<std::int64_t>(i) + a] = acc[a];
}

__device__ __forceinline__ void normalise3(double* v) {
    const double n = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (n > 0.0)
        for (int i = 0; i < 3; ++i) v[i] = v[i] / n;
}

__global__ void gather_faces_kernel(const double* __restrict__ node, const int* __restrict__ tris, int s,
                                    double* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= s) return;
    double acc[3];
    for (int a = 0; a < 3; ++a)
        acc[a] = node[3 * static_cast<std::int64_t>(tris[3 * t]) + a] + node[3 * static_cast<std::int64_t>(tris[3 * t + 1]) + a] +
                 node[3 * static_cast<std::int64_t>(tris[3 * t + 2]) + a];
    normalise3(acc);
    for (int a = 0; a < 3; ++a) out[3 * t + a] = acc[a];
}

__global__ void normalise_rows_kernel(double* __restrict__ v, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) normalise3(v + 3 * static_cast<std::int64_t>(i));
}

__global__ void gm_flags_kernel(const int* __restrict__ tags, int m, int tag, int* __restrict__ flags) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < m) flags[e] = (tags[e] == tag) ? 1 : 0;
}

__global__ void compact_kernel(const int* __restrict__ flags, const int* __restrict__ pos, int m, int* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < m && flags[e]) out[pos[e]] = e;
}

int read_int(const int* dev, cudaStream_t s) {
    int h = 0;
    CUNIBS_CHECK(cudaMemcpyAsync(&h, dev, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUNIBS_CHECK(cudaStreamSynchronize(s));
    return h;
}

// node -> corner CSR over `per`-node elements: stable sort of corner ids by node.
void build_node2corner(const int* elems, int n_elems, int per, int n_nodes, DevArray<int>& ptr, DevArray<int>& idx,
                       cudaStream_t s) {
    const std::int64_t nc = static_cast<std::int64_t>(n_elems) * per;
    ptr.resize(n_nodes + 1);
    idx.resize(nc > 0 ? nc : 1);
    if (nc == 0) {
        CUNIBS_CHECK(cudaMemsetAsync(ptr.get(), 0, sizeof(int) * (n_nodes + 1), s));
        return;
    }
    DevArray<int> ids(nc), keys_sorted(nc);
    iota_kernel<<<grid_for(nc), kBlock, 0, s>>>(ids.get(), static_cast<int>(nc)); count_launch();
    sort_pairs(elems, keys_sorted.get(), ids.get(), idx.get(), nc, bits_for(n_nodes), s);
    segment_starts_kernel<<<grid_for(n_nodes + 1), kBlock, 0, s>>>(keys_sorted.get(), nc, n_nodes, ptr.get()); count_launch();
    CUNIBS_LAUNCH_CHECK("node2corner");
}

}  // namespace

void build_mesh(Mesh& m, const double* nodes_mm, int n_nodes, const int* tets, const int* tags, int n_tets,
                const int* skin, int n_skin, cudaStream_t s) {
    if (n_nodes < 2 || n_tets < 1) fail(kEInval, "mesh needs at least two nodes and one tetrahedron");
    m.n_nodes = n_nodes;
    m.n_tets = n_tets;
    m.n_skin = n_skin;
    const std::int64_t N = n_nodes, M = n_tets, S = n_skin;
    DevArray<double> nodes_in;
    DevArray<int> tets_in, tags_in, skin_in;
    nodes_in.upload(nodes_mm, 3 * N, s);
    tets_in.upload(tets, 4 * M, s);
    tags_in.upload(tags, M, s);
    if (S) skin_in.upload(skin, 3 * S, s);
    DevArray<int> bad(1);
    bad.zero(s);
    count_out_of_range_kernel<<<grid_for(4 * M), kBlock, 0, s>>>(tets_in.get(), 4 * M, n_nodes, bad.get()); count_launch();
    if (S) {
        count_out_of_range_kernel<<<grid_for(3 * S), kBlock, 0, s>>>(skin_in.get(), 3 * S, n_nodes, bad.get());
        count_launch();
    }
    if (read_int(bad.get(), s)) fail(kEInval, "tet_nodes or skin_tris reference a node outside the node table");

    // Morton order of the nodes, then tets by their lowest renumbered node.
    DevArray<double> box(6);
    bbox_kernel<<<3, 1024, 0, s>>>(nodes_in.get(), n_nodes, box.get()); count_launch();
    DevArray<std::uint64_t> key(N), key_sorted(N);
    DevArray<int> ids(N);
    morton_key_kernel<<<grid_for(N), kBlock, 0, s>>>(nodes_in.get(), n_nodes, box.get(), key.get()); count_launch();
    iota_kernel<<<grid_for(N), kBlock, 0, s>>>(ids.get(), n_nodes); count_launch();
    m.node_perm.resize(N);
    sort_pairs(key.get(), key_sorted.get(), ids.get(), m.node_perm.get(), N, 63, s);
    DevArray<int> inverse(N);
    invert_perm_kernel<<<grid_for(N), kBlock, 0, s>>>(m.node_perm.get(), inverse.get(), n_nodes); count_launch();
    DevArray<int> lowest(M), lowest_sorted(M), tid(M);
    tet_lowest_kernel<<<grid_for(M), kBlock, 0, s>>>(inverse.get(), tets_in.get(), n_tets, lowest.get()); count_launch();
    iota_kernel<<<grid_for(M), kBlock, 0, s>>>(tid.get(), n_tets); count_launch();
    m.tet_perm.resize(M);
    sort_pairs(lowest.get(), lowest_sorted.get(), tid.get(), m.tet_perm.get(), M, bits_for(n_nodes), s);
    m.nodes.resize(3 * N);
    gather_nodes_kernel<<<grid_for(N), kBlock, 0, s>>>(nodes_in.get(), m.node_perm.get(), n_nodes, m.nodes.get()); count_launch();
    m.tets.resize(4 * M);
    m.tags.resize(M);
    gather_tets_kernel<<<grid_for(M), kBlock, 0, s>>>(tets_in.get(), tags_in.get(), m.tet_perm.get(), inverse.get(),
                                                      n_tets, m.tets.get(), m.tags.get()); count_launch();
    if (S) {
        m.skin.resize(3 * S);
        renumber_kernel<<<grid_for(3 * S), kBlock, 0, s>>>(skin_in.get(), inverse.get(), 3 * S, m.skin.get()); count_launch();
    }
    CUNIBS_LAUNCH_CHECK("morton layout");

    // P1 operator and conductivity.
    m.g.resize(12 * M);
    m.vols.resize(M);
    bad.zero(s);
    p1_gradients_kernel<<<grid_for(M), kBlock, 0, s>>>(m.nodes.get(), m.tets.get(), n_tets, m.g.get(), m.vols.get(),
                                                       bad.get()); count_launch();
    const int n_bad_vol = read_int(bad.get(), s);
    if (n_bad_vol) {
        fail(kEInval, std::to_string(n_bad_vol) + (n_bad_vol == 1 ? " tetrahedron has" : " tetrahedra have") +
                          " zero or non-finite volume");
    }
    const double sigma[11] = {NAN, 0.126, 0.275, 1.654, 0.010, 0.465, 0.5, 0.008, 0.025, 0.6, 0.16};
    m.cond.resize(M);
    bad.zero(s);
    conductivity_kernel<<<grid_for(M), kBlock, 0, s>>>(m.tags.get(), n_tets, sigma_table(sigma), m.cond.get(), bad.get());
    count_launch();
    if (read_int(bad.get(), s)) fail(kEInval, "tetrahedra with unknown tissue tags");

    m.g32.resize(12 * M);
    m.vols32.resize(M);
    m.neg_vc32.resize(M);
    m.bary.resize(3 * M);
    resident_kernel<<<grid_for(M), kBlock, 0, s>>>(m.g.get(), m.vols.get(), m.cond.get(), m.nodes.get(), m.tets.get(),
                                                   n_tets, m.g32.get(), m.vols32.get(), m.neg_vc32.get(), m.bary.get()); count_launch();
    build_node2corner(m.tets.get(), n_tets, 4, n_nodes, m.n2c_ptr, m.n2c_idx, s);

    // Stiffness pattern and contribution map from one stable sort of the 16 entries per element.
    {
        const std::int64_t Q = 16 * M;
        DevArray<std::uint64_t> pk(Q), pk_sorted(Q);
        DevArray<int> pv(Q);
        pair_keys_kernel<<<grid_for(Q), kBlock, 0, s>>>(m.tets.get(), n_tets, pk.get(), pv.get()); count_launch();
        m.contrib_idx.resize(Q);
        sort_pairs(pk.get(), pk_sorted.get(), pv.get(), m.contrib_idx.get(), Q, 32 + bits_for(n_nodes), s);
        DevArray<int> flags(Q + 1), pos(Q + 1);
        head_flags_kernel<<<grid_for(Q), kBlock, 0, s>>>(pk_sorted.get(), Q, flags.get()); count_launch();
        CUNIBS_CHECK(cudaMemsetAsync(flags.get() + Q, 0, sizeof(int), s));
        exclusive_scan(flags.get(), pos.get(), Q + 1, s);
        const int nnz = read_int(pos.get() + Q, s);
        m.k_nnz = nnz;
        m.k_col.resize(nnz);
        m.contrib_ptr.resize(nnz + 1);
        DevArray<int> row_of(nnz);
        pattern_fill_kernel<<<grid_for(Q), kBlock, 0, s>>>(pk_sorted.get(), flags.get(), pos.get(), Q, m.k_col.get(),
                                                           row_of.get(), m.contrib_ptr.get()); count_launch();
        const int q_end = static_cast<int>(Q);
        CUNIBS_CHECK(cudaMemcpyAsync(m.contrib_ptr.get() + nnz, &q_end, sizeof(int), cudaMemcpyHostToDevice, s));
        m.k_ptr.resize(N + 1);
        segment_starts_kernel<<<grid_for(N + 1), kBlock, 0, s>>>(row_of.get(), nnz, n_nodes, m.k_ptr.get()); count_launch();
        CUNIBS_LAUNCH_CHECK("stiffness pattern");
        CUNIBS_CHECK(cudaStreamSynchronize(s));  // q_end is a host temporary
    }
    assemble_stiffness(m, nullptr, s);

    // Ground node.
    {
        DevArray<int> gdev(1);
        ground_kernel<<<1, 1024, 0, s>>>(m.nodes.get(), n_nodes, gdev.get()); count_launch();
        m.ground = read_int(gdev.get(), s);
    }

    // Smoothed skin normals: face normals spread to nodes and gathered back twice.
    m.skin_normals.resize(S ? 3 * S : 1);
    if (S) {
        DevArray<int> sptr, sidx;
        build_node2corner(m.skin.get(), n_skin, 3, n_nodes, sptr, sidx, s);
        DevArray<double> face(3 * S), node(3 * N);
        face_normals_kernel<<<grid_for(S), kBlock, 0, s>>>(m.nodes.get(), m.skin.get(), n_skin, face.get()); count_launch();
        spread_kernel<<<grid_for(N), kBlock, 0, s>>>(face.get(), sptr.get(), sidx.get(), n_nodes, node.get()); count_launch();
        gather_faces_kernel<<<grid_for(S), kBlock, 0, s>>>(node.get(), m.skin.get(), n_skin, face.get()); count_launch();
        spread_kernel<<<grid_for(N), kBlock, 0, s>>>(face.get(), sptr.get(), sidx.get(), n_nodes, node.get()); count_launch();
        normalise_rows_kernel<<<grid_for(N), kBlock, 0, s>>>(node.get(), n_nodes); count_launch();
        gather_faces_kernel<<<grid_for(S), kBlock, 0, s>>>(node.get(), m.skin.get(), n_skin, m.skin_normals.get()); count_launch();
        CUNIBS_LAUNCH_CHECK("skin normals");
        CUNIBS_CHECK(cudaStreamSynchronize(s));
    }

    // Gray-matter slice, in element order.
    {
        DevArray<int> flags(M + 1), pos(M + 1);
        gm_flags_kernel<<<grid_for(M), kBlock, 0, s>>>(m.tags.get(), n_tets, 2, flags.get()); count_launch();
        CUNIBS_CHECK(cudaMemsetAsync(flags.get() + M, 0, sizeof(int), s));
        exclusive_scan(flags.get(), pos.get(), M + 1, s);
        m.n_gm = read_int(pos.get() + M, s);
        m.gm_index.resize(m.n_gm ? m.n_gm : 1);
        compact_kernel<<<grid_for(M), kBlock, 0, s>>>(flags.get(), pos.get(), n_tets, m.gm_index.get()); count_launch();
        CUNIBS_LAUNCH_CHECK("gm slice");
    }
    CUNIBS_CHECK(cudaStreamSynchronize(s));
}

void set_element_conductivity(Mesh& m, const double* sigma_by_tag, cudaStream_t s, bool validate) {
    m.cond_bad.resize(1);
    if (validate) m.cond_bad.zero(s);
    conductivity_kernel<<<grid_for(m.n_tets), kBlock, 0, s>>>(m.tags.get(), m.n_tets, sigma_table(sigma_by_tag),
                                                              m.cond.get(), m.cond_bad.get());
    count_launch();
    if (validate && read_int(m.cond_bad.get(), s)) fail(kEInval, "conductivity table leaves a tag undefined");
    // The right-hand side weighs each element by the same conductivity.
    neg_vc_kernel<<<grid_for(m.n_tets), kBlock, 0, s>>>(m.vols32.get(), m.cond.get(), m.n_tets, m.neg_vc32.get());
    count_launch();
    m.rhs_w_ok = false;
}

void assemble_stiffness(Mesh& m, const double* sigma_by_tag, cudaStream_t s) {
    if (sigma_by_tag != nullptr) set_element_conductivity(m, sigma_by_tag, s);
    m.k_val.resize(m.k_nnz);
    assemble_entries_kernel<<<grid_for(m.k_nnz), kBlock, 0, s>>>(m.g.get(), m.vols.get(), m.cond.get(),
                                                                 m.contrib_ptr.get(), m.contrib_idx.get(), m.k_nnz,
                                                                 m.k_val.get()); count_launch();
    CUNIBS_LAUNCH_CHECK("stiffness values");
    CUNIBS_CHECK(cudaStreamSynchronize(s));
}

void reduce_grounded_values(const Mesh& m, const DevCsr<double>& pattern, double* out, cudaStream_t s) {
    if (pattern.n != m.n_nodes - 1) fail(kEInternal, "grounded pattern of another mesh");
    reduced_values_kernel<<<grid_for(m.n_nodes - 1), kBlock, 0, s>>>(m.k_ptr.get(), m.k_col.get(), m.k_val.get(),
                                                                     m.n_nodes, m.ground, pattern.ptr.get(), out);
    count_launch();
    CUNIBS_LAUNCH_CHECK("grounded values");
}

void assemble_reduced_values(const Mesh& m, const double* tables, int n_tables, const DevCsr<double>& pattern,
                             double* out, cudaStream_t s) {
    if (pattern.n != m.n_nodes - 1) fail(kEInternal, "grounded pattern of another mesh");
    const int M = m.n_tets;
    DevArray<double> cond(M), full(m.k_nnz);
    DevArray<int> bad(1);
    for (int t = 0; t < n_tables; ++t) {
        bad.zero(s);
        conductivity_kernel<<<grid_for(M), kBlock, 0, s>>>(m.tags.get(), M, sigma_table(tables + 11 * t), cond.get(),
                                                           bad.get());
        count_launch();
        if (read_int(bad.get(), s)) fail(kEInval, "conductivity table leaves a tag undefined");
        assemble_entries_kernel<<<grid_for(m.k_nnz), kBlock, 0, s>>>(m.g.get(), m.vols.get(), cond.get(),
                                                                     m.contrib_ptr.get(), m.contrib_idx.get(), m.k_nnz,
                                                                     full.get()); count_launch();
        reduced_values_kernel<<<grid_for(m.n_nodes - 1), kBlock, 0, s>>>(m.k_ptr.get(), m.k_col.get(), full.get(),
                                                                         m.n_nodes, m.ground, pattern.ptr.get(),
                                                                         out + static_cast<std::size_t>(t) * pattern.nnz);
        count_launch();
    }
    CUNIBS_LAUNCH_CHECK("reduced stiffness values");
    CUNIBS_CHECK(cudaStreamSynchronize(s));
}

void reduce_grounded(const Mesh& m, DevCsr<double>& out, cudaStream_t s) {
    const int n = m.n_nodes;
    out.n = out.ncol = n - 1;
    DevArray<int> cnt(n);
    CUNIBS_CHECK(cudaMemsetAsync(cnt.get() + (n - 1), 0, sizeof(int), s));
    reduced_count_kernel<<<grid_for(n - 1), kBlock, 0, s>>>(m.k_ptr.get(), m.k_col.get(), n, m.ground, cnt.get()); count_launch();
    out.ptr.resize(n);
    exclusive_scan(cnt.get(), out.ptr.get(), n, s);
    out.nnz = read_int(out.ptr.get() + (n - 1), s);
    out.col.resize(out.nnz);
    out.val.resize(out.nnz);
    reduced_fill_kernel<<<grid_for(n - 1), kBlock, 0, s>>>(m.k_ptr.get(), m.k_col.get(), m.k_val.get(), n, m.ground,
                                                           out.ptr.get(), out.col.get(), out.val.get()); count_launch();
    CUNIBS_LAUNCH_CHECK("reduce grounded");
}

}  // namespace cunibs
