// Field recovery: the smoothed E-field the reference reports by default.
//
// Reference behaviour restated: fem/recovery.py:1-552 and recovery.cu:1-774. Three modes:
//   spr_global  - a linear least-squares fit of the per-element E over each node's incident
//                 tetrahedra, evaluated at the node (Zienkiewicz-Zhu SPR); one FP32 weight per
//                 node-to-corner entry; boundary nodes and ill-posed fits take the volume average.
//   spr_tissue  - the same over (node, tissue) slots, so the jump at a conductivity interface
//                 survives; nodes touching two tissues count as boundary nodes of each.
//   harmonic    - the potential v fitted over a same-tissue node patch in the space of harmonic
//                 polynomials (16 cubic terms, 9 quadratic, else 4 linear), differentiated at the
//                 node, and the exact nodal dA/dt added: E = -grad v - dA/dt. The default.
// The recovered slot field is sampled back at each tetrahedron's barycentre as the mean of its
// four corner slots.
//
// Everything the operator holds is integer or FP32 produced from FP64 arithmetic with every
// multiply-add written out (this file is compiled with -fmad=false), so the operator and the
// applied field are reproducible bit for bit by a CPU restatement.
//
// B200 layout: the harmonic operator is one float4 per patch entry {w_x, w_y, w_z, node} so the
// apply streams one 16-byte load per entry, shared by the K column lanes of a slot (a broadcast);
// the potential is read from the solver's row-major (n, K) block, one 8-byte lane per column.
#include <cstdlib>

#include <cub/cub.cuh>

#include "internal.hpp"

namespace cunibs {
namespace {

constexpr int kMinPatchNodes = 16;    // grow to the 2-ring below this many nodes (recovery.py:246-250)
constexpr double kMaxLebesgue = 8.0;  // SPR: largest sum|w| of an accepted fit
constexpr double kMaxGradAmp = 50.0;  // harmonic: largest h * max_c sum_p |w_pc| of an accepted rung
constexpr int kTagBits = 4;           // tissue tags are 1..10

struct CubTemp {
    DevArray<unsigned char> buf;
    void* get(std::size_t bytes) {
        buf.reserve(bytes ? bytes : 1);
        return buf.get();
    }
};

int bits_for(std::int64_t max_value) {
    int b = 1;
    while (b < 63 && (std::int64_t{1} << b) <= max_value) ++b;
    return b;
}

template <typename T>
void exclusive_scan(const T* in, T* out, std::size_t n, cudaStream_t s) {
    std::size_t bytes = 0;
    CUNIBS_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, s));
    CubTemp t;
    CUNIBS_CHECK(cub::DeviceScan::ExclusiveSum(t.get(bytes), bytes, in, out, n, s));
}

void sort_keys(const std::uint64_t* in, std::uint64_t* out, std::size_t n, int end_bit, cudaStream_t s) {
    std::size_t bytes = 0;
    CUNIBS_CHECK(cub::DeviceRadixSort::SortKeys(nullptr, bytes, in, out, n, 0, end_bit, s));
    CubTemp t;
    CUNIBS_CHECK(cub::DeviceRadixSort::SortKeys(t.get(bytes), bytes, in, out, n, 0, end_bit, s));
}

template <typename V>
void sort_pairs(const std::uint32_t* kin, std::uint32_t* kout, const V* vin, V* vout, std::size_t n, int end_bit,
                cudaStream_t s) {
    std::size_t bytes = 0;
    CUNIBS_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, n, 0, end_bit, s));
    CubTemp t;
    CUNIBS_CHECK(cub::DeviceRadixSort::SortPairs(t.get(bytes), bytes, kin, kout, vin, vout, n, 0, end_bit, s));
}

template <typename T>
T read_one(const T* dev, cudaStream_t s) {
    T h{};
    CUNIBS_CHECK(cudaMemcpyAsync(&h, dev, sizeof(T), cudaMemcpyDeviceToHost, s));
    CUNIBS_CHECK(cudaStreamSynchronize(s));
    return h;
}

// --- slots ------------------------------------------------------------------------------------

__global__ void corner_slot_keys_kernel(const int* __restrict__ tets, const int* __restrict__ tags, std::int64_t nc,
                                        std::uint32_t* __restrict__ keys, int* __restrict__ ids) {
    const std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= nc) return;
    keys[q] = (static_cast<std::uint32_t>(tets[q]) << kTagBits) | static_cast<std::uint32_t>(tags[q >> 2]);
    ids[q] = static_cast<int>(q);
}

__global__ void key_heads_kernel(const std::uint32_t* __restrict__ keys, std::int64_t n, int* __restrict__ flags) {
    const std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q < n) flags[q] = (q == 0 || keys[q] != keys[q - 1]) ? 1 : 0;
}

// From the sorted (node, tag) keys: slot CSR, slot maps and the corner -> slot map.
__global__ void slot_fill_kernel(const std::uint32_t* __restrict__ keys, const int* __restrict__ flags,
                                 const int* __restrict__ pos, const int* __restrict__ corner, std::int64_t n,
                                 int* __restrict__ ptr, int* __restrict__ slot_node, int* __restrict__ slot_tag,
                                 std::uint32_t* __restrict__ slot_key, int* __restrict__ slot_of_corner) {
    const std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int s = pos[q] + flags[q] - 1;
    slot_of_corner[corner[q]] = s;
    if (flags[q]) {
        ptr[s] = static_cast<int>(q);
        slot_node[s] = static_cast<int>(keys[q] >> kTagBits);
        slot_tag[s] = static_cast<int>(keys[q] & ((1u << kTagBits) - 1));
        slot_key[s] = keys[q];
    }
}

__global__ void iota_kernel(int* __restrict__ out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = i;
}

// --- boundary marks ---------------------------------------------------------------------------

// One thread per face (tet e, corner `skip` left out). The face is on the outer boundary when only
// one tetrahedron holds all three of its nodes; the owners are counted along the incidence list of
// whichever of the three nodes has the shortest one. Every writer stores 1, so the marks need no
// ordering.
__global__ void outer_boundary_kernel(const int* __restrict__ tets, const int* __restrict__ n2c_ptr,
                                      const int* __restrict__ n2c_idx, std::int64_t n_face,
                                      int* __restrict__ is_boundary) {
    const std::int64_t f = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (f >= n_face) return;
    const int4 t = reinterpret_cast<const int4*>(tets)[f >> 2];
    const int all[4] = {t.x, t.y, t.z, t.w};
    const int skip = static_cast<int>(f & 3);
    int v0 = 0, v1 = 0, v2 = 0, m = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (i == skip) continue;
        if (m == 0) v0 = all[i];
        else if (m == 1) v1 = all[i];
        else v2 = all[i];
        ++m;
    }
    int pivot = v0, a = v1, b = v2;
    int len = n2c_ptr[v0 + 1] - n2c_ptr[v0];
    const int len1 = n2c_ptr[v1 + 1] - n2c_ptr[v1];
    const int len2 = n2c_ptr[v2 + 1] - n2c_ptr[v2];
    if (len1 < len) {
        len = len1;
        pivot = v1;
        a = v0;
        b = v2;
    }
    if (len2 < len) {
        len = len2;
        pivot = v2;
        a = v0;
        b = v1;
    }
    int owners = 0;
    for (int p = n2c_ptr[pivot], end = p + len; p < end && owners < 2; ++p) {
        const int4 o = reinterpret_cast<const int4*>(tets)[n2c_idx[p] >> 2];
        const bool has_a = o.x == a || o.y == a || o.z == a || o.w == a;
        const bool has_b = o.x == b || o.y == b || o.z == b || o.w == b;
        owners += has_a && has_b;
    }
    if (owners == 1) {
        is_boundary[v0] = 1;
        is_boundary[v1] = 1;
        is_boundary[v2] = 1;
    }
}

// A node carrying two tissues sits on the boundary of each tissue's submesh (recovery.py:127-158).
__global__ void mixed_node_kernel(const int* __restrict__ slot_node, int n_slots, int* __restrict__ is_boundary) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= 1 && s < n_slots && slot_node[s] == slot_node[s - 1]) is_boundary[slot_node[s]] = 1;
}

// --- small dense SPD algebra (lower triangle, row-major n x n, n <= 16) ----------------------

// Cholesky with the pivot floor 1e-12 * A[0][0]; false on a pivot at or below it.
template <int N>
__device__ bool chol4_factor(double (&A)[N * N]) {
    const double floor_pivot = 1e-12 * A[0];
    for (int j = 0; j < N; ++j) {
        double d = A[j * N + j];
        for (int k = 0; k < j; ++k) d = d - A[j * N + k] * A[j * N + k];
        if (!(d > floor_pivot)) return false;
        A[j * N + j] = sqrt(d);
        for (int i = j + 1; i < N; ++i) {
            double s = A[i * N + j];
            for (int k = 0; k < j; ++k) s = s - A[i * N + k] * A[j * N + k];
            A[i * N + j] = s / A[j * N + j];
        }
    }
    return true;
}

// --- SPR weights ------------------------------------------------------------------------------

// One thread per slot. Linear fit in the node-centred frame [1, (b - x_n)/h] over the barycentres of
// the slot's corners, evaluated at the node: solve A z = e_0, w_c = z . q_c. Boundary slots, fewer
// than four corners, a failed pivot or sum|w| > 8 take the volume-weighted average.
__global__ void spr_weights_kernel(const double* __restrict__ nodes, const double* __restrict__ bary,
                                   const float* __restrict__ vols32, const int* __restrict__ ptr,
                                   const int* __restrict__ idx, const int* __restrict__ slot_node,
                                   const int* __restrict__ is_boundary, int n_slots, float* __restrict__ w,
                                   int* __restrict__ fallback) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_slots) return;
    const int node = slot_node ? slot_node[s] : s;
    const int begin = ptr[s], end = ptr[s + 1], count = end - begin;
    fallback[s] = 0;
    if (count <= 0) return;
    const double xn[3] = {nodes[3 * node], nodes[3 * node + 1], nodes[3 * node + 2]};
    bool fit = count >= 4 && !is_boundary[node];
    double h = 1.0;
    if (fit) {
        h = 0.0;
        for (int p = begin; p < end; ++p) {
            const double* b = bary + 3 * static_cast<std::int64_t>(idx[p] >> 2);
#pragma unroll
            for (int a = 0; a < 3; ++a) h = fmax(h, fabs(b[a] - xn[a]));
        }
        fit = h > 0.0;
    }
    double z[4] = {1.0, 0.0, 0.0, 0.0};
    if (fit) {
        double A[16] = {};
        for (int p = begin; p < end; ++p) {
            const double* b = bary + 3 * static_cast<std::int64_t>(idx[p] >> 2);
            const double q[4] = {1.0, (b[0] - xn[0]) / h, (b[1] - xn[1]) / h, (b[2] - xn[2]) / h};
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j <= i; ++j) A[i * 4 + j] = fma(q[i], q[j], A[i * 4 + j]);
        }
        fit = chol4_factor<4>(A);
        if (fit) {
            double y[4];
            for (int i = 0; i < 4; ++i) {
                double t = (i == 0) ? 1.0 : 0.0;
                for (int k = 0; k < i; ++k) t = t - A[i * 4 + k] * y[k];
                y[i] = t / A[i * 4 + i];
            }
            for (int i = 3; i >= 0; --i) {
                double t = y[i];
                for (int k = i + 1; k < 4; ++k) t = t - A[k * 4 + i] * z[k];
                z[i] = t / A[i * 4 + i];
            }
        }
    }
    auto weight = [&](int p) {
        const double* b = bary + 3 * static_cast<std::int64_t>(idx[p] >> 2);
        const double q[4] = {1.0, (b[0] - xn[0]) / h, (b[1] - xn[1]) / h, (b[2] - xn[2]) / h};
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) acc = fma(z[i], q[i], acc);
        return acc;
    };
    if (fit) {
        double leb = 0.0;
        for (int p = begin; p < end; ++p) leb = leb + fabs(weight(p));
        fit = leb <= kMaxLebesgue;
    }
    if (!fit) {
        fallback[s] = 1;
        double total = 0.0;
        for (int p = begin; p < end; ++p) total = total + static_cast<double>(vols32[idx[p] >> 2]);
        const bool by_volume = total > 0.0;
        const double inv = by_volume ? 1.0 / total : 1.0 / static_cast<double>(count);
        for (int p = begin; p < end; ++p) {
            const double num = by_volume ? static_cast<double>(vols32[idx[p] >> 2]) : 1.0;
            w[p] = static_cast<float>(num * inv);
        }
        return;
    }
    for (int p = begin; p < end; ++p) w[p] = static_cast<float>(weight(p));
}

// --- harmonic patches ------------------------------------------------------------------------

// Ring candidates: every node of every tetrahedron of a slot, keyed (slot << nb) | node.
__global__ void ring_candidates_kernel(const int* __restrict__ tets, const int* __restrict__ idx,
                                       const int* __restrict__ slot_of_corner, std::int64_t nc, int nb,
                                       std::uint64_t* __restrict__ keys) {
    const std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= 4 * nc) return;
    const int corner = idx[q >> 2];
    const std::uint64_t slot = static_cast<std::uint32_t>(slot_of_corner[corner]);
    const int node = tets[4 * static_cast<std::int64_t>(corner >> 2) + (q & 3)];
    keys[q] = (slot << nb) | static_cast<std::uint32_t>(node);
}

__global__ void u64_heads_kernel(const std::uint64_t* __restrict__ keys, std::int64_t n, int* __restrict__ flags) {
    const std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q < n) flags[q] = (q == 0 || keys[q] != keys[q - 1]) ? 1 : 0;
}

// Compacts the distinct (slot, node) keys into a CSR over slots: entry node and its owning slot.
__global__ void compact_pairs_kernel(const std::uint64_t* __restrict__ keys, const int* __restrict__ flags,
                                     const int* __restrict__ pos, std::int64_t n, int nb, int* __restrict__ node_out,
                                     int* __restrict__ slot_out) {
    const std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= n || !flags[q]) return;
    const int p = pos[q];
    node_out[p] = static_cast<int>(keys[q] & ((std::uint64_t{1} << nb) - 1));
    slot_out[p] = static_cast<int>(keys[q] >> nb);
}

// ptr[s] = first entry whose owning slot is >= s (owners ascending).
__global__ void lower_bound_ptr_kernel(const int* __restrict__ owner, std::int64_t len, int n_seg,
                                       int* __restrict__ ptr) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s > n_seg) return;
    std::int64_t lo = 0, hi = len;
    while (lo < hi) {
        const std::int64_t mid = (lo + hi) >> 1;
        if (owner[mid] < s) lo = mid + 1;
        else hi = mid;
    }
    ptr[s] = static_cast<int>(lo);
}

// For each ring entry (slot s, node m): the slot (m, tag of s). It exists: m was reached through a
// tetrahedron of s's own tissue.
__global__ void neighbour_slot_kernel(const int* __restrict__ ring_node, const int* __restrict__ ring_owner,
                                      std::int64_t n, const int* __restrict__ slot_tag,
                                      const std::uint32_t* __restrict__ slot_key, int n_slots,
                                      int* __restrict__ neighbour) {
    const std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const std::uint32_t key = (static_cast<std::uint32_t>(ring_node[q]) << kTagBits) |
                              static_cast<std::uint32_t>(slot_tag[ring_owner[q]]);
    int lo = 0, hi = n_slots;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (slot_key[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    neighbour[q] = lo;
}

__global__ void patch_count_kernel(const int* __restrict__ rptr, const int* __restrict__ neighbour, int n_slots,
                                   std::int64_t* __restrict__ count) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_slots) return;
    const int begin = rptr[s], end = rptr[s + 1];
    std::int64_t c = end - begin;
    if (c < kMinPatchNodes) {
        c = 0;
        for (int j = begin; j < end; ++j) c += rptr[neighbour[j] + 1] - rptr[neighbour[j]];
    }
    count[s] = c;
}

__global__ void patch_fill_kernel(const int* __restrict__ rptr, const int* __restrict__ rnode,
                                  const int* __restrict__ neighbour, const std::int64_t* __restrict__ off,
                                  int n_slots, int nb, std::uint64_t* __restrict__ keys) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_slots) return;
    const int begin = rptr[s], end = rptr[s + 1];
    const std::uint64_t hi = static_cast<std::uint64_t>(s) << nb;
    std::int64_t o = off[s];
    if (end - begin >= kMinPatchNodes) {
        for (int j = begin; j < end; ++j) keys[o++] = hi | static_cast<std::uint32_t>(rnode[j]);
        return;
    }
    for (int j = begin; j < end; ++j) {
        const int nbs = neighbour[j];
        for (int t = rptr[nbs]; t < rptr[nbs + 1]; ++t) keys[o++] = hi | static_cast<std::uint32_t>(rnode[t]);
    }
}

// --- harmonic weights -------------------------------------------------------------------------

__device__ __forceinline__ int eval_basis(int rung, double u, double v, double t, double* p) {
    p[0] = 1.0;
    p[1] = u;
    p[2] = v;
    p[3] = t;
    if (rung == 2) return 4;
    p[4] = u * u - v * v;
    p[5] = v * v - t * t;
    p[6] = u * v;
    p[7] = u * t;
    p[8] = v * t;
    if (rung == 1) return 9;
    const double uu = u * u, vv = v * v, tt = t * t;
    p[9] = t * (2.0 * tt - 3.0 * uu - 3.0 * vv);
    p[10] = u * (4.0 * tt - uu - vv);
    p[11] = v * (4.0 * tt - uu - vv);
    p[12] = t * (uu - vv);
    p[13] = u * v * t;
    p[14] = u * (uu - 3.0 * vv);
    p[15] = v * (3.0 * uu - vv);
    return 16;
}

constexpr int kFitWarps = 4;
constexpr int kMaxTerms = 16;

struct FitShared {
    double q[32 * kMaxTerms];         // basis of one chunk of 32 patch entries
    double a[kMaxTerms * kMaxTerms];  // normal matrix, then its Cholesky factor in place
    double y[3 * kMaxTerms];
    double z[3 * kMaxTerms];          // rows 1..3 of the inverse
    int bad;
};

// One rung of the potential fit for the warp's slot. Returns whether it was accepted; the weights
// are written either way (a later rung overwrites them).
__device__ bool fit_rung(int rung, const double* __restrict__ nodes, const int* __restrict__ pidx, int begin,
                         int end, const double* xn, double h, float4* __restrict__ wq, FitShared& sh, int lane) {
    const int n = rung == 0 ? 16 : (rung == 1 ? 9 : 4);
    const int min_patch = rung == 0 ? 20 : (rung == 1 ? 9 : 4);
    if (end - begin < min_patch) return false;
    const int entries = n * (n + 1) / 2;
    // Lane l owns lower-triangle entries l, l+32, ... (at most 5 for n = 16).
    int ei[5], ej[5];
    double acc[5];
#pragma unroll
    for (int t = 0; t < 5; ++t) {
        const int e = lane + 32 * t;
        int i = 0;
        while ((i + 1) * (i + 2) / 2 <= e) ++i;
        ei[t] = i;
        ej[t] = e - i * (i + 1) / 2;
        acc[t] = 0.0;
    }
    for (int base = begin; base < end; base += 32) {
        const int cnt = min(32, end - base);
        if (lane < cnt) {
            const int m = pidx[base + lane];
            const double u = (nodes[3 * m] * 1e-3 - xn[0]) / h;
            const double v = (nodes[3 * m + 1] * 1e-3 - xn[1]) / h;
            const double t = (nodes[3 * m + 2] * 1e-3 - xn[2]) / h;
            eval_basis(rung, u, v, t, sh.q + lane * kMaxTerms);
        }
        __syncwarp();
        for (int p = 0; p < cnt; ++p) {
            const double* q = sh.q + p * kMaxTerms;
#pragma unroll
            for (int t = 0; t < 5; ++t)
                if (lane + 32 * t < entries) acc[t] = fma(q[ei[t]], q[ej[t]], acc[t]);
        }
        __syncwarp();
    }
#pragma unroll
    for (int t = 0; t < 5; ++t)
        if (lane + 32 * t < entries) sh.a[ei[t] * n + ej[t]] = acc[t];
    if (lane == 0) sh.bad = 0;
    __syncwarp();
    const double floor_pivot = 1e-12 * sh.a[0];
    __syncwarp();
    for (int j = 0; j < n; ++j) {
        if (lane == j) {
            double d = sh.a[j * n + j];
            for (int k = 0; k < j; ++k) d = d - sh.a[j * n + k] * sh.a[j * n + k];
            if (!(d > floor_pivot)) sh.bad = 1;
            else sh.a[j * n + j] = sqrt(d);
        }
        __syncwarp();
        if (sh.bad) return false;
        if (lane > j && lane < n) {
            double s = sh.a[lane * n + j];
            for (int k = 0; k < j; ++k) s = s - sh.a[lane * n + k] * sh.a[j * n + k];
            sh.a[lane * n + j] = s / sh.a[j * n + j];
        }
        __syncwarp();
    }
    if (lane < 3) {
        const int row = lane + 1;
        double* y = sh.y + lane * kMaxTerms;
        double* z = sh.z + lane * kMaxTerms;
        for (int i = 0; i < n; ++i) {
            double s = (i == row) ? 1.0 : 0.0;
            for (int k = 0; k < i; ++k) s = s - sh.a[i * n + k] * y[k];
            y[i] = s / sh.a[i * n + i];
        }
        for (int i = n - 1; i >= 0; --i) {
            double s = y[i];
            for (int k = i + 1; k < n; ++k) s = s - sh.a[k * n + i] * z[k];
            z[i] = s / sh.a[i * n + i];
        }
    }
    __syncwarp();
    double part[3] = {0.0, 0.0, 0.0};
    for (int p = begin + lane; p < end; p += 32) {
        const int m = pidx[p];
        double q[kMaxTerms];
        eval_basis(rung, (nodes[3 * m] * 1e-3 - xn[0]) / h, (nodes[3 * m + 1] * 1e-3 - xn[1]) / h,
                   (nodes[3 * m + 2] * 1e-3 - xn[2]) / h, q);
        float out[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double g = 0.0;
            for (int i = 0; i < n; ++i) g = fma(sh.z[c * kMaxTerms + i], q[i], g);
            part[c] = part[c] + fabs(g);
            out[c] = static_cast<float>(g / h);
        }
        wq[p] = make_float4(out[0], out[1], out[2], __int_as_float(m));
    }
    // Fixed tree: lane l folds in lane l + off for off = 16, 8, 4, 2, 1; lane 0 decides.
#pragma unroll
    for (int c = 0; c < 3; ++c)
        for (int off = 16; off >= 1; off >>= 1) part[c] = part[c] + __shfl_down_sync(0xffffffffu, part[c], off);
    int ok = 0;
    if (lane == 0) ok = fmax(part[0], fmax(part[1], part[2])) <= kMaxGradAmp;
    return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

__global__ void __launch_bounds__(32 * kFitWarps) harmonic_weights_kernel(const double* __restrict__ nodes,
                                                                          const int* __restrict__ pptr,
                                                                          const int* __restrict__ pidx,
                                                                          const int* __restrict__ slot_node,
                                                                          int n_slots, float4* __restrict__ wq,
                                                                          int* __restrict__ status) {
    __shared__ FitShared shared[kFitWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.x * kFitWarps + warp;
    if (s >= n_slots) return;  // warp-uniform
    FitShared& sh = shared[warp];
    const int begin = pptr[s], end = pptr[s + 1];
    const int node = slot_node[s];
    const double xn[3] = {nodes[3 * node] * 1e-3, nodes[3 * node + 1] * 1e-3, nodes[3 * node + 2] * 1e-3};
    double h = 0.0;
    for (int p = begin + lane; p < end; p += 32) {
        const int m = pidx[p];
#pragma unroll
        for (int a = 0; a < 3; ++a) h = fmax(h, fabs(nodes[3 * m + a] * 1e-3 - xn[a]));
    }
    for (int off = 16; off >= 1; off >>= 1) h = fmax(h, __shfl_xor_sync(0xffffffffu, h, off));
    int rung = 3;
    if (h > 0.0) {
        for (int t = 0; t < 3 && rung == 3; ++t)
            if (fit_rung(t, nodes, pidx, begin, end, xn, h, wq, sh, lane)) rung = t;
    }
    if (rung == 3)
        for (int p = begin + lane; p < end; p += 32) wq[p] = make_float4(0.f, 0.f, 0.f, __int_as_float(pidx[p]));
    if (lane == 0) status[s] = rung;
}

// --- apply ------------------------------------------------------------------------------------

// Harmonic: E_s = -sum_p w_p v_m - dA/dt(node), FP64 accumulation in patch order; one thread per
// (slot, column), K column threads of a slot adjacent so the operator entry is one broadcast load.
__global__ void harmonic_apply_kernel(const float4* __restrict__ wq, const int* __restrict__ pptr,
                                      const int* __restrict__ slot_node, int n_slots, const double* __restrict__ x,
                                      int K, int ground, const float* __restrict__ dadt_nodes, int n_nodes, int k,
                                      float* __restrict__ e_slots) {
    const std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int s = static_cast<int>(q / K), c = static_cast<int>(q % K);
    if (s >= n_slots || c >= k) return;
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int p = pptr[s], end = pptr[s + 1]; p < end; ++p) {
        const float4 e = wq[p];
        const int m = __float_as_int(e.w);
        const double vm = (m == ground) ? 0.0 : x[static_cast<std::int64_t>(m - (m > ground ? 1 : 0)) * K + c];
        ax = fma(static_cast<double>(e.x), vm, ax);
        ay = fma(static_cast<double>(e.y), vm, ay);
        az = fma(static_cast<double>(e.z), vm, az);
    }
    const int node = slot_node[s];
    const float* da = dadt_nodes + (static_cast<std::int64_t>(c) * n_nodes + node) * 3;
    float* o = e_slots + (static_cast<std::int64_t>(c) * n_slots + s) * 3;
    o[0] = static_cast<float>(-ax - static_cast<double>(da[0]));
    o[1] = static_cast<float>(-ay - static_cast<double>(da[1]));
    o[2] = static_cast<float>(-az - static_cast<double>(da[2]));
}

// The same with one thread per (slot, column pair): one operator load serves both columns and the
// potential pair is one 16-byte gather; each column's sums are bitwise the one-column kernel's.
__global__ void harmonic_apply_pair_kernel(const float4* __restrict__ wq, const int* __restrict__ pptr,
                                           const int* __restrict__ slot_node, int n_slots,
                                           const double* __restrict__ x, int K, int ground,
                                           const float* __restrict__ dadt_nodes, int n_nodes, int k,
                                           float* __restrict__ e_slots) {
    const std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int L = K / 2;
    const int s = static_cast<int>(q / L), c0 = 2 * static_cast<int>(q % L);
    if (s >= n_slots || c0 >= k) return;
    const double2* xv = reinterpret_cast<const double2*>(x);
    double ax0 = 0.0, ay0 = 0.0, az0 = 0.0, ax1 = 0.0, ay1 = 0.0, az1 = 0.0;
    for (int p = pptr[s], end = pptr[s + 1]; p < end; ++p) {
        const float4 e = wq[p];
        const int m = __float_as_int(e.w);
        const double2 vm = (m == ground) ? make_double2(0.0, 0.0)
                                         : xv[static_cast<std::int64_t>(m - (m > ground ? 1 : 0)) * L + c0 / 2];
        ax0 = fma(static_cast<double>(e.x), vm.x, ax0);
        ay0 = fma(static_cast<double>(e.y), vm.x, ay0);
        az0 = fma(static_cast<double>(e.z), vm.x, az0);
        ax1 = fma(static_cast<double>(e.x), vm.y, ax1);
        ay1 = fma(static_cast<double>(e.y), vm.y, ay1);
        az1 = fma(static_cast<double>(e.z), vm.y, az1);
    }
    const int node = slot_node[s];
    const double a[2][3] = {{ax0, ay0, az0}, {ax1, ay1, az1}};
    for (int h = 0; h < 2 && c0 + h < k; ++h) {
        const int c = c0 + h;
        const float* da = dadt_nodes + (static_cast<std::int64_t>(c) * n_nodes + node) * 3;
        float* o = e_slots + (static_cast<std::int64_t>(c) * n_slots + s) * 3;
        o[0] = static_cast<float>(-a[h][0] - static_cast<double>(da[0]));
        o[1] = static_cast<float>(-a[h][1] - static_cast<double>(da[1]));
        o[2] = static_cast<float>(-a[h][2] - static_cast<double>(da[2]));
    }
}

// SPR: E_s = sum_c w_c E_{e(c)}, FP32 accumulation in slot order; one thread per (slot, column).
__global__ void spr_apply_kernel(const float* __restrict__ w, const int* __restrict__ ptr,
                                 const int* __restrict__ idx, int n_slots, const float* __restrict__ e_elem,
                                 int n_tets, int k, float* __restrict__ e_slots) {
    const std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<std::int64_t>(n_slots) * k) return;
    const int c = static_cast<int>(q / n_slots), s = static_cast<int>(q % n_slots);
    const float* ec = e_elem + static_cast<std::int64_t>(c) * n_tets * 3;
    float ax = 0.f, ay = 0.f, az = 0.f;
    for (int p = ptr[s], end = ptr[s + 1]; p < end; ++p) {
        const float wp = w[p];
        const float* ee = ec + 3 * static_cast<std::int64_t>(idx[p] >> 2);
        ax = fmaf(wp, ee[0], ax);
        ay = fmaf(wp, ee[1], ay);
        az = fmaf(wp, ee[2], az);
    }
    float* o = e_slots + q * 3;
    o[0] = ax;
    o[1] = ay;
    o[2] = az;
}

// Barycentre sample: the mean of the four corner slots, FP64, then |E|.
__global__ void recover_elements_kernel(const float* __restrict__ e_slots, int n_slots,
                                        const int* __restrict__ slot_of_corner, int n_tets, int k,
                                        float* __restrict__ E, float* __restrict__ magn) {
    const std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<std::int64_t>(n_tets) * k) return;
    const int c = static_cast<int>(q / n_tets), e = static_cast<int>(q % n_tets);
    const int4 sl = reinterpret_cast<const int4*>(slot_of_corner)[e];
    const int slots[4] = {sl.x, sl.y, sl.z, sl.w};
    const float* src = e_slots + static_cast<std::int64_t>(c) * n_slots * 3;
    double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float* v = src + 3 * static_cast<std::int64_t>(slots[i]);
        sx = sx + static_cast<double>(v[0]);
        sy = sy + static_cast<double>(v[1]);
        sz = sz + static_cast<double>(v[2]);
    }
    sx = sx * 0.25;
    sy = sy * 0.25;
    sz = sz * 0.25;
    if (E != nullptr) {
        float* o = E + q * 3;
        o[0] = static_cast<float>(sx);
        o[1] = static_cast<float>(sy);
        o[2] = static_cast<float>(sz);
    }
    magn[q] = static_cast<float>(sqrt(sx * sx + sy * sy + sz * sz));
}

// (node << 4 | tag) slots of the corners, and everything derived from them.
void build_tissue_slots(const Mesh& m, RecoveryOp& op, DevArray<std::uint32_t>& slot_key, cudaStream_t s) {
    const std::int64_t nc = 4 * static_cast<std::int64_t>(m.n_tets);
    DevArray<std::uint32_t> keys(nc), keys_sorted(nc);
    DevArray<int> ids(nc), flags(nc), pos(nc);
    op.idx.resize(nc);
    corner_slot_keys_kernel<<<grid_for(nc), kBlock, 0, s>>>(m.tets.get(), m.tags.get(), nc, keys.get(), ids.get());
    count_launch();
    sort_pairs(keys.get(), keys_sorted.get(), ids.get(), op.idx.get(), nc, bits_for(m.n_nodes) + kTagBits, s);
    key_heads_kernel<<<grid_for(nc), kBlock, 0, s>>>(keys_sorted.get(), nc, flags.get());
    count_launch();
    exclusive_scan(flags.get(), pos.get(), nc, s);
    const int n_slots = read_one(pos.get() + nc - 1, s) + read_one(flags.get() + nc - 1, s);
    op.n_slots = n_slots;
    op.ptr.resize(n_slots + 1);
    op.slot_node.resize(n_slots);
    op.slot_tag.resize(n_slots);
    slot_key.resize(n_slots);
    op.slot_of_corner.resize(nc);
    slot_fill_kernel<<<grid_for(nc), kBlock, 0, s>>>(keys_sorted.get(), flags.get(), pos.get(), op.idx.get(), nc,
                                                       op.ptr.get(), op.slot_node.get(), op.slot_tag.get(),
                                                       slot_key.get(), op.slot_of_corner.get());
    count_launch();
    const int total = static_cast<int>(nc);
    CUNIBS_CHECK(cudaMemcpyAsync(op.ptr.get() + n_slots, &total, sizeof(int), cudaMemcpyHostToDevice, s));
    CUNIBS_CHECK(cudaStreamSynchronize(s));
    CUNIBS_LAUNCH_CHECK("tissue slots");
}

void build_boundary(const Mesh& m, RecoveryOp& op, bool tissue, cudaStream_t s) {
    op.is_boundary.resize(m.n_nodes);
    op.is_boundary.zero(s);
    const std::int64_t n_face = 4 * static_cast<std::int64_t>(m.n_tets);
    outer_boundary_kernel<<<grid_for(n_face), kBlock, 0, s>>>(m.tets.get(), m.n2c_ptr.get(), m.n2c_idx.get(), n_face,
                                                              op.is_boundary.get());
    count_launch();
    if (tissue) {
        mixed_node_kernel<<<grid_for(op.n_slots), kBlock, 0, s>>>(op.slot_node.get(), op.n_slots,
                                                                  op.is_boundary.get());
        count_launch();
    }
    CUNIBS_LAUNCH_CHECK("boundary marks");
}

void build_spr(const Mesh& m, RecoveryOp& op, bool node_slots, cudaStream_t s) {
    op.nnz = 4 * static_cast<std::int64_t>(m.n_tets);
    op.w.resize(op.nnz);
    DevArray<int> fallback(op.n_slots);
    spr_weights_kernel<<<grid_for(op.n_slots), kBlock, 0, s>>>(
        m.nodes.get(), m.bary.get(), m.vols32.get(), node_slots ? m.n2c_ptr.get() : op.ptr.get(),
        node_slots ? m.n2c_idx.get() : op.idx.get(), node_slots ? nullptr : op.slot_node.get(), op.is_boundary.get(),
        op.n_slots, op.w.get(), fallback.get());
    count_launch();
    CUNIBS_LAUNCH_CHECK("spr weights");
    const std::vector<int> fb = fallback.to_host(s);
    op.n_fallback = 0;
    for (int f : fb) op.n_fallback += f;
}

void build_harmonic(const Mesh& m, RecoveryOp& op, const DevArray<std::uint32_t>& slot_key, cudaStream_t s) {
    const std::int64_t nc = 4 * static_cast<std::int64_t>(m.n_tets);
    const int S = op.n_slots;
    const int nb = bits_for(m.n_nodes);
    const int key_bits = nb + bits_for(S);
    if (key_bits > 63) fail(kEInval, "mesh too large for the recovery patch keys");
    // First rings: distinct nodes of each slot's tetrahedra.
    DevArray<int> rptr(S + 1), rnode, rowner, neighbour;
    std::int64_t n_ring = 0;
    {
        DevArray<std::uint64_t> keys(4 * nc), sorted(4 * nc);
        ring_candidates_kernel<<<grid_for(4 * nc), kBlock, 0, s>>>(m.tets.get(), op.idx.get(),
                                                                   op.slot_of_corner.get(), nc, nb, keys.get());
        count_launch();
        sort_keys(keys.get(), sorted.get(), 4 * nc, key_bits, s);
        keys.release();
        DevArray<int> flags(4 * nc), pos(4 * nc);
        u64_heads_kernel<<<grid_for(4 * nc), kBlock, 0, s>>>(sorted.get(), 4 * nc, flags.get());
        count_launch();
        exclusive_scan(flags.get(), pos.get(), 4 * nc, s);
        n_ring = read_one(pos.get() + 4 * nc - 1, s) + read_one(flags.get() + 4 * nc - 1, s);
        rnode.resize(n_ring);
        rowner.resize(n_ring);
        compact_pairs_kernel<<<grid_for(4 * nc), kBlock, 0, s>>>(sorted.get(), flags.get(), pos.get(), 4 * nc, nb,
                                                                 rnode.get(), rowner.get());
        count_launch();
        lower_bound_ptr_kernel<<<grid_for(S + 1), kBlock, 0, s>>>(rowner.get(), n_ring, S, rptr.get());
        count_launch();
        neighbour.resize(n_ring);
        neighbour_slot_kernel<<<grid_for(n_ring), kBlock, 0, s>>>(rnode.get(), rowner.get(), n_ring,
                                                                  op.slot_tag.get(), slot_key.get(), S,
                                                                  neighbour.get());
        count_launch();
        CUNIBS_LAUNCH_CHECK("first rings");
    }
    // Patches: the ring, or the union of the neighbours' rings where the ring is small.
    DevArray<std::int64_t> count(S + 1), off(S + 1);
    patch_count_kernel<<<grid_for(S), kBlock, 0, s>>>(rptr.get(), neighbour.get(), S, count.get());
    count_launch();
    CUNIBS_CHECK(cudaMemsetAsync(count.get() + S, 0, sizeof(std::int64_t), s));
    exclusive_scan(count.get(), off.get(), S + 1, s);
    const std::int64_t n_cand = read_one(off.get() + S, s);
    DevArray<std::uint64_t> keys(n_cand), sorted(n_cand);
    patch_fill_kernel<<<grid_for(S), kBlock, 0, s>>>(rptr.get(), rnode.get(), neighbour.get(), off.get(), S, nb,
                                                     keys.get());
    count_launch();
    sort_keys(keys.get(), sorted.get(), n_cand, key_bits, s);
    keys.release();
    DevArray<int> flags(n_cand), pos(n_cand);
    u64_heads_kernel<<<grid_for(n_cand), kBlock, 0, s>>>(sorted.get(), n_cand, flags.get());
    count_launch();
    exclusive_scan(flags.get(), pos.get(), n_cand, s);
    const std::int64_t nnz = read_one(pos.get() + n_cand - 1, s) + read_one(flags.get() + n_cand - 1, s);
    if (nnz >= (std::int64_t{1} << 31)) fail(kEInval, "recovery patches exceed 2^31 entries");
    DevArray<int> powner(nnz);
    op.pidx.resize(nnz);
    compact_pairs_kernel<<<grid_for(n_cand), kBlock, 0, s>>>(sorted.get(), flags.get(), pos.get(), n_cand, nb,
                                                             op.pidx.get(), powner.get());
    count_launch();
    op.ptr.resize(S + 1);  // the patch CSR replaces the corner CSR as the operator's rows
    lower_bound_ptr_kernel<<<grid_for(S + 1), kBlock, 0, s>>>(powner.get(), nnz, S, op.ptr.get());
    count_launch();
    op.nnz = nnz;
    op.wq.resize(nnz);
    op.status.resize(S);
    harmonic_weights_kernel<<<grid_for(S, kFitWarps), 32 * kFitWarps, 0, s>>>(
        m.nodes.get(), op.ptr.get(), op.pidx.get(), op.slot_node.get(), S, op.wq.get(), op.status.get());
    count_launch();
    CUNIBS_LAUNCH_CHECK("harmonic weights");
    const std::vector<int> st = op.status.to_host(s);
    op.n_fallback = op.n_undetermined = 0;
    for (int v : st) {
        op.n_fallback += v >= 2;
        op.n_undetermined += v == 3;
    }
}

}  // namespace

void build_recovery(const Mesh& m, RecoveryOp& op, int mode, cudaStream_t s) {
    op = RecoveryOp();
    op.mode = mode;
    if (mode == kRecSprGlobal) {
        op.n_slots = m.n_nodes;
        op.slot_node.resize(m.n_nodes);
        iota_kernel<<<grid_for(m.n_nodes), kBlock, 0, s>>>(op.slot_node.get(), m.n_nodes);
        count_launch();
        build_boundary(m, op, false, s);
        build_spr(m, op, true, s);
        return;
    }
    if (mode != kRecSprTissue && mode != kRecHarmonic) fail(kEInval, "unknown recovery mode");
    DevArray<std::uint32_t> slot_key;
    build_tissue_slots(m, op, slot_key, s);
    if (mode == kRecSprTissue) {
        build_boundary(m, op, true, s);
        build_spr(m, op, false, s);
    } else {
        build_harmonic(m, op, slot_key, s);
    }
}

const int* recovery_slot_of_corner(const Mesh& m, const RecoveryOp& op) {
    return op.mode == kRecSprGlobal ? m.tets.get() : op.slot_of_corner.get();
}

void apply_recovery(const Mesh& m, const RecoveryOp& op, const double* x_red, int K, const float* dadt_nodes,
                    const float* e_elem, int k, float* e_slots, float* E, float* magn, cudaStream_t s) {
    if (op.mode == kRecHarmonic) {
        const char* lanes = std::getenv("CUNIBS_LANE_COLUMNS");
        if (K % 2 == 0 && !(lanes != nullptr && lanes[0] == '1')) {
            const std::int64_t n = static_cast<std::int64_t>(op.n_slots) * (K / 2);
            harmonic_apply_pair_kernel<<<grid_for(n), kBlock, 0, s>>>(op.wq.get(), op.ptr.get(), op.slot_node.get(),
                                                                      op.n_slots, x_red, K, m.ground, dadt_nodes,
                                                                      m.n_nodes, k, e_slots);
        } else {
            const std::int64_t n = static_cast<std::int64_t>(op.n_slots) * K;
            harmonic_apply_kernel<<<grid_for(n), kBlock, 0, s>>>(op.wq.get(), op.ptr.get(), op.slot_node.get(),
                                                                 op.n_slots, x_red, K, m.ground, dadt_nodes, m.n_nodes,
                                                                 k, e_slots);
        }
    } else {
        const bool nodes = op.mode == kRecSprGlobal;
        const std::int64_t n = static_cast<std::int64_t>(op.n_slots) * k;
        spr_apply_kernel<<<grid_for(n), kBlock, 0, s>>>(op.w.get(), nodes ? m.n2c_ptr.get() : op.ptr.get(),
                                                        nodes ? m.n2c_idx.get() : op.idx.get(), op.n_slots, e_elem,
                                                        m.n_tets, k, e_slots);
    }
    count_launch();
    const std::int64_t ne = static_cast<std::int64_t>(m.n_tets) * k;
    recover_elements_kernel<<<grid_for(ne), kBlock, 0, s>>>(e_slots, op.n_slots, recovery_slot_of_corner(m, op),
                                                             m.n_tets, k, E, magn);
    count_launch();
    CUNIBS_LAUNCH_CHECK("recovery apply");
}

}  // namespace cunibs
