// Block PCG with a smoothed-aggregation V-cycle, for k right-hand sides in lockstep.
//
// Two precisions share one set of kernels, templated on the arithmetic type T:
//   * plain: FP64 PCG over an FP64 V-cycle (the baseline method).
//   * mixed: FP64 iterative refinement. Each outer step forms the true residual B - A X in FP64,
//     then an inner PCG in FP32 (FP32 matrix values, FP32 vectors, FP32 V-cycle; FP64 inner
//     products) reduces it by `inner_reduction`, and X += correction in FP64.
//
// Layout: every dense operand is row-major (n, K), so a mesh node's K values are contiguous. Every
// row-parallel kernel runs on tiles of kTileRows rows with K lanes per row (lane = column): a lane
// walks its row's nonzeros in CSR order, so each column's sum has the same order whatever K is.
// Column reductions are two-stage and fixed-order (rows of a tile sequentially, then tiles in a
// fixed tree by the grid's last block), so a placement's answer is bitwise independent of the block
// width and of the other placements in its block. A column that meets its tolerance freezes
// (alpha = beta = 0) on the device, which keeps the iteration body identical from launch to launch
// and lets it replay as a CUDA graph with the convergence test read back only every few iterations.
//
// Reference semantics restated: solver.cpp:84-198 (lockstep k-RHS PCG, per-column freeze,
// ||r||/||b|| <= tol), block_cg.cu:188-226 (freeze via alpha = beta = 0), vcycle.cu:560-648
// (cycle order: Chebyshev pre-smooth from zero, residual, restrict; dense coarse solve; prolongate,
// Chebyshev post-smooth).
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <memory>
#include <tuple>
#include <type_traits>

#include "internal.hpp"

namespace cunibs {
namespace {

constexpr int kTileRows = 64;

template <int K>
constexpr int tile_threads() {
    return kTileRows * K;
}

int n_tiles(int n) { return (n + kTileRows - 1) / kTileRows; }
__device__ __forceinline__ int n_tiles_dev(int n) { return (n + kTileRows - 1) / kTileRows; }

// --- deterministic column reductions ---------------------------------------------------------

// True in the last block to finish; that block then owns the final reduction. It resets the
// arrival counter, which no other block touches again in this launch.
__device__ __forceinline__ bool last_block(unsigned* counter) {
    __shared__ bool is_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(counter, 1u);
        is_last = (prev == gridDim.x - 1);
        if (is_last) *counter = 0u;
    }
    __syncthreads();
    return is_last;
}

// In the last block: total[c] = fixed tree over kTileRows strided sums of the tile partials.
template <int K>
__device__ __forceinline__ void final_reduce(const double* __restrict__ partials, int tiles, double* total) {
    __shared__ double sh[kTileRows][K];
    const int slot = threadIdx.x / K;
    const int c = threadIdx.x % K;
    double acc = 0.0;
    for (int t = slot; t < tiles; t += kTileRows) acc += __ldcg(partials + static_cast<long>(c) * tiles + t);
    sh[slot][c] = acc;
    __syncthreads();
#pragma unroll
    for (int off = kTileRows / 2; off > 0; off >>= 1) {
        if (slot < off) sh[slot][c] += sh[slot + off][c];
        __syncthreads();
    }
    if (threadIdx.x < K) total[threadIdx.x] = sh[0][threadIdx.x];
    __syncthreads();
}

// acc + sum of val[p] * x[col[p] * ld + c] over p = p0, p0 + S, ... < e, added in that order.
// Operators walked by sub-lanes (S > 1, the coarse levels' long rows) take their terms eight at a
// time: every index and value load of a batch is issued, then every gather, then the multiply-adds
// in order (predicated off past the row's end). One lane per row (S = 1, the finest levels) takes
// the plain loop: measured on the 1M-tet operator (178k rows, ~15 entries per row, 8 columns) the
// batches of 4, 8, 12 and 16 cost registers and occupancy for more than the chains they put in
// flight (PCG iteration 0.266 ms at 8, 0.247 ms plain). Both keep the plain loop's order of
// additions, so the result does not depend on the batch.
template <typename T, int S, typename TX = T>
__device__ __forceinline__ T strided_dot(const int* __restrict__ col, const T* __restrict__ val,
                                         const TX* __restrict__ x, int p, int e, long ld, int c, T acc) {
    constexpr int B = S == 1 ? 1 : 8;
    for (; p < e; p += B * S) {
        int cj[B];
        T vj[B];
        TX xj[B];
#pragma unroll
        for (int j = 0; j < B; ++j) {
            const int q = p + j * S;
            const bool ok = q < e;
            cj[j] = ok ? col[q] : 0;
            vj[j] = ok ? val[q] : T(0);
        }
#pragma unroll
        for (int j = 0; j < B; ++j) xj[j] = (p + j * S < e) ? x[cj[j] * ld + c] : TX(0);
#pragma unroll
        for (int j = 0; j < B; ++j)
            if (p + j * S < e) acc += vj[j] * static_cast<T>(xj[j]);
    }
    return acc;
}

template <typename T>
__device__ __forceinline__ T row_dot(const int* __restrict__ ptr, const int* __restrict__ col,
                                     const T* __restrict__ val, const T* __restrict__ x, int row, int c, int K) {
    return strided_dot<T, 1>(col, val, x, ptr[row], ptr[row + 1], K, c, T(0));
}

// Programmatic dependent launch (sm_90 and later): a kernel of the solve loop launched with the
// programmatic-serialization attribute may be scheduled while its predecessor in the stream drains.
// It waits here, before touching any memory, for that predecessor to complete and its writes to be
// visible, and at once lets its own successor be scheduled, so block dispatch and launch latency
// overlap the previous kernel's tail. Launched without the attribute, both are no-ops.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// --- V-cycle kernels ---------------------------------------------------------------------
//
// A row group is TPR x K threads: K lanes per column-slot (lane = column, so a nonzero's K values
// are one coalesced read) times TPR sub-lanes that stride the row's nonzeros. TPR is chosen per
// operator from its shape alone (choose_tpr), never from K, and the TPR partial sums are combined
// in shared memory by a sequential walk over the sub-lanes: the summation order of every column is
// then fixed by the operator, which keeps a placement's answer bitwise independent of the block
// width.

template <int K, int TPR>
struct Group {
    static constexpr int kThreads = TPR * K;
    static constexpr int kRows = kThreads >= 256 ? 1 : 256 / kThreads;
    static constexpr int kBlock = kRows * kThreads;
};

template <typename T, int K, int TPR>
struct RowSlot {
    int row;  // global row
    int r;    // row within the block
    int sub;  // sub-lane
    int c;    // column
    __device__ __forceinline__ RowSlot() {
        const int t = threadIdx.x;
        r = t / Group<K, TPR>::kThreads;
        sub = (t / K) % TPR;
        c = t % K;
        row = blockIdx.x * Group<K, TPR>::kRows + r;
    }
};

// Row-times-block for one (row, column): each sub-lane sums its strided share of the row, then the
// shares are combined by one fixed pairing tree ((s0+s4)+(s2+s6))+((s1+s5)+(s3+s7)) for TPR = 8:
// as an XOR butterfly over the sub-lanes when a row group fits in a warp (every sub-lane ends with
// the same total, since each pair adds the same two values and addition is commutative), otherwise
// by sub-lane 0 in shared memory. The tree depends on TPR alone, never on K. Every thread of the
// block must call this.
template <typename T, int K, int TPR, int ROWS, typename TX = T>
__device__ __forceinline__ T group_row_dot(const int* __restrict__ ptr, const int* __restrict__ col,
                                           const T* __restrict__ val, const TX* __restrict__ x, int row, int r,
                                           int sub, int c, bool valid) {
    T acc = T(0);
    if (valid) acc = strided_dot<T, TPR, TX>(col, val, x, ptr[row] + sub, ptr[row + 1], K, c, acc);
    if constexpr (TPR == 1) {
        return acc;
    } else if constexpr (TPR * K <= kWarp) {
#pragma unroll
        for (int off = TPR / 2; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off * K);
        return acc;
    } else {
        // The same pairing tree as the butterfly above, so the two paths agree bit for bit.
        __shared__ T sh[ROWS][TPR][K];
        sh[r][sub][c] = acc;
        __syncthreads();
        T tot = T(0);
        if (sub == 0) {
            T a[TPR];
#pragma unroll
            for (int q = 0; q < TPR; ++q) a[q] = sh[r][q][c];
#pragma unroll
            for (int off = TPR / 2; off > 0; off >>= 1)
#pragma unroll
                for (int q = 0; q < off; ++q) a[q] = a[q] + a[q + off];
            tot = a[0];
        }
        __syncthreads();
        return tot;
    }
}

template <typename T, int K, int TPR>
__device__ __forceinline__ T group_row_dot(const int* __restrict__ ptr, const int* __restrict__ col,
                                           const T* __restrict__ val, const T* __restrict__ x,
                                           const RowSlot<T, K, TPR>& s, bool valid) {
    return group_row_dot<T, K, TPR, Group<K, TPR>::kRows>(ptr, col, val, x, s.row, s.r, s.sub, s.c, valid);
}

// Reducing kernels tile the rows 64/TPR at a time so a block is always 64*K threads.
template <int TPR>
struct ReduceTile {
    static constexpr int kRows = kTileRows / TPR;
};

template <typename T, int K>
__global__ void __launch_bounds__(tile_threads<K>()) jz_kernel(int n, const T* __restrict__ dinv, const T* __restrict__ b,
                                                               T alpha0, T* __restrict__ x) {
    pdl_enter();
    const int row = blockIdx.x * kTileRows + threadIdx.x / K;
    const int c = threadIdx.x % K;
    if (row < n) x[static_cast<long>(row) * K + c] = alpha0 * dinv[row] * b[static_cast<long>(row) * K + c];
}

// out = c_cur*x_cur + c_prev*x_prev + alpha*dinv*(b - A x_cur). out may alias x_prev (read only
// at this row), never x_cur.
template <typename T, int K, int TPR>
__global__ void __launch_bounds__(Group<K, TPR>::kBlock) cheby_kernel(
    int n, const int* __restrict__ ptr, const int* __restrict__ col, const T* __restrict__ val,
    const T* __restrict__ dinv, const T* __restrict__ b, const T* __restrict__ x_cur, const T* x_prev, T c_cur,
    T c_prev, T alpha, T* out) {
    pdl_enter();
    const RowSlot<T, K, TPR> s;
    const bool valid = s.row < n;
    const T ax = group_row_dot<T, K, TPR>(ptr, col, val, x_cur, s, valid);
    if (!valid || s.sub != 0) return;
    const long q = static_cast<long>(s.row) * K + s.c;
    const T cur = x_cur[q];
    const T prev = x_prev[q];
    const T rhs = b[q];
    out[q] = c_cur * cur + c_prev * prev + alpha * dinv[s.row] * (rhs - ax);
}

template <typename T, int K, int TPR>
__global__ void __launch_bounds__(Group<K, TPR>::kBlock) residual_kernel(int n, const int* __restrict__ ptr,
                                                                         const int* __restrict__ col,
                                                                         const T* __restrict__ val,
                                                                         const T* __restrict__ x,
                                                                         const T* __restrict__ b, T* __restrict__ r) {
    pdl_enter();
    const RowSlot<T, K, TPR> s;
    const bool valid = s.row < n;
    const T ax = group_row_dot<T, K, TPR>(ptr, col, val, x, s, valid);
    if (!valid || s.sub != 0) return;
    const long q = static_cast<long>(s.row) * K + s.c;
    r[q] = b[q] - ax;
}

// b_c = R r_f; with dinv_c given, also the coarse level's first smoothing step x_c = alpha0*dinv*b_c.
template <typename T, int K, int TPR>
__global__ void __launch_bounds__(Group<K, TPR>::kBlock) restrict_kernel(int nc, const int* __restrict__ ptr,
                                                                         const int* __restrict__ col,
                                                                         const T* __restrict__ val,
                                                                         const T* __restrict__ rf, T* __restrict__ bc,
                                                                         const T* __restrict__ dinv_c, T alpha0,
                                                                         T* __restrict__ xc) {
    pdl_enter();
    const RowSlot<T, K, TPR> s;
    const bool valid = s.row < nc;
    const T v = group_row_dot<T, K, TPR>(ptr, col, val, rf, s, valid);
    if (!valid || s.sub != 0) return;
    const long q = static_cast<long>(s.row) * K + s.c;
    bc[q] = v;
    if (dinv_c != nullptr) xc[q] = alpha0 * dinv_c[s.row] * v;
}

template <typename T, int K, int TPR>
__global__ void __launch_bounds__(Group<K, TPR>::kBlock) prolong_kernel(int n, const int* __restrict__ ptr,
                                                                        const int* __restrict__ col,
                                                                        const T* __restrict__ val,
                                                                        const T* __restrict__ xc, T* __restrict__ xf) {
    pdl_enter();
    const RowSlot<T, K, TPR> s;
    const bool valid = s.row < n;
    const T v = group_row_dot<T, K, TPR>(ptr, col, val, xc, s, valid);
    if (!valid || s.sub != 0) return;
    xf[static_cast<long>(s.row) * K + s.c] += v;
}

// --- one lane per row and C adjacent columns (operators walked by one lane per row) -------------
//
// A lane takes C adjacent columns of its row (C = 2 or 4): one index and one value load per nonzero
// serve them all, and the gather is one 8- or 16-byte load (FP32; FP64 takes 16-byte pairs). A
// C-th of the lanes carry the same memory work, so each has C times the loads in flight at the same
// occupancy. Each column's terms are added in CSR order exactly as by strided_dot<T, 1> (one fused
// multiply-add per term), so the results are bitwise those of the one-column kernels.
template <typename T, int C>
struct ColGroup;
template <>
struct ColGroup<float, 2> {
    using V = float2;
    __device__ static void split(const V& v, float* o) { o[0] = v.x; o[1] = v.y; }
};
template <>
struct ColGroup<float, 4> {
    using V = float4;
    __device__ static void split(const V& v, float* o) { o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w; }
};
template <>
struct ColGroup<double, 2> {
    using V = double2;
    __device__ static void split(const V& v, double* o) { o[0] = v.x; o[1] = v.y; }
};

constexpr int kColBlock = 256;

template <int K, int C>
struct ColLanes {
    static constexpr int kLanes = K / C;                // lanes per row
    static constexpr int kRows = kColBlock / kLanes;    // rows per block
};

template <int K, int C>
unsigned col_grid(int n) {
    return static_cast<unsigned>((n + ColLanes<K, C>::kRows - 1) / ColLanes<K, C>::kRows);
}

// The C columns' gathers of row j: x[j * K + g * C + 0 .. C-1].
template <typename T, int K, int C>
__device__ __forceinline__ void gather_cols(const T* __restrict__ x, long j, int g, T out[C]) {
    if constexpr (std::is_same<T, double>::value && C == 4) {
        const double2* xv = reinterpret_cast<const double2*>(x + j * K + g * C);
        const double2 a = xv[0], b = xv[1];
        out[0] = a.x;
        out[1] = a.y;
        out[2] = b.x;
        out[3] = b.y;
    } else {
        using G = ColGroup<T, C>;
        G::split(reinterpret_cast<const typename G::V*>(x)[j * (K / C) + g], out);
    }
}

template <typename T, int K, int C>
__device__ __forceinline__ void row_dot_cols(const int* __restrict__ ptr, const int* __restrict__ col,
                                             const T* __restrict__ val, const T* __restrict__ x, int row, int g,
                                             T acc[C]) {
#pragma unroll
    for (int u = 0; u < C; ++u) acc[u] = T(0);
    const int e = ptr[row + 1];
    for (int p = ptr[row]; p < e; ++p) {
        const int j = col[p];
        const T v = val[p];
        T xx[C];
        gather_cols<T, K, C>(x, j, g, xx);
#pragma unroll
        for (int u = 0; u < C; ++u) acc[u] += v * xx[u];
    }
}

template <typename T, int K, int C>
__global__ void __launch_bounds__(kColBlock) cheby_cols_kernel(int n, const int* __restrict__ ptr,
                                                               const int* __restrict__ col, const T* __restrict__ val,
                                                               const T* __restrict__ dinv, const T* __restrict__ b,
                                                               const T* __restrict__ x_cur, const T* x_prev, T c_cur,
                                                               T c_prev, T alpha, T* out) {
    pdl_enter();
    const int row = blockIdx.x * ColLanes<K, C>::kRows + threadIdx.x / ColLanes<K, C>::kLanes;
    const int g = threadIdx.x % ColLanes<K, C>::kLanes;
    if (row >= n) return;
    T ax[C];
    row_dot_cols<T, K, C>(ptr, col, val, x_cur, row, g, ax);
    const long q = static_cast<long>(row) * K + g * C;
    const T d = dinv[row];
#pragma unroll
    for (int u = 0; u < C; ++u) {
        const T cur = x_cur[q + u];
        const T prev = x_prev[q + u];
        const T rhs = b[q + u];
        out[q + u] = c_cur * cur + c_prev * prev + alpha * d * (rhs - ax[u]);
    }
}

template <typename T, int K, int C>
__global__ void __launch_bounds__(kColBlock) residual_cols_kernel(int n, const int* __restrict__ ptr,
                                                                  const int* __restrict__ col,
                                                                  const T* __restrict__ val, const T* __restrict__ x,
                                                                  const T* __restrict__ b, T* __restrict__ r) {
    pdl_enter();
    const int row = blockIdx.x * ColLanes<K, C>::kRows + threadIdx.x / ColLanes<K, C>::kLanes;
    const int g = threadIdx.x % ColLanes<K, C>::kLanes;
    if (row >= n) return;
    T ax[C];
    row_dot_cols<T, K, C>(ptr, col, val, x, row, g, ax);
    const long q = static_cast<long>(row) * K + g * C;
#pragma unroll
    for (int u = 0; u < C; ++u) r[q + u] = b[q + u] - ax[u];
}

template <typename T, int K, int C>
__global__ void __launch_bounds__(kColBlock) prolong_cols_kernel(int n, const int* __restrict__ ptr,
                                                                 const int* __restrict__ col,
                                                                 const T* __restrict__ val, const T* __restrict__ xc,
                                                                 T* __restrict__ xf) {
    pdl_enter();
    const int row = blockIdx.x * ColLanes<K, C>::kRows + threadIdx.x / ColLanes<K, C>::kLanes;
    const int g = threadIdx.x % ColLanes<K, C>::kLanes;
    if (row >= n) return;
    T v[C];
    row_dot_cols<T, K, C>(ptr, col, val, xc, row, g, v);
    const long q = static_cast<long>(row) * K + g * C;
#pragma unroll
    for (int u = 0; u < C; ++u) xf[q + u] += v[u];
}

// The same for operators walked by TPR sub-lanes per row (coarse levels, long rows), when a row's
// TPR x K/C threads fit in one warp: each sub-lane takes its strided share of the row eight entries
// at a time (index and value loads, then the gathers, then the multiply-adds in order, as
// strided_dot<T, TPR>), and the shares are combined by the XOR butterfly of group_row_dot: the same
// pairing tree per column, so the sums are bitwise those of the one-column kernels.
template <int K, int TPR, int C>
struct SubColLanes {
    static constexpr int kLanes = K / C;                     // column groups per row
    static constexpr int kThreads = TPR * kLanes;            // threads per row (<= 32)
    static constexpr int kRows = kColBlock / kThreads;       // rows per block
};

template <int K, int TPR, int C>
unsigned subcol_grid(int n) {
    return static_cast<unsigned>((n + SubColLanes<K, TPR, C>::kRows - 1) / SubColLanes<K, TPR, C>::kRows);
}

template <typename T, int K, int TPR, int C>
__device__ __forceinline__ void sub_row_dot_cols(const int* __restrict__ ptr, const int* __restrict__ col,
                                                 const T* __restrict__ val, const T* __restrict__ x, int row,
                                                 bool valid, int sub, int g, T acc[C]) {
    constexpr int B = 8;
#pragma unroll
    for (int u = 0; u < C; ++u) acc[u] = T(0);
    if (valid) {
        const int e = ptr[row + 1];
        for (int p = ptr[row] + sub; p < e; p += B * TPR) {
            int cj[B];
            T vj[B];
#pragma unroll
            for (int j = 0; j < B; ++j) {
                const int q = p + j * TPR;
                const bool ok = q < e;
                cj[j] = ok ? col[q] : 0;
                vj[j] = ok ? val[q] : T(0);
            }
            T xj[B][C];
#pragma unroll
            for (int j = 0; j < B; ++j) {
                if (p + j * TPR < e) {
                    gather_cols<T, K, C>(x, cj[j], g, xj[j]);
                } else {
#pragma unroll
                    for (int u = 0; u < C; ++u) xj[j][u] = T(0);
                }
            }
#pragma unroll
            for (int j = 0; j < B; ++j)
                if (p + j * TPR < e) {
#pragma unroll
                    for (int u = 0; u < C; ++u) acc[u] += vj[j] * xj[j][u];
                }
        }
    }
#pragma unroll
    for (int off = TPR / 2; off > 0; off >>= 1)
#pragma unroll
        for (int u = 0; u < C; ++u) acc[u] += __shfl_xor_sync(0xffffffffu, acc[u], off * (K / C));
}

template <typename T, int K, int TPR, int C>
struct SubColSlot {
    int row, sub, g;
    __device__ __forceinline__ SubColSlot() {
        using S = SubColLanes<K, TPR, C>;
        const int t = threadIdx.x;
        row = blockIdx.x * S::kRows + t / S::kThreads;
        sub = (t / S::kLanes) % TPR;
        g = t % S::kLanes;
    }
};

template <typename T, int K, int TPR, int C>
__global__ void __launch_bounds__(kColBlock) cheby_subcols_kernel(int n, const int* __restrict__ ptr,
                                                                  const int* __restrict__ col,
                                                                  const T* __restrict__ val,
                                                                  const T* __restrict__ dinv, const T* __restrict__ b,
                                                                  const T* __restrict__ x_cur, const T* x_prev,
                                                                  T c_cur, T c_prev, T alpha, T* out) {
    pdl_enter();
    const SubColSlot<T, K, TPR, C> s;
    const bool valid = s.row < n;
    T ax[C];
    sub_row_dot_cols<T, K, TPR, C>(ptr, col, val, x_cur, s.row, valid, s.sub, s.g, ax);
    if (!valid || s.sub != 0) return;
    const long q = static_cast<long>(s.row) * K + s.g * C;
    const T d = dinv[s.row];
#pragma unroll
    for (int u = 0; u < C; ++u) {
        const T cur = x_cur[q + u];
        const T prev = x_prev[q + u];
        const T rhs = b[q + u];
        out[q + u] = c_cur * cur + c_prev * prev + alpha * d * (rhs - ax[u]);
    }
}

template <typename T, int K, int TPR, int C>
__global__ void __launch_bounds__(kColBlock) residual_subcols_kernel(int n, const int* __restrict__ ptr,
                                                                     const int* __restrict__ col,
                                                                     const T* __restrict__ val,
                                                                     const T* __restrict__ x, const T* __restrict__ b,
                                                                     T* __restrict__ r) {
    pdl_enter();
    const SubColSlot<T, K, TPR, C> s;
    const bool valid = s.row < n;
    T ax[C];
    sub_row_dot_cols<T, K, TPR, C>(ptr, col, val, x, s.row, valid, s.sub, s.g, ax);
    if (!valid || s.sub != 0) return;
    const long q = static_cast<long>(s.row) * K + s.g * C;
#pragma unroll
    for (int u = 0; u < C; ++u) r[q + u] = b[q + u] - ax[u];
}

template <typename T, int K, int TPR, int C>
__global__ void __launch_bounds__(kColBlock) restrict_subcols_kernel(int nc, const int* __restrict__ ptr,
                                                                     const int* __restrict__ col,
                                                                     const T* __restrict__ val,
                                                                     const T* __restrict__ rf, T* __restrict__ bc,
                                                                     const T* __restrict__ dinv_c, T alpha0,
                                                                     T* __restrict__ xc) {
    pdl_enter();
    const SubColSlot<T, K, TPR, C> s;
    const bool valid = s.row < nc;
    T v[C];
    sub_row_dot_cols<T, K, TPR, C>(ptr, col, val, rf, s.row, valid, s.sub, s.g, v);
    if (!valid || s.sub != 0) return;
    const long q = static_cast<long>(s.row) * K + s.g * C;
#pragma unroll
    for (int u = 0; u < C; ++u) {
        bc[q + u] = v[u];
        if (dinv_c != nullptr) xc[q + u] = alpha0 * dinv_c[s.row] * v[u];
    }
}

template <typename T, int K, int TPR, int C>
__global__ void __launch_bounds__(kColBlock) prolong_subcols_kernel(int n, const int* __restrict__ ptr,
                                                                    const int* __restrict__ col,
                                                                    const T* __restrict__ val,
                                                                    const T* __restrict__ xc, T* __restrict__ xf) {
    pdl_enter();
    const SubColSlot<T, K, TPR, C> s;
    const bool valid = s.row < n;
    T v[C];
    sub_row_dot_cols<T, K, TPR, C>(ptr, col, val, xc, s.row, valid, s.sub, s.g, v);
    if (!valid || s.sub != 0) return;
    const long q = static_cast<long>(s.row) * K + s.g * C;
#pragma unroll
    for (int u = 0; u < C; ++u) xf[q + u] += v[u];
}

// Calls f(std::integral_constant<int, C>) with the widest lane width C <= lane_cols that divides K
// (C > 1), and returns whether it did.
template <int K, typename F>
bool dispatch_cols(int lane_cols, F&& f) {
    if constexpr (K % 4 == 0) {
        if (lane_cols >= 4) {
            f(std::integral_constant<int, 4>{});
            return true;
        }
    }
    if constexpr (K % 2 == 0) {
        if (lane_cols >= 2) {
            f(std::integral_constant<int, 2>{});
            return true;
        }
    }
    return false;
}

// Calls f(std::integral_constant<int, TPR>, std::integral_constant<int, 2>) when an operator walked by
// tpr > 1 sub-lanes takes column pairs (lane_cols >= 2, K even, a row's threads within one warp),
// and returns whether it did.
template <int K, typename F>
bool dispatch_subcols(int tpr, int lane_cols, F&& f) {
    if constexpr (K % 2 == 0) {
        if (lane_cols < 2) return false;
        constexpr int L = K / 2;
        auto go = [&](auto tc) {
            constexpr int TPR = decltype(tc)::value;
            if constexpr (TPR * L <= 32) {
                f(tc, std::integral_constant<int, 2>{});
                return true;
            } else {
                return false;
            }
        };
        switch (tpr) {
            case 2: return go(std::integral_constant<int, 2>{});
            case 4: return go(std::integral_constant<int, 4>{});
            case 8: return go(std::integral_constant<int, 8>{});
            case 16: return go(std::integral_constant<int, 16>{});
            case 32: return go(std::integral_constant<int, 32>{});
            default: return false;
        }
    } else {
        (void)tpr;
        (void)lane_cols;
        (void)f;
        return false;
    }
}

template <int K, typename F>
void dispatch_tpr(int tpr, F&& f) {
    switch (tpr) {
        case 1: f(std::integral_constant<int, 1>{}); break;
        case 2: f(std::integral_constant<int, 2>{}); break;
        case 4: f(std::integral_constant<int, 4>{}); break;
        case 8: f(std::integral_constant<int, 8>{}); break;
        case 16: f(std::integral_constant<int, 16>{}); break;
        case 32: f(std::integral_constant<int, 32>{}); break;
        default: fail(kEInternal, "threads-per-row must be a power of two up to 32");
    }
}

// A solve-loop kernel launch, with programmatic stream serialization when `dep` is set (the
// kernel then starts with pdl_enter()); a plain launch otherwise.
template <typename... KArgs, typename... Args>
void launch_loop(bool dep, void (*kernel)(KArgs...), dim3 grid, unsigned block, cudaStream_t s, Args... args) {
    if (!dep) {
        kernel<<<grid, block, 0, s>>>(args...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CUNIBS_CHECK(cudaLaunchKernelEx(&cfg, kernel, args...));
}

template <int K, int TPR>
unsigned group_grid(int n) {
    return static_cast<unsigned>((n + Group<K, TPR>::kRows - 1) / Group<K, TPR>::kRows);
}

// x = inv b for the dense bottom of the V-cycle (n rows of ld entries, zero past column n). inv is
// symmetric, so x_i = sum_j inv[j][i] b_j: a lane owns V consecutive outputs i and walks rows j of
// inv, every warp load 512 contiguous bytes of one row, with no reduction across lanes. Pass 1: the
// grid is about one block per SM (DenseGrid): block (I, S) owns the outputs of column block I and
// the rows j of split S, and streams them once. Each thread copies its own 16 bytes of each row
// into a private ring of shared-memory slots with asynchronous copies (cp.async, kDenseRing stages
// of kDenseRows rows ahead), so the bytes in flight do not take registers, and a thread only ever
// waits for its own copies (cp.async.wait_group: no barrier, no spinning). b's rows of the split are
// staged once in shared memory and read as broadcasts. Pass 2 adds the splits' partials in order.
// Every (output, column of b) sum runs over the same terms in the same order whatever K is (the
// grid depends on n, the type and the GPU only), so a column's result does not depend on the block
// width.
constexpr int kDenseMaxThreads = 512;
constexpr int kDenseRows = 8;
constexpr std::size_t kDenseSmemBudget = 220 * 1024;

template <typename T>
struct DenseGrid {
    static constexpr int V = 16 / static_cast<int>(sizeof(T));  // outputs per lane (one 16-byte load)
    static constexpr int kRing = sizeof(T) == 8 ? 2 : 3;         // stages in flight
    int col_blocks = 1, cols = 0, threads = 0, splits = 1, split_rows = 0;
    std::size_t ring_bytes = 0, b_bytes = 0;
    DenseGrid(int n, int K, int sm_count) {
        const int ld = dense_ld(n);
        col_blocks = (ld + kDenseMaxThreads * V - 1) / (kDenseMaxThreads * V);
        const int span = kWarp * V;
        cols = ((ld + col_blocks - 1) / col_blocks + span - 1) / span * span;
        threads = cols / V;
        ring_bytes = static_cast<std::size_t>(kRing) * kDenseRows * threads * 16;
        splits = std::max(1, std::min(sm_count / col_blocks, (n + 15) / 16));
        // b's rows of a split share the block's shared memory with the ring; the splits are sized
        // for the widest block (16 columns) so that they never depend on K.
        const std::size_t widest = 16 * sizeof(T);
        const std::size_t room = kDenseSmemBudget - ring_bytes;
        splits = std::max<int>(splits, static_cast<int>((static_cast<std::size_t>(n) * widest + room - 1) / room));
        split_rows = (n + splits - 1) / splits;
        b_bytes = static_cast<std::size_t>(split_rows) * K * sizeof(T);
    }
    std::size_t smem() const { return ring_bytes + b_bytes; }
};

// The inverse streams past L2 marked evict-first, so that it does not push the finest level's
// operator and vectors (which stay L2-resident from one PCG iteration to the next) out of L2.
__device__ __forceinline__ std::uint64_t evict_first_policy() {
    std::uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, std::uint64_t policy) {
    const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(dst), "l"(gmem), "l"(policy)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <typename T>
__device__ __forceinline__ void load16(const T* p, T* o);
template <>
__device__ __forceinline__ void load16<float>(const float* p, float* o) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
}
template <>
__device__ __forceinline__ void load16<double>(const double* p, double* o) {
    const double2 v = *reinterpret_cast<const double2*>(p);
    o[0] = v.x;
    o[1] = v.y;
}

// A lane's V outputs += a (its V entries of one row of inv) * b_j, for each of b's K columns. FP32 pairs
// the outputs for packed FMAs (FFMA2, each lane an fmaf rounded once: the same sums as scalar).
template <typename T, int K>
struct DenseAcc {
    static constexpr int V = DenseGrid<T>::V;
    T v[V][K];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int u = 0; u < V; ++u)
#pragma unroll
            for (int c = 0; c < K; ++c) v[u][c] = T(0);
    }
    __device__ __forceinline__ void add(const T* a, const T* bj) {
#pragma unroll
        for (int c = 0; c < K; ++c)
#pragma unroll
            for (int u = 0; u < V; ++u) v[u][c] = fma(a[u], bj[c], v[u][c]);
    }
    __device__ __forceinline__ T get(int u, int c) const { return v[u][c]; }
};
template <int K>
struct DenseAcc<float, K> {
    float2 v[2][K];  // outputs (0, 1) and (2, 3)
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int c = 0; c < K; ++c) v[h][c] = make_float2(0.0f, 0.0f);
    }
    __device__ __forceinline__ void add(const float* a, const float* bj) {
        const float2 a01 = make_float2(a[0], a[1]), a23 = make_float2(a[2], a[3]);
#pragma unroll
        for (int c = 0; c < K; ++c) {
            const float2 bb = make_float2(bj[c], bj[c]);
            v[0][c] = __ffma2_rn(a01, bb, v[0][c]);
            v[1][c] = __ffma2_rn(a23, bb, v[1][c]);
        }
    }
    __device__ __forceinline__ float get(int u, int c) const {
        const float2 p = v[u >> 1][c];
        return (u & 1) ? p.y : p.x;
    }
};

template <typename T, int K>
__global__ void __launch_bounds__(kDenseMaxThreads) dense_part_kernel(int n, int ld, int cols, int split_rows,
                                                                      const T* __restrict__ inv,
                                                                      const T* __restrict__ b,
                                                                      T* __restrict__ part) {
    pdl_enter();
    constexpr int V = DenseGrid<T>::V, R = DenseGrid<T>::kRing, U = kDenseRows;
    extern __shared__ __align__(16) unsigned char dense_smem[];
    // Ring slot (stage, row t) of thread x: 16 bytes at ((stage * U + t) * blockDim.x + x) * 16.
    uint4* ring = reinterpret_cast<uint4*>(dense_smem);
    T* bs = reinterpret_cast<T*>(dense_smem + static_cast<std::size_t>(R) * U * blockDim.x * 16);
    const int j0 = blockIdx.y * split_rows;
    const int j1 = min(n, j0 + split_rows);
    for (int q = threadIdx.x; q < (j1 - j0) * K; q += blockDim.x) bs[q] = b[static_cast<long>(j0) * K + q];
    __syncthreads();
    const int i0 = blockIdx.x * cols + threadIdx.x * V;
    if (i0 >= ld) return;
    const T* src = inv + static_cast<long>(j0) * ld + i0;  // this thread's 16 bytes of row j0
    uint4* mine = ring + threadIdx.x;
    const int stride = blockDim.x;  // slots from one row of a stage to the next
    const std::uint64_t policy = evict_first_policy();
    const int stages = (j1 - j0 + U - 1) / U;
    // Stage st holds rows j0 + st U + t (t < U); slots of rows past j1 are neither filled nor read.
    auto issue = [&](int st) {
        if (st < stages) {
            const T* s = src + static_cast<long>(st) * U * ld;
            uint4* d = mine + (st % R) * U * stride;
            const int left = j1 - j0 - st * U;
#pragma unroll
            for (int t = 0; t < U; ++t)
                if (t < left) cp_async16(d + t * stride, s + static_cast<long>(t) * ld, policy);
        }
        cp_async_commit();  // an empty group past the last stage keeps the group count uniform
    };
#pragma unroll
    for (int st = 0; st < R; ++st) issue(st);
    DenseAcc<T, K> acc;
    acc.zero();
    for (int st = 0; st < stages; ++st) {
        cp_async_wait<R - 1>();  // this thread's copies of stage st have landed
        const int rows = min(U, j1 - j0 - st * U);
        const uint4* d = mine + (st % R) * U * stride;
        const T* bj = bs + st * U * K;
#pragma unroll
        for (int t = 0; t < U; ++t) {
            if (t < rows) {
                T a[V];
                load16<T>(reinterpret_cast<const T*>(d + t * stride), a);
                acc.add(a, bj + t * K);
            }
        }
        issue(st + R);  // into the slots just read (this thread's own)
    }
    cp_async_wait<0>();
    T* out = part + (static_cast<long>(blockIdx.y) * n + i0) * K;
#pragma unroll
    for (int u = 0; u < V; ++u)
        if (i0 + u < n)
#pragma unroll
            for (int c = 0; c < K; ++c) out[u * K + c] = acc.get(u, c);
}

template <typename T, int K>
__global__ void __launch_bounds__(kBlock) dense_sum_kernel(int n, int blocks, const T* __restrict__ part,
                                                          T* __restrict__ x) {
    pdl_enter();
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long nk = static_cast<long>(n) * K;
    if (q >= nk) return;
    T v = part[q];
    for (int J = 1; J < blocks; ++J) v += part[J * nk + q];
    x[q] = v;
}

// --- PCG kernels -------------------------------------------------------------------------
//
// Column reductions run over a grid of at most kMaxReduceBlocks blocks that stride the 64-row
// tiles; each thread keeps a running sum of its rows, a block combines its 64 row slots by a fixed
// tree, and the last block to finish adds the block partials by a fixed tree. The grid size is a
// function of n alone, so every column is summed in the same order whatever the block width.

constexpr int kMaxReduceBlocks = 592;

// Per-block partial of each column into partials[c * gridDim.x + blockIdx.x].
template <int K>
__device__ __forceinline__ void block_partial(double v, double* __restrict__ partials) {
    __shared__ double sh[kTileRows][K];
    const int slot = threadIdx.x / K;
    const int c = threadIdx.x % K;
    sh[slot][c] = v;
    __syncthreads();
#pragma unroll
    for (int off = kTileRows / 2; off > 0; off >>= 1) {
        if (slot < off) sh[slot][c] += sh[slot + off][c];
        __syncthreads();
    }
    if (threadIdx.x < K) {
        partials[static_cast<long>(threadIdx.x) * gridDim.x + blockIdx.x] = sh[0][threadIdx.x];
        __threadfence();
    }
}

// ||x_c||^2 per column into out[c].
template <typename T, int K>
__global__ void __launch_bounds__(tile_threads<K>()) norm2_kernel(int n, const T* __restrict__ x, double* partials,
                                                                  unsigned* counter, double* __restrict__ out) {
    const int slot = threadIdx.x / K;
    const int c = threadIdx.x % K;
    const int tiles = n_tiles_dev(n);
    double v = 0.0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int row = t * kTileRows + slot;
        if (row < n) {
            const double xv = static_cast<double>(x[static_cast<long>(row) * K + c]);
            v += xv * xv;
        }
    }
    block_partial<K>(v, partials);
    if (last_block(counter)) {
        __shared__ double tot[K];
        final_reduce<K>(partials, gridDim.x, tot);
        if (threadIdx.x < K) out[threadIdx.x] = tot[threadIdx.x];
    }
}

// The search direction and its product, fused: p = z + beta p and Ap = A z + beta Ap (the product
// carried by its recurrence, so the SpMV gathers the V-cycle's output z, FP32 under an FP32
// V-cycle, instead of the FP64 direction), then pAp per column and alpha = rz / pAp. Columns frozen
// before this iteration keep p and Ap; alpha is 0 on every frozen column.
template <typename T, typename TZ, int K, int TPR>
__global__ void __launch_bounds__(tile_threads<K>()) spmv_alpha_kernel(
    int n, const int* __restrict__ ptr, const int* __restrict__ col, const T* __restrict__ val,
    const TZ* __restrict__ z, T* __restrict__ p, T* __restrict__ ap, double* partials, unsigned* counter,
    const double* __restrict__ rz, const double* __restrict__ beta, const int* __restrict__ frozen,
    double* __restrict__ alpha) {
    pdl_enter();
    constexpr int ROWS = ReduceTile<TPR>::kRows;
    const int r = threadIdx.x / (TPR * K);
    const int sub = (threadIdx.x / K) % TPR;
    const int c = threadIdx.x % K;
    const int tiles = (n + ROWS - 1) / ROWS;
    const bool update = frozen[c] != 1;
    const T b = static_cast<T>(beta[c]);
    double v = 0.0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int row = t * ROWS + r;
        const bool valid = row < n;
        const T s = group_row_dot<T, K, TPR, ROWS, TZ>(ptr, col, val, z, row, r, sub, c, valid);
        if (valid && sub == 0) {
            const long q = static_cast<long>(row) * K + c;
            T pq = p[q], aq = ap[q];
            if (update) {
                pq = static_cast<T>(z[q]) + b * pq;
                aq = s + b * aq;
                p[q] = pq;
                ap[q] = aq;
            }
            v += static_cast<double>(pq) * static_cast<double>(aq);
        }
    }
    block_partial<K>(v, partials);
    if (last_block(counter)) {
        __shared__ double tot[K];
        final_reduce<K>(partials, gridDim.x, tot);
        if (threadIdx.x < K) {
            const int cc = threadIdx.x;
            alpha[cc] = frozen[cc] ? 0.0 : rz[cc] / tot[cc];
        }
    }
}

// x += alpha p; r -= alpha Ap; rr = ||r||^2. A column freezes when sqrt(rr) <= tol_c*sqrt(ref[c])
// (tol_c = tol_vec[c] when given, else tol); the iteration it froze at and its relative residual
// are recorded on the device. With z0 given, also writes the V-cycle's first smoothing step
// z0 = alpha0*dinv*r from the new residual.
// With a V-cycle in a narrower type TZ than the Krylov vectors (FP64 PCG over an FP32 V-cycle),
// r_lo receives the residual rounded to TZ, the V-cycle's input, and z0 is formed from it.
template <typename T, typename TZ, int K>
__global__ void __launch_bounds__(tile_threads<K>()) update_xr_kernel(
    int n, const double* __restrict__ alpha, const T* __restrict__ p, const T* __restrict__ ap, T* __restrict__ x,
    T* __restrict__ r, double* partials, unsigned* counter, const double* __restrict__ ref, double tol,
    const double* __restrict__ tol_vec, int* __restrict__ frozen, int* __restrict__ iter_counter,
    int* __restrict__ conv_iter, double* __restrict__ rel_out, int record, const TZ* __restrict__ dinv, TZ alpha0,
    TZ* __restrict__ z0, TZ* __restrict__ r_lo, cudaGraphConditionalHandle loop, int use_loop,
    const int* __restrict__ cap) {
    pdl_enter();
    const int slot = threadIdx.x / K;
    const int c = threadIdx.x % K;
    const int tiles = n_tiles_dev(n);
    const T a = static_cast<T>(alpha[c]);
    double v = 0.0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int row = t * kTileRows + slot;
        if (row < n) {
            const long q = static_cast<long>(row) * K + c;
            x[q] += a * p[q];
            const T rn = r[q] - a * ap[q];
            r[q] = rn;
            const TZ rl = static_cast<TZ>(rn);
            if (r_lo != nullptr) r_lo[q] = rl;
            if (z0 != nullptr) z0[q] = alpha0 * dinv[row] * rl;
            v += static_cast<double>(rn) * static_cast<double>(rn);
        }
    }
    block_partial<K>(v, partials);
    if (last_block(counter)) {
        __shared__ double tot[K];
        final_reduce<K>(partials, gridDim.x, tot);
        const int it = *iter_counter + 1;
        if (threadIdx.x < K) {
            const int cc = threadIdx.x;
            const double rel = sqrt(tot[cc]) / sqrt(ref[cc]);
            const double tc = tol_vec ? tol_vec[cc] : tol;
            // frozen: 0 running, 2 met its target this iteration (its direction update still runs,
            // so the sequence can resume after a residual replacement), 1 frozen before.
            if (frozen[cc] == 2) frozen[cc] = 1;
            if (!frozen[cc]) {
                if (record) rel_out[cc] = rel;
                if (rel <= tc) {
                    frozen[cc] = 2;
                    if (record) conv_iter[cc] = it;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            *iter_counter = it;
            // Inside a device-side WHILE graph: run another iteration unless every column has
            // frozen or the iteration budget is spent.
            if (use_loop) {
                bool all = true;
                for (int cc = 0; cc < K; ++cc) all = all && frozen[cc];
                cudaGraphSetConditional(loop, (!all && it < *cap) ? 1u : 0u);
            }
        }
    }
}

// Finishes the beta update in the last block: rz_new = sum; beta = rz_new / rz. A column frozen
// before this iteration (frozen == 1) keeps its rz and gets beta = 0 (its direction is not touched).
template <int K>
__device__ __forceinline__ void finish_beta(double* partials, double* rz, const int* frozen, double* beta) {
    __shared__ double tot[K];
    final_reduce<K>(partials, gridDim.x, tot);
    if (threadIdx.x < K) {
        const int cc = threadIdx.x;
        if (frozen[cc] == 1) {
            beta[cc] = 0.0;
        } else {
            beta[cc] = tot[cc] / rz[cc];
            rz[cc] = tot[cc];
        }
    }
}

// rz_new = r . z; beta = rz_new / rz (0 on a frozen column); rz = rz_new.
template <typename T, int K>
__global__ void __launch_bounds__(tile_threads<K>()) dot_beta_kernel(int n, const T* __restrict__ r,
                                                                     const T* __restrict__ z, double* partials,
                                                                     unsigned* counter, double* __restrict__ rz,
                                                                     const int* __restrict__ frozen,
                                                                     double* __restrict__ beta) {
    pdl_enter();
    const int slot = threadIdx.x / K;
    const int c = threadIdx.x % K;
    const int tiles = n_tiles_dev(n);
    double v = 0.0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int row = t * kTileRows + slot;
        if (row < n) {
            const long q = static_cast<long>(row) * K + c;
            v += static_cast<double>(r[q]) * static_cast<double>(z[q]);
        }
    }
    block_partial<K>(v, partials);
    if (last_block(counter)) finish_beta<K>(partials, rz, frozen, beta);
}

// The V-cycle's last Chebyshev step on the finest level fused with r . z:
// z = c_cur*x_cur + c_prev*x_prev + alpha*dinv*(r - A x_cur), then beta as in dot_beta_kernel.
template <typename T, int K, int TPR>
__global__ void __launch_bounds__(tile_threads<K>()) cheby_dot_kernel(
    int n, const int* __restrict__ ptr, const int* __restrict__ col, const T* __restrict__ val,
    const T* __restrict__ dinv, const T* __restrict__ b, const T* __restrict__ x_cur, const T* __restrict__ x_prev,
    T c_cur, T c_prev, T alpha, T* __restrict__ z, double* partials, unsigned* counter, double* __restrict__ rz,
    const int* __restrict__ frozen, double* __restrict__ beta) {
    pdl_enter();
    constexpr int ROWS = ReduceTile<TPR>::kRows;
    const int r = threadIdx.x / (TPR * K);
    const int sub = (threadIdx.x / K) % TPR;
    const int c = threadIdx.x % K;
    const int tiles = (n + ROWS - 1) / ROWS;
    double v = 0.0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int row = t * ROWS + r;
        const bool valid = row < n;
        const T s = group_row_dot<T, K, TPR, ROWS>(ptr, col, val, x_cur, row, r, sub, c, valid);
        if (valid && sub == 0) {
            const long q = static_cast<long>(row) * K + c;
            const T rhs = b[q];
            const T out = c_cur * x_cur[q] + c_prev * x_prev[q] + alpha * dinv[row] * (rhs - s);
            z[q] = out;
            v += static_cast<double>(rhs) * static_cast<double>(out);
        }
    }
    block_partial<K>(v, partials);
    if (last_block(counter)) finish_beta<K>(partials, rz, frozen, beta);
}

// r_lo = r rounded to the V-cycle's type (the first V-cycle input of FP64 PCG over an FP32 V-cycle).
template <typename T, typename TZ>
__global__ void narrow_kernel(std::int64_t count, const T* __restrict__ r, TZ* __restrict__ r_lo) {
    const std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q < count) r_lo[q] = static_cast<TZ>(r[q]);
}

// Mixed refinement outer step: R = B - A X in FP64; r32 = (float)R; per column the true relative
// residual, the outer freeze, the inner solve's reference norm, its starting freeze, and the
// inner target: reduce the residual by eta = max(eta_min, 0.3 * tol / rel), just enough (with a
// margin) for the next outer step to meet tol.
template <int K, int TPR>
__global__ void __launch_bounds__(tile_threads<K>()) true_residual_kernel(
    int n, const int* __restrict__ ptr, const int* __restrict__ col, const double* __restrict__ val,
    const double* __restrict__ B, const double* __restrict__ X, float* __restrict__ r32, double* partials,
    unsigned* counter, const double* __restrict__ ref_sq, double tol, double eta_min, int* __restrict__ outer_conv,
    int* __restrict__ inner_frozen, double* __restrict__ rr0, double* __restrict__ eta,
    const int* __restrict__ iter_counter, int* __restrict__ conv_iter, double* __restrict__ rel_out) {
    constexpr int ROWS = ReduceTile<TPR>::kRows;
    const int r = threadIdx.x / (TPR * K);
    const int sub = (threadIdx.x / K) % TPR;
    const int c = threadIdx.x % K;
    const int tiles = (n + ROWS - 1) / ROWS;
    double v = 0.0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int row = t * ROWS + r;
        const bool valid = row < n;
        const double ax = group_row_dot<double, K, TPR, ROWS>(ptr, col, val, X, row, r, sub, c, valid);
        if (valid && sub == 0) {
            const long q = static_cast<long>(row) * K + c;
            const float rf = static_cast<float>(B[q] - ax);
            r32[q] = rf;
            v += static_cast<double>(rf) * static_cast<double>(rf);
        }
    }
    block_partial<K>(v, partials);
    if (last_block(counter)) {
        __shared__ double tot[K];
        final_reduce<K>(partials, gridDim.x, tot);
        if (threadIdx.x < K) {
            const int cc = threadIdx.x;
            const double rel = sqrt(tot[cc]) / sqrt(ref_sq[cc]);
            if (!outer_conv[cc]) {
                rel_out[cc] = rel;
                if (rel <= tol) {
                    outer_conv[cc] = 1;
                    conv_iter[cc] = *iter_counter;
                }
            }
            inner_frozen[cc] = outer_conv[cc];
            rr0[cc] = tot[cc];
            eta[cc] = fmax(eta_min, fmin(0.1, 0.3 * tol / rel));
        }
    }
}

// FP64 residual R = B - A X for a warm start of the plain solve.
template <int K, int TPR>
__global__ void __launch_bounds__(tile_threads<K>()) residual64_kernel(int n, const int* __restrict__ ptr,
                                                                       const int* __restrict__ col,
                                                                       const double* __restrict__ val,
                                                                       const double* __restrict__ B,
                                                                       const double* __restrict__ X,
                                                                       double* __restrict__ R) {
    constexpr int ROWS = ReduceTile<TPR>::kRows;
    const int r = threadIdx.x / (TPR * K);
    const int sub = (threadIdx.x / K) % TPR;
    const int c = threadIdx.x % K;
    const int row = blockIdx.x * ROWS + r;
    const bool valid = row < n;
    const double ax = group_row_dot<double, K, TPR, ROWS>(ptr, col, val, X, row, r, sub, c, valid);
    if (!valid || sub != 0) return;
    const long q = static_cast<long>(row) * K + c;
    R[q] = B[q] - ax;
}

// The zero-guess fallback of a warm start: a column whose guess leaves ||R|| >= ||B|| restarts from
// X = 0, R = B. init_rel[c] receives the kept guess's relative residual (1 when dropped).
template <int K>
__global__ void __launch_bounds__(tile_threads<K>()) guess_fallback_kernel(int n, double* __restrict__ X,
                                                                           double* __restrict__ R,
                                                                           const double* __restrict__ B,
                                                                           const double* __restrict__ ref_sq,
                                                                           const double* __restrict__ r0sq,
                                                                           double* __restrict__ init_rel) {
    const int row = blockIdx.x * kTileRows + threadIdx.x / K;
    const int c = threadIdx.x % K;
    const bool keep = r0sq[c] < ref_sq[c];
    if (blockIdx.x == 0 && threadIdx.x < K) init_rel[c] = keep ? sqrt(r0sq[c] / ref_sq[c]) : 1.0;
    if (row >= n || keep) return;
    const long q = static_cast<long>(row) * K + c;
    X[q] = 0.0;
    R[q] = B[q];
}

template <int K>
__global__ void __launch_bounds__(tile_threads<K>()) add_correction_kernel(int n, double* __restrict__ X,
                                                                           const float* __restrict__ d) {
    const int row = blockIdx.x * kTileRows + threadIdx.x / K;
    const int c = threadIdx.x % K;
    if (row >= n) return;
    const long q = static_cast<long>(row) * K + c;
    X[q] += static_cast<double>(d[q]);
}

int reduce_grid(int n) { return std::min(n_tiles(n), kMaxReduceBlocks); }
template <int TPR>
int reduce_grid_rows(int n) {
    return std::min((n + ReduceTile<TPR>::kRows - 1) / ReduceTile<TPR>::kRows, kMaxReduceBlocks);
}

}  // namespace

// Per-precision V-cycle workspace.
template <typename T>
struct VWork {
    std::vector<DevArray<T>> x, r, b;
    DevArray<T> cb, cx;
    DevArray<T> part;  // the dense bottom's per-column-block partial sums
};

class Solver {
  public:
    const Hierarchy* h = nullptr;
    int n = 0;
    int kcap = 0;
    // Solve-loop kernels launched with programmatic stream serialization (pdl_enter): off by default,
    // on with CUNIBS_PROGRAMMATIC_LAUNCH=1. With the V-cycle's bottom at level 1 the loop is mostly
    // multi-wave finest-level kernels, whose early-resident successors take their later waves'
    // slots: split solve 3.38 ms per block of 8 with it, 3.26 ms without.
    bool pdl = false;
    // Columns per lane of the one-lane-per-row operators (the *_cols kernels; bitwise the same
    // results): 2 by default, CUNIBS_LANE_COLUMNS=1 or 4 to choose.
    int lane_cols = 2;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    // FP64 CG / outer workspace (n, kcap)
    DevArray<double> B, X, R, P, AP, Z;
    // FP32 inner workspace
    DevArray<float> d32, r32, p32, ap32, z32;
    VWork<float> v32;
    VWork<double> v64;
    // Per-column scalars.
    DevArray<double> rz, alpha, beta, ref_sq, rr0, rel, eta, partials, r0sq, init_rel;
    // The call's tolerance per column, written before every solve: the cached loop graphs read it
    // from here, so a call with another tolerance than the one the graph was captured under still
    // stops at its own.
    DevArray<double> tolv;
    DevArray<int> frozen, outer_conv, conv_iter, iter_counter;
    DevArray<unsigned> counter;
    int* h_flags = nullptr;   // pinned
    double* h_dbl = nullptr;  // pinned
    // Deferred readbacks of the last solve_plain: h_dbl[2K..3K) holds the right-hand side norms
    // (check_ref), h_flags[2K] the device loop's iteration count (st.iterations == -1).
    bool check_ref = false;
    long long loop_nodes = 0;
    std::map<std::tuple<int, int, int>, std::pair<cudaGraphExec_t, long long>> graphs;

    ~Solver() {
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second.first);
        if (h_flags) cudaFreeHost(h_flags);
        if (h_dbl) cudaFreeHost(h_dbl);
        if (stream) cudaStreamDestroy(stream);
    }

    void ensure(int K) {
        if (kcap >= K) return;
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second.first);
        graphs.clear();
        const std::size_t nk = static_cast<std::size_t>(n) * K;
        for (auto* a : {&B, &X, &R, &P, &AP, &Z}) a->resize(nk);
        for (auto* a : {&d32, &r32, &p32, &ap32, &z32}) a->resize(nk);
        const std::size_t L = h->levels.size();
        v32.x.resize(L);
        v32.r.resize(L);
        v32.b.resize(L);
        v64.x.resize(L);
        v64.r.resize(L);
        v64.b.resize(L);
        for (std::size_t l = 0; l < L; ++l) {
            const std::size_t m = static_cast<std::size_t>(h->levels[l].n) * K;
            v32.x[l].resize(m);
            v32.r[l].resize(m);
            v64.x[l].resize(m);
            v64.r[l].resize(m);
            if (l > 0) {
                v32.b[l].resize(m);
                v64.b[l].resize(m);
            }
        }
        const std::size_t mc = static_cast<std::size_t>(h->bottom_n) * K;
        v32.cb.resize(mc);
        v32.cx.resize(mc);
        v64.cb.resize(mc);
        v64.cx.resize(mc);
        v32.part.resize(mc * DenseGrid<float>(h->bottom_n, K, sm_count).splits);
        v64.part.resize(mc * DenseGrid<double>(h->bottom_n, K, sm_count).splits);
        for (auto* a : {&rz, &alpha, &beta, &ref_sq, &rr0, &rel, &eta, &r0sq, &init_rel, &tolv}) a->resize(K);
        for (auto* a : {&frozen, &outer_conv, &conv_iter}) a->resize(K);
        iter_counter.resize(1);
        cap.resize(1);
        counter.resize(1);
        counter.zero(stream);
        partials.resize(static_cast<std::size_t>(kMaxReduceBlocks) * K);
        if (h_flags) cudaFreeHost(h_flags);
        if (h_dbl) cudaFreeHost(h_dbl);
        CUNIBS_CHECK(cudaMallocHost(&h_flags, sizeof(int) * 4 * K));
        CUNIBS_CHECK(cudaMallocHost(&h_dbl, sizeof(double) * 4 * K));
        kcap = K;
        CUNIBS_CHECK(cudaStreamSynchronize(stream));
    }

    // Level accessors per precision.
    template <typename T>
    const T* lval(int l) const;
    template <typename T>
    const T* ldinv(int l) const;
    template <typename T>
    const T* pval(int l) const;
    template <typename T>
    const T* rval(int l) const;
    template <typename T>
    const T* cinv() const;
    template <typename T>
    VWork<T>& vw();

    // z = M b. jz_done: the finest level's first smoothing step is already in its buffer (fused into
    // the PCG update). dot: fuse r . z and the beta update into the last step (finest level, one lane
    // per row); returns whether it did.
    template <typename T, int K>
    bool vcycle(const T* b, T* z, bool jz_done = false, bool dot = false);
    // x = inv b at the V-cycle's bottom (bottom_n rows, K columns).
    template <typename T, int K>
    void dense_bottom(const T* b, T* x);
    template <typename T>
    T* first0() {
        VWork<T>& w = vw<T>();
        return (h->cheby.degree % 2) ? w.x[0].get() : w.r[0].get();
    }
    // z = M r_v (V-cycle in TZ) and beta; the next iteration's SpMV forms p = z + beta p.
    template <typename TZ, int K>
    void pcg_tail(TZ* r_v, TZ* z, bool jz_done);
    // Sub-lanes per row on the finest operator (the PCG's own matrix), capped where the reducing
    // kernels' 64/TPR-row tiles need at least four rows.
    int tpr0() const {
        const int t = h->levels.empty() ? choose_tpr(h->nc, h->coarse.nnz) : h->levels[0].tpr_a;
        return t > 16 ? 16 : t;
    }
    void set_cap(int v) {
        h_flags[0] = v;
        CUNIBS_CHECK(cudaMemcpyAsync(cap.get(), h_flags, sizeof(int), cudaMemcpyHostToDevice, stream));
    }
    // One PCG iteration with Krylov vectors in T and the V-cycle in TZ (r_v is r in TZ; the same
    // buffer as r when the types agree).
    template <typename T, typename TZ, int K>
    void pcg_iteration(const int* ptr, const int* col, const T* val, T* x, T* r, T* p, T* ap, TZ* r_v, TZ* z,
                       double tol, const double* tol_vec, const double* ref, int record,
                       cudaGraphConditionalHandle loop = 0, int use_loop = 0);
    DevArray<int> cap;
    // Device-side loop: body(handle) is captured once into the body of a conditional WHILE node and
    // replayed until a kernel in it clears the condition. Returns false when the driver cannot
    // build such a graph (the caller then loops on the host).
    template <typename Body>
    bool run_while(std::tuple<int, int, int> key, Body&& body, long long* nodes_out) {
        auto it = graphs.find(key);
        if (it == graphs.end()) {
            if (while_unsupported) return false;
            cudaGraph_t g = nullptr;
            if (cudaGraphCreate(&g, 0) != cudaSuccess) return fail_while();
            cudaGraphConditionalHandle handle;
            if (cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
                cudaGraphDestroy(g);
                return fail_while();
            }
            cudaGraphNodeParams np = {};
            np.type = cudaGraphNodeTypeConditional;
            np.conditional.handle = handle;
            np.conditional.type = cudaGraphCondTypeWhile;
            np.conditional.size = 1;
            cudaGraphNode_t node;
            if (cudaGraphAddNode(&node, g, nullptr, 0, &np) != cudaSuccess) {
                cudaGraphDestroy(g);
                return fail_while();
            }
            cudaGraph_t bodyg = np.conditional.phGraph_out[0];
            const long long before = launch_counter().load();
            if (cudaStreamBeginCaptureToGraph(stream, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
                cudaSuccess) {
                cudaGraphDestroy(g);
                return fail_while();
            }
            body(handle);
            cudaGraph_t captured = nullptr;
            const cudaError_t end = cudaStreamEndCapture(stream, &captured);
            launch_counter().store(before);
            if (end != cudaSuccess) {
                cudaGraphDestroy(g);
                return fail_while();
            }
            std::size_t n_nodes = 0;
            CUNIBS_CHECK(cudaGraphGetNodes(bodyg, nullptr, &n_nodes));
            cudaGraphExec_t ex = nullptr;
            const cudaError_t inst = cudaGraphInstantiate(&ex, g, 0);
            cudaGraphDestroy(g);
            if (inst != cudaSuccess) return fail_while();
            it = graphs.emplace(key, std::make_pair(ex, static_cast<long long>(n_nodes))).first;
        }
        CUNIBS_CHECK(cudaGraphLaunch(it->second.first, stream));
        *nodes_out = it->second.second;
        return true;
    }
    bool while_unsupported = false;
    bool fail_while() {
        (void)cudaGetLastError();
        while_unsupported = true;
        return false;
    }
    template <int K, typename TZ>
    void solve_plain(int k, const Params& prm, SolveStats& st, bool warm);
    template <int K>
    void solve_mixed(int k, const Params& prm, SolveStats& st, bool warm);
    // R = B - A X in FP64 for a warm start, then the per-column zero-guess fallback.
    template <int K>
    void warm_residual(const DevCsr<double>& A) {
        constexpr int TT = tile_threads<K>();
        dispatch_tpr<K>(tpr0(), [&](auto tc) {
            constexpr int TPR = decltype(tc)::value;
            residual64_kernel<K, TPR><<<(n + ReduceTile<TPR>::kRows - 1) / ReduceTile<TPR>::kRows, TT, 0, stream>>>(
                n, A.ptr.get(), A.col.get(), A.val.get(), B.get(), X.get(), R.get());
        });
        norm2_kernel<double, K><<<reduce_grid(n), TT, 0, stream>>>(n, R.get(), partials.get(), counter.get(),
                                                                  r0sq.get());
        guess_fallback_kernel<K><<<n_tiles(n), TT, 0, stream>>>(n, X.get(), R.get(), B.get(), ref_sq.get(),
                                                                r0sq.get(), init_rel.get());
        count_launch(3);
    }

    template <typename Body>
    void run_graph(std::tuple<int, int, int> key, Body&& body) {
        auto it = graphs.find(key);
        if (it == graphs.end()) {
            cudaGraph_t g = nullptr;
            // Captured launches do not execute; the replays below count the graph's kernels.
            const long long before = launch_counter().load();
            CUNIBS_CHECK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            body();
            const cudaError_t end = cudaStreamEndCapture(stream, &g);
            launch_counter().store(before);
            if (end != cudaSuccess || g == nullptr) {
                if (g) cudaGraphDestroy(g);
                (void)cudaGetLastError();
                body();  // capture failed: run eagerly
                return;
            }
            std::size_t n_nodes = 0;
            CUNIBS_CHECK(cudaGraphGetNodes(g, nullptr, &n_nodes));
            cudaGraphExec_t ex = nullptr;
            const cudaError_t inst = cudaGraphInstantiate(&ex, g, 0);
            cudaGraphDestroy(g);
            if (inst != cudaSuccess) {
                (void)cudaGetLastError();
                body();
                return;
            }
            it = graphs.emplace(key, std::make_pair(ex, static_cast<long long>(n_nodes))).first;
        }
        CUNIBS_CHECK(cudaGraphLaunch(it->second.first, stream));
        count_launch(it->second.second);
    }
};

template <>
const float* Solver::lval<float>(int l) const { return h->levels[l].a32.get(); }
template <>
const double* Solver::lval<double>(int l) const { return h->levels[l].a.val.get(); }
template <>
const float* Solver::ldinv<float>(int l) const { return h->levels[l].dinv32.get(); }
template <>
const double* Solver::ldinv<double>(int l) const { return h->levels[l].dinv.get(); }
template <>
const float* Solver::pval<float>(int l) const { return h->levels[l].p32.get(); }
template <>
const double* Solver::pval<double>(int l) const { return h->levels[l].p.val.get(); }
template <>
const float* Solver::rval<float>(int l) const { return h->levels[l].r32.get(); }
template <>
const double* Solver::rval<double>(int l) const { return h->levels[l].r.val.get(); }
// The dense inverse at the V-cycle's bottom (see Hierarchy::vcycle_levels).
template <>
const float* Solver::cinv<float>() const {
    return h->vcycle_levels < static_cast<int>(h->levels.size()) ? h->level_inv32.get() : h->coarse_inv32.get();
}
template <>
const double* Solver::cinv<double>() const {
    return h->vcycle_levels < static_cast<int>(h->levels.size()) ? h->level_inv.get() : h->coarse_inv.get();
}
template <>
VWork<float>& Solver::vw<float>() { return v32; }
template <>
VWork<double>& Solver::vw<double>() { return v64; }

template <typename T, int K>
void Solver::dense_bottom(const T* b, T* x) {
    const int nb = h->bottom_n;
    const DenseGrid<T> g(nb, K, sm_count);
    const std::size_t smem = g.smem();
    if (smem > 48 * 1024) {
        static std::once_flag opt_in;
        std::call_once(opt_in, [] {
            CUNIBS_CHECK(cudaFuncSetAttribute(dense_part_kernel<T, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              static_cast<int>(kDenseSmemBudget)));
        });
        if (smem > kDenseSmemBudget) fail(kEInternal, "dense bottom split too large for shared memory");
    }
    T* part = vw<T>().part.get();
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(g.col_blocks), static_cast<unsigned>(g.splits));
    cfg.blockDim = dim3(static_cast<unsigned>(g.threads));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    // Launched without programmatic serialization: its blocks (one per SM, most of the SM's shared
    // memory) would otherwise be made resident early and wait beside the restriction that feeds it.
    cfg.numAttrs = 0;
    CUNIBS_CHECK(cudaLaunchKernelEx(&cfg, dense_part_kernel<T, K>, nb, dense_ld(nb), g.cols, g.split_rows, cinv<T>(), b,
                                    part));
    launch_loop(pdl, dense_sum_kernel<T, K>, grid_for(static_cast<std::int64_t>(nb) * K), kBlock, stream, nb, g.splits,
                static_cast<const T*>(part), x);
    count_launch(2);
}

template <typename T, int K>
bool Solver::vcycle(const T* b, T* z, bool jz_done, bool dot) {
    const Hierarchy& H = *h;
    const Cheby& ch = H.cheby;
    const int L = H.vcycle_levels;
    VWork<T>& w = vw<T>();
    constexpr int TT = tile_threads<K>();
    cudaStream_t s = stream;
    if (L == 0) {
        dense_bottom<T, K>(b, z);
        return false;
    }
    const bool fuse_dot = dot && H.levels[0].tpr_a <= 16;
    const int cols = lane_cols;
    const int deg = ch.degree;
    const bool odd = (deg % 2) != 0;
    // One Chebyshev sweep of `deg` steps (vcycle.cu:585-617 buffer discipline). x0 == nullptr is a
    // zero initial guess whose first step, x = alpha0*dinv*b, the caller has already written into
    // `first`. Otherwise step 0 reads x0 and writes `first`; later steps alternate, writing over
    // the buffer that holds x_{i-1}, which the step kernel reads only at the row it writes.
    auto launch_cheby = [&](int l, const T* bi, const T* cur, const T* prev, T cc, T cp, T al, T* out) {
        const Level& lv = H.levels[l];
        if (lv.tpr_a == 1 && dispatch_cols<K>(cols, [&](auto cc_) {
                constexpr int C = decltype(cc_)::value;
                if constexpr (std::is_same<T, double>::value && C == 4) {
                    launch_loop(pdl, cheby_cols_kernel<T, K, 2>, col_grid<K, 2>(lv.n), kColBlock, s, lv.n,
                                lv.a.ptr.get(), lv.a.col.get(), lval<T>(l), ldinv<T>(l), bi, cur, prev, cc, cp, al,
                                out);
                } else {
                    launch_loop(pdl, cheby_cols_kernel<T, K, C>, col_grid<K, C>(lv.n), kColBlock, s, lv.n,
                                lv.a.ptr.get(), lv.a.col.get(), lval<T>(l), ldinv<T>(l), bi, cur, prev, cc, cp, al,
                                out);
                }
            })) {
            count_launch();
            return;
        }
        if (lv.tpr_a > 1 && dispatch_subcols<K>(lv.tpr_a, cols, [&](auto tc, auto cc_) {
                constexpr int TPR = decltype(tc)::value;
                constexpr int C = decltype(cc_)::value;
                launch_loop(pdl, cheby_subcols_kernel<T, K, TPR, C>, subcol_grid<K, TPR, C>(lv.n), kColBlock, s, lv.n,
                            lv.a.ptr.get(), lv.a.col.get(), lval<T>(l), ldinv<T>(l), bi, cur, prev, cc, cp, al, out);
            })) {
            count_launch();
            return;
        }
        dispatch_tpr<K>(lv.tpr_a, [&](auto tc) {
            constexpr int TPR = decltype(tc)::value;
            launch_loop(pdl, cheby_kernel<T, K, TPR>, group_grid<K, TPR>(lv.n), Group<K, TPR>::kBlock, s, lv.n,
                        lv.a.ptr.get(), lv.a.col.get(), lval<T>(l), ldinv<T>(l), bi, cur, prev, cc, cp, al, out);
        });
        count_launch();
    };
    auto sweep = [&](int l, const T* bi, T* x0, T* first, T* other, T* final_out) {
        auto target = [&](int st) -> T* {
            if (st + 1 == deg && final_out) return final_out;
            return (st % 2) ? other : first;
        };
        T* cur;
        T* prev;
        if (x0 == nullptr) {
            cur = first;
            prev = first;
        } else {
            T* out = target(0);
            launch_cheby(l, bi, x0, x0, T(1), T(0), static_cast<T>(ch.alpha0), out);
            prev = x0;
            cur = out;
        }
        for (int st = 1; st < deg; ++st) {
            T* out = target(st);
            const T cp = (st == 1 && x0 == nullptr) ? T(0) : static_cast<T>(ch.c_prev[st - 1]);
            if (fuse_dot && l == 0 && final_out != nullptr && st + 1 == deg) {
                const Level& lv = H.levels[0];
                dispatch_tpr<K>(lv.tpr_a, [&](auto tc) {
                    constexpr int TPR = decltype(tc)::value;
                    launch_loop(pdl, cheby_dot_kernel<T, K, TPR>, reduce_grid_rows<TPR>(lv.n), TT, s, lv.n,
                                lv.a.ptr.get(), lv.a.col.get(), lval<T>(0), ldinv<T>(0), bi, cur, prev,
                                static_cast<T>(ch.c_cur[st - 1]), cp, static_cast<T>(ch.alpha[st - 1]), out,
                                partials.get(), counter.get(), rz.get(), frozen.get(), beta.get());
                });
                count_launch();
                prev = cur;
                cur = out;
                continue;
            }
            launch_cheby(l, bi, cur, prev, static_cast<T>(ch.c_cur[st - 1]), cp, static_cast<T>(ch.alpha[st - 1]), out);
            prev = cur;
            cur = out;
        }
        return cur;
    };
    // Down-sweep.
    for (int l = 0; l < L; ++l) {
        const Level& lv = H.levels[l];
        const T* bi = (l == 0) ? b : w.b[l].get();
        T* first = odd ? w.x[l].get() : w.r[l].get();
        T* other = odd ? w.r[l].get() : w.x[l].get();
        const unsigned g = n_tiles(lv.n);
        if (l == 0 && !jz_done) {
            launch_loop(pdl, jz_kernel<T, K>, g, TT, s, lv.n, ldinv<T>(0), bi, static_cast<T>(ch.alpha0), first);
            count_launch();
        }
        sweep(l, bi, nullptr, first, other, nullptr);
        const bool grouped =
            (lv.tpr_a == 1 && dispatch_cols<K>(cols, [&](auto cc_) {
                 constexpr int C =
                     (std::is_same<T, double>::value && decltype(cc_)::value == 4) ? 2 : decltype(cc_)::value;
                 launch_loop(pdl, residual_cols_kernel<T, K, C>, col_grid<K, C>(lv.n), kColBlock, s, lv.n,
                             lv.a.ptr.get(), lv.a.col.get(), lval<T>(l), w.x[l].get(), bi, w.r[l].get());
             })) ||
            (lv.tpr_a > 1 && dispatch_subcols<K>(lv.tpr_a, cols, [&](auto tc, auto cc_) {
                 constexpr int TPR = decltype(tc)::value;
                 constexpr int C = decltype(cc_)::value;
                 launch_loop(pdl, residual_subcols_kernel<T, K, TPR, C>, subcol_grid<K, TPR, C>(lv.n), kColBlock, s,
                             lv.n, lv.a.ptr.get(), lv.a.col.get(), lval<T>(l), w.x[l].get(), bi, w.r[l].get());
             }));
        if (!grouped) {
            dispatch_tpr<K>(lv.tpr_a, [&](auto tc) {
                constexpr int TPR = decltype(tc)::value;
                launch_loop(pdl, residual_kernel<T, K, TPR>, group_grid<K, TPR>(lv.n), Group<K, TPR>::kBlock, s,
                            lv.n, lv.a.ptr.get(), lv.a.col.get(), lval<T>(l), w.x[l].get(), bi, w.r[l].get());
            });
        }
        count_launch();
        const bool next_is_level = (l + 1 < L);
        T* nb = next_is_level ? w.b[l + 1].get() : w.cb.get();
        T* nx = nullptr;
        const T* nd = nullptr;
        if (next_is_level) {
            const bool nodd = odd;
            nx = nodd ? w.x[l + 1].get() : w.r[l + 1].get();
            nd = ldinv<T>(l + 1);
        }
        const bool rgrouped = lv.tpr_r > 1 && dispatch_subcols<K>(lv.tpr_r, cols, [&](auto tc, auto cc_) {
            constexpr int TPR = decltype(tc)::value;
            constexpr int C = decltype(cc_)::value;
            launch_loop(pdl, restrict_subcols_kernel<T, K, TPR, C>, subcol_grid<K, TPR, C>(lv.n_coarse), kColBlock, s,
                        lv.n_coarse, lv.r.ptr.get(), lv.r.col.get(), rval<T>(l), w.r[l].get(), nb, nd,
                        static_cast<T>(ch.alpha0), nx);
        });
        if (!rgrouped) dispatch_tpr<K>(lv.tpr_r, [&](auto tc) {
            constexpr int TPR = decltype(tc)::value;
            launch_loop(pdl, restrict_kernel<T, K, TPR>, group_grid<K, TPR>(lv.n_coarse), Group<K, TPR>::kBlock, s,
                        lv.n_coarse, lv.r.ptr.get(), lv.r.col.get(), rval<T>(l), w.r[l].get(), nb, nd,
                        static_cast<T>(ch.alpha0), nx);
        });
        count_launch();
    }
    dense_bottom<T, K>(w.cb.get(), w.cx.get());
    // Up-sweep.
    const T* xc = w.cx.get();
    for (int l = L - 1; l >= 0; --l) {
        const Level& lv = H.levels[l];
        const T* bi = (l == 0) ? b : w.b[l].get();
        const bool grouped =
            (lv.tpr_p == 1 && dispatch_cols<K>(cols, [&](auto cc_) {
                 constexpr int C =
                     (std::is_same<T, double>::value && decltype(cc_)::value == 4) ? 2 : decltype(cc_)::value;
                 launch_loop(pdl, prolong_cols_kernel<T, K, C>, col_grid<K, C>(lv.n), kColBlock, s, lv.n,
                             lv.p.ptr.get(), lv.p.col.get(), pval<T>(l), xc, w.x[l].get());
             })) ||
            (lv.tpr_p > 1 && dispatch_subcols<K>(lv.tpr_p, cols, [&](auto tc, auto cc_) {
                 constexpr int TPR = decltype(tc)::value;
                 constexpr int C = decltype(cc_)::value;
                 launch_loop(pdl, prolong_subcols_kernel<T, K, TPR, C>, subcol_grid<K, TPR, C>(lv.n), kColBlock, s,
                             lv.n, lv.p.ptr.get(), lv.p.col.get(), pval<T>(l), xc, w.x[l].get());
             }));
        if (!grouped) {
            dispatch_tpr<K>(lv.tpr_p, [&](auto tc) {
                constexpr int TPR = decltype(tc)::value;
                launch_loop(pdl, prolong_kernel<T, K, TPR>, group_grid<K, TPR>(lv.n), Group<K, TPR>::kBlock, s,
                            lv.n, lv.p.ptr.get(), lv.p.col.get(), pval<T>(l), xc, w.x[l].get());
            });
        }
        count_launch();
        // The level's smoothed correction stays wherever its sweep left it; the next finer
        // prolongation reads it from there.
        xc = sweep(l, bi, w.x[l].get(), w.r[l].get(), w.x[l].get(), (l == 0) ? z : nullptr);
    }
    // The fused step exists only when the sweep has a step after its first (degree >= 2).
    return fuse_dot && deg >= 2;
}

// Before a first tail: p = 0 and rz = 1, so beta is finite and p becomes z.
// Per-column start of a PCG solve: a zero right-hand side column starts (and stays) frozen at
// iteration 0, so the loop never waits on it; the host reports it after the solve.
__global__ void start_columns_kernel(const double* __restrict__ ref_sq, int K, int max_iters, int* __restrict__ frozen,
                                     int* __restrict__ conv_iter, double* __restrict__ rel) {
    const int c = threadIdx.x;
    if (c < K) {
        const bool live = ref_sq[c] > 0.0;
        frozen[c] = live ? 0 : 1;
        conv_iter[c] = live ? max_iters : 0;
        rel[c] = 0.0;
    }
}

__global__ void fill_kernel(double* v, int n, double x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = x;
}

template <typename TZ, int K>
void Solver::pcg_tail(TZ* r_v, TZ* z, bool jz_done) {
    constexpr int TT = tile_threads<K>();
    const bool fused = vcycle<TZ, K>(r_v, z, jz_done, true);
    if (!fused) {
        launch_loop(pdl, dot_beta_kernel<TZ, K>, reduce_grid(n), TT, stream, n, r_v, z, partials.get(), counter.get(),
                    rz.get(), frozen.get(), beta.get());
        count_launch();
    }
}

template <typename T, typename TZ, int K>
void Solver::pcg_iteration(const int* ptr, const int* col, const T* val, T* x, T* r, T* p, T* ap, TZ* r_v, TZ* z,
                           double tol, const double* tol_vec, const double* ref, int record,
                           cudaGraphConditionalHandle loop, int use_loop) {
    constexpr int TT = tile_threads<K>();
    const unsigned g = reduce_grid(n);
    dispatch_tpr<K>(tpr0(), [&](auto tc) {
        constexpr int TPR = decltype(tc)::value;
        launch_loop(pdl, spmv_alpha_kernel<T, TZ, K, TPR>, reduce_grid_rows<TPR>(n), TT, stream, n, ptr, col, val, z,
                    p, ap, partials.get(), counter.get(), rz.get(), beta.get(), frozen.get(), alpha.get());
    });
    count_launch();
    const bool has_levels = !h->levels.empty();
    constexpr bool narrow = !std::is_same<T, TZ>::value;
    launch_loop(pdl, update_xr_kernel<T, TZ, K>, g, TT, stream, n, alpha.get(), p, ap, x, r, partials.get(),
                counter.get(), ref, tol, tol_vec, frozen.get(), iter_counter.get(), conv_iter.get(), rel.get(), record,
                has_levels ? ldinv<TZ>(0) : nullptr, static_cast<TZ>(h->cheby.alpha0),
                has_levels ? first0<TZ>() : nullptr, narrow ? r_v : nullptr, loop, use_loop, cap.get());
    count_launch();
    pcg_tail<TZ, K>(r_v, z, has_levels);
}

template <int K, typename TZ>
void Solver::solve_plain(int k, const Params& prm, SolveStats& st, bool warm) {
    constexpr bool narrow = !std::is_same<TZ, double>::value;
    TZ* rv = nullptr;
    TZ* zv = nullptr;
    if constexpr (narrow) {
        rv = r32.get();
        zv = z32.get();
    } else {
        rv = R.get();
        zv = Z.get();
    }
    const int key = narrow ? 4 : 2;
    constexpr int TT = tile_threads<K>();
    const unsigned g = n_tiles(n);
    cudaStream_t s = stream;
    const DevCsr<double>& A = h->levels.empty() ? h->coarse : h->levels[0].a;
    const std::size_t nk = static_cast<std::size_t>(n) * K;
    norm2_kernel<double, K><<<reduce_grid(n), TT, 0, s>>>(n, B.get(), partials.get(), counter.get(), ref_sq.get()); count_launch();
    if (warm) {
        warm_residual<K>(A);
    } else {
        X.zero(s);
        CUNIBS_CHECK(cudaMemcpyAsync(R.get(), B.get(), nk * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    iter_counter.zero(s);
    P.zero(s);
    AP.zero(s);  // the first iteration's Ap = A z + beta Ap reads it
    start_columns_kernel<<<1, 32, 0, s>>>(ref_sq.get(), K, prm.max_iters, frozen.get(), conv_iter.get(), rel.get());
    count_launch();
    fill_kernel<<<1, 32, 0, s>>>(rz.get(), K, 1.0);
    fill_kernel<<<1, 32, 0, s>>>(tolv.get(), K, prm.tolerance);
    count_launch(2);
    if constexpr (narrow) {
        const std::int64_t count = static_cast<std::int64_t>(n) * K;
        narrow_kernel<double, TZ><<<grid_for(count), kBlock, 0, s>>>(count, R.get(), rv);
        count_launch();
    }
    pcg_tail<TZ, K>(rv, zv, false);
    int it = 0;
    set_cap(prm.max_iters);
    long long nodes = 0;
    const bool device_loop = run_while({key, K, 0}, [&](cudaGraphConditionalHandle hnd) {
        pcg_iteration<double, TZ, K>(A.ptr.get(), A.col.get(), A.val.get(), X.get(), R.get(), P.get(), AP.get(), rv,
                                     zv, 0.0, tolv.get(), ref_sq.get(), 1, hnd, 1);
    }, &nodes);
    // The right-hand side norms (zero columns) and, after a device loop, its iteration count are
    // read with the caller's final readback: no host round trip of their own.
    CUNIBS_CHECK(cudaMemcpyAsync(h_dbl + 2 * K, ref_sq.get(), sizeof(double) * K, cudaMemcpyDeviceToHost, s));
    check_ref = true;
    if (device_loop) {
        CUNIBS_CHECK(cudaMemcpyAsync(h_flags + 2 * K, iter_counter.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        loop_nodes = nodes;
        st.iterations = -1;
        st.outer_steps = 1;
        return;
    }
    while (it < prm.max_iters) {
        const int m = std::min(prm.iters_per_sync, prm.max_iters - it);
        for (int j = 0; j < m; ++j) {
            run_graph({key + 10, K, 0}, [&] {
                pcg_iteration<double, TZ, K>(A.ptr.get(), A.col.get(), A.val.get(), X.get(), R.get(), P.get(),
                                             AP.get(), rv, zv, 0.0, tolv.get(), ref_sq.get(), 1);
            });
        }
        it += m;
        CUNIBS_CHECK(cudaMemcpyAsync(h_flags, frozen.get(), sizeof(int) * K, cudaMemcpyDeviceToHost, s));
        CUNIBS_CHECK(cudaStreamSynchronize(s));
        bool all = true;
        for (int c = 0; c < k; ++c) all = all && h_flags[c];
        if (all) break;
    }
    st.iterations = it;
    st.outer_steps = 1;
}

template <int K>
void Solver::solve_mixed(int k, const Params& prm, SolveStats& st, bool warm) {
    constexpr int TT = tile_threads<K>();
    const unsigned g = n_tiles(n);
    cudaStream_t s = stream;
    const DevCsr<double>& A = h->levels.empty() ? h->coarse : h->levels[0].a;
    const float* A32 = h->levels.empty() ? nullptr : h->levels[0].a32.get();
    DevArray<float> coarse32;
    if (A32 == nullptr) fail(kEInval, "mixed precision needs at least one AMG level");
    norm2_kernel<double, K><<<reduce_grid(n), TT, 0, s>>>(n, B.get(), partials.get(), counter.get(), ref_sq.get()); count_launch();
    if (warm) warm_residual<K>(A);
    outer_conv.zero(s);
    iter_counter.zero(s);
    CUNIBS_CHECK(cudaMemcpyAsync(h_dbl, ref_sq.get(), sizeof(double) * K, cudaMemcpyDeviceToHost, s));
    CUNIBS_CHECK(cudaStreamSynchronize(s));
    for (int c = 0; c < k; ++c)
        if (!(h_dbl[c] > 0.0)) fail(kEInval, "zero right-hand side column " + std::to_string(c));
    std::vector<int> init_iters(K, prm.max_iters);
    CUNIBS_CHECK(cudaMemcpyAsync(conv_iter.get(), init_iters.data(), sizeof(int) * K, cudaMemcpyHostToDevice, s));
    rel.zero(s);
    int total_inner = 0;
    int outer = 0;
    const int max_outer = 64;
    for (; outer < max_outer; ++outer) {
        dispatch_tpr<K>(tpr0(), [&](auto tc) {
            constexpr int TPR = decltype(tc)::value;
            true_residual_kernel<K, TPR><<<reduce_grid_rows<TPR>(n), TT, 0, s>>>(
                n, A.ptr.get(), A.col.get(), A.val.get(), B.get(), X.get(), r32.get(), partials.get(), counter.get(),
                ref_sq.get(), prm.tolerance, prm.inner_reduction, outer_conv.get(), frozen.get(), rr0.get(), eta.get(),
                iter_counter.get(), conv_iter.get(), rel.get());
        });
        count_launch();
        CUNIBS_CHECK(cudaMemcpyAsync(h_flags, outer_conv.get(), sizeof(int) * K, cudaMemcpyDeviceToHost, s));
        CUNIBS_CHECK(cudaStreamSynchronize(s));
        bool all = true;
        for (int c = 0; c < k; ++c) all = all && h_flags[c];
        if (all || total_inner >= prm.max_iters) break;
        // Each inner solve starts a fresh FP32 Krylov sequence on the true residual. (Continuing the
        // previous sequence across the replacement was measured: the FP32 recurrence drifts too far
        // from the true residual for the old direction to stay useful.)
        d32.zero(s);
        p32.zero(s);
        ap32.zero(s);
        fill_kernel<<<1, 32, 0, s>>>(rz.get(), K, 1.0);
        count_launch();
        pcg_tail<float, K>(r32.get(), z32.get(), false);
        int it = 0;
        const int cap_n = std::min(prm.inner_max_iters, prm.max_iters - total_inner);
        set_cap(total_inner + cap_n);
        long long nodes = 0;
        const bool device_loop = run_while({3, K, 0}, [&](cudaGraphConditionalHandle hnd) {
            pcg_iteration<float, float, K>(A.ptr.get(), A.col.get(), A32, d32.get(), r32.get(), p32.get(), ap32.get(),
                                           r32.get(), z32.get(), 0.0, eta.get(), rr0.get(), 0, hnd, 1);
        }, &nodes);
        if (device_loop) {
            CUNIBS_CHECK(cudaMemcpyAsync(h_flags, iter_counter.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
            CUNIBS_CHECK(cudaStreamSynchronize(s));
            it = h_flags[0] - total_inner;
            count_launch(nodes * it);
        }
        while (!device_loop && it < cap_n) {
            const int m = std::min(prm.iters_per_sync, cap_n - it);
            for (int j = 0; j < m; ++j) {
                run_graph({1, K, 0}, [&] {
                    pcg_iteration<float, float, K>(A.ptr.get(), A.col.get(), A32, d32.get(), r32.get(), p32.get(),
                                                   ap32.get(), r32.get(), z32.get(), 0.0, eta.get(), rr0.get(), 0);
                });
            }
            it += m;
            CUNIBS_CHECK(cudaMemcpyAsync(h_flags, frozen.get(), sizeof(int) * K, cudaMemcpyDeviceToHost, s));
            CUNIBS_CHECK(cudaStreamSynchronize(s));
            bool done = true;
            for (int c = 0; c < k; ++c) done = done && h_flags[c];
            if (done) break;
        }
        total_inner += it;
        add_correction_kernel<K><<<g, TT, 0, s>>>(n, X.get(), d32.get()); count_launch();
    }
    st.iterations = total_inner;
    st.outer_steps = outer + 1;
}

void SolverDeleter::operator()(Solver* s) const { delete s; }

SolverPtr make_solver(const Hierarchy& h, const Params& p) {
    (void)p;
    SolverPtr sv(new Solver());
    sv->h = &h;
    sv->n = h.levels.empty() ? h.nc : h.levels[0].n;
    // CUNIBS_SOLVER_HOST_LOOP=1 runs the same iteration graphs under a host loop instead of a
    // device-side WHILE node, for profilers that do not step into conditional graph bodies.
    const char* host_loop = std::getenv("CUNIBS_SOLVER_HOST_LOOP");
    sv->while_unsupported = host_loop != nullptr && host_loop[0] == '1';
    const char* pdl = std::getenv("CUNIBS_PROGRAMMATIC_LAUNCH");
    sv->pdl = pdl != nullptr && pdl[0] == '1';
    const char* lanes = std::getenv("CUNIBS_LANE_COLUMNS");
    if (lanes != nullptr && (lanes[0] == '1' || lanes[0] == '2' || lanes[0] == '4')) sv->lane_cols = lanes[0] - '0';
    int dev = 0;
    CUNIBS_CHECK(cudaGetDevice(&dev));
    CUNIBS_CHECK(cudaDeviceGetAttribute(&sv->sm_count, cudaDevAttrMultiProcessorCount, dev));
    // The solver's kernels go at the highest stream priority: block preparation may run beside them.
    int least = 0, greatest = 0;
    CUNIBS_CHECK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    CUNIBS_CHECK(cudaStreamCreateWithPriority(&sv->stream, cudaStreamNonBlocking, greatest));
    return sv;
}

template <typename F>
void dispatch_k(int K, F&& f) {
    switch (K) {
        case 1: f(std::integral_constant<int, 1>{}); break;
        case 2: f(std::integral_constant<int, 2>{}); break;
        case 4: f(std::integral_constant<int, 4>{}); break;
        case 8: f(std::integral_constant<int, 8>{}); break;
        case 16: f(std::integral_constant<int, 16>{}); break;
        default: fail(kEInval, "block width must be one of {1, 2, 4, 8, 16}");
    }
}

void solver_solve(Solver& sv, const double* Bin, double* Xout, int k, int K, const Params& prm, cudaStream_t s,
                  SolveStats& st, const double* X0) {
    if (k < 1 || k > K) fail(kEInval, "k must be in [1, block width]");
    dispatch_k(K, [&](auto kc) {
        constexpr int KK = decltype(kc)::value;
        sv.ensure(KK);
        sv.check_ref = false;
        // Join the caller's stream.
        cudaEvent_t ev;
        CUNIBS_CHECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        CUNIBS_CHECK(cudaEventRecord(ev, s));
        CUNIBS_CHECK(cudaStreamWaitEvent(sv.stream, ev, 0));
        const std::size_t nk = static_cast<std::size_t>(sv.n) * KK;
        CUNIBS_CHECK(cudaMemcpyAsync(sv.B.get(), Bin, nk * sizeof(double), cudaMemcpyDeviceToDevice, sv.stream));
        if (X0) CUNIBS_CHECK(cudaMemcpyAsync(sv.X.get(), X0, nk * sizeof(double), cudaMemcpyDeviceToDevice, sv.stream));
        else sv.X.zero(sv.stream);
        if (prm.precision == kMixed) sv.solve_mixed<KK>(k, prm, st, X0 != nullptr);
        else if (prm.precision == kFp64CgFp32Mg) sv.solve_plain<KK, float>(k, prm, st, X0 != nullptr);
        else sv.solve_plain<KK, double>(k, prm, st, X0 != nullptr);
        if (X0)
            CUNIBS_CHECK(cudaMemcpyAsync(sv.h_dbl + 3 * KK, sv.init_rel.get(), sizeof(double) * KK,
                                         cudaMemcpyDeviceToHost, sv.stream));
        CUNIBS_CHECK(cudaMemcpyAsync(Xout, sv.X.get(), nk * sizeof(double), cudaMemcpyDeviceToDevice, sv.stream));
        CUNIBS_CHECK(cudaMemcpyAsync(sv.h_flags, sv.conv_iter.get(), sizeof(int) * KK, cudaMemcpyDeviceToHost, sv.stream));
        CUNIBS_CHECK(cudaMemcpyAsync(sv.h_dbl, sv.rel.get(), sizeof(double) * KK, cudaMemcpyDeviceToHost, sv.stream));
        CUNIBS_CHECK(cudaEventRecord(ev, sv.stream));
        CUNIBS_CHECK(cudaStreamWaitEvent(s, ev, 0));
        CUNIBS_CHECK(cudaStreamSynchronize(sv.stream));
        cudaEventDestroy(ev);
        st.col_iters.assign(sv.h_flags, sv.h_flags + k);
        st.col_rel.assign(sv.h_dbl, sv.h_dbl + k);
        if (X0) st.col_init_rel.assign(sv.h_dbl + 3 * KK, sv.h_dbl + 3 * KK + k);
        if (st.iterations < 0) {
            st.iterations = sv.h_flags[2 * KK];
            count_launch(sv.loop_nodes * st.iterations);
        }
        if (sv.check_ref) {
            sv.check_ref = false;
            for (int c = 0; c < k; ++c)
                if (!(sv.h_dbl[2 * KK + c] > 0.0)) fail(kEInval, "zero right-hand side column " + std::to_string(c));
        }
    });
}

int solver_width_capacity(const Solver& sv) { return sv.kcap; }

void solver_vcycle(Solver& sv, const double* r, double* z, int k, bool fp32, cudaStream_t s) {
    (void)fp32;
    dispatch_k(k, [&](auto kc) {
        constexpr int KK = decltype(kc)::value;
        sv.ensure(KK);
        CUNIBS_CHECK(cudaStreamSynchronize(s));
        const std::size_t nk = static_cast<std::size_t>(sv.n) * KK;
        if (fp32) {
            // r (FP64) -> FP32, cycle, back to FP64. Every copy goes on the solver's stream: a plain
            // cudaMemcpy from pageable memory may return before its DMA has landed, and the solver's
            // non-blocking stream would not wait for it.
            std::vector<double> hr(nk);
            CUNIBS_CHECK(cudaMemcpyAsync(hr.data(), r, nk * sizeof(double), cudaMemcpyDeviceToHost, sv.stream));
            CUNIBS_CHECK(cudaStreamSynchronize(sv.stream));
            std::vector<float> hf(hr.begin(), hr.end());
            CUNIBS_CHECK(cudaMemcpyAsync(sv.r32.get(), hf.data(), nk * sizeof(float), cudaMemcpyHostToDevice, sv.stream));
            sv.vcycle<float, KK>(sv.r32.get(), sv.z32.get());
            CUNIBS_CHECK(cudaMemcpyAsync(hf.data(), sv.z32.get(), nk * sizeof(float), cudaMemcpyDeviceToHost, sv.stream));
            CUNIBS_CHECK(cudaStreamSynchronize(sv.stream));
            std::vector<double> hz(hf.begin(), hf.end());
            CUNIBS_CHECK(cudaMemcpyAsync(z, hz.data(), nk * sizeof(double), cudaMemcpyHostToDevice, sv.stream));
            CUNIBS_CHECK(cudaStreamSynchronize(sv.stream));
        } else {
            CUNIBS_CHECK(cudaMemcpyAsync(sv.R.get(), r, nk * sizeof(double), cudaMemcpyDeviceToDevice, sv.stream));
            sv.vcycle<double, KK>(sv.R.get(), sv.Z.get());
            CUNIBS_CHECK(cudaMemcpyAsync(z, sv.Z.get(), nk * sizeof(double), cudaMemcpyDeviceToDevice, sv.stream));
            CUNIBS_CHECK(cudaStreamSynchronize(sv.stream));
        }
        CUNIBS_LAUNCH_CHECK("vcycle");
    });
}

}  // namespace cunibs
