// Smoothed-aggregation AMG hierarchy on the device: SIZE_4 pairwise aggregation, l1-Jacobi
// diagonal, tentative and smoothed prolongators, deterministic sparse products for the Galerkin
// operators, and an FP64 Cholesky inverse of the coarsest operator.
//
// Compiled with -fmad=false so the CPU oracle reproduces every operator bit for bit, which is what
// keeps the aggregation (a function of floating-point edge weights) identical between the two.
//
// Reference behaviour restated: aggregate.cu:13-472 (AMGx SIZE_4 selector semantics: hash
// perturbation, tie-breaks, round-1/2 rules, leftover merge, order-preserving relabel),
// l1.cu:15-35, fem/solve.py:69-256 (tentative/smoothed prolongator, composed rounds, level loop,
// stopping rules). The sparse products are this project's own expand-sort-reduce design: row i's
// partial products are listed in (A entry, B entry) order, stably sorted by column, and summed in
// that order from zero, which makes the result a pure function of the inputs.
#include <cub/cub.cuh>

#include <cmath>

#include "internal.hpp"

namespace cunibs {
namespace {

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

template <typename T>
T read_scalar(const T* dev, cudaStream_t s) {
    T h{};
    CUNIBS_CHECK(cudaMemcpyAsync(&h, dev, sizeof(T), cudaMemcpyDeviceToHost, s));
    CUNIBS_CHECK(cudaStreamSynchronize(s));
    return h;
}

// --- SIZE_4 aggregation -------------------------------------------------------------------

__device__ __forceinline__ unsigned agg_hash(unsigned a, unsigned seed) {
    a ^= seed;
    a = (a + 0x7ed55d16u) + (a << 12);
    a = (a ^ 0xc761c23cu) + (a >> 19);
    a = (a + 0x165667b1u) + (a << 5);
    a = (a ^ 0xd3a2646cu) + (a << 9);
    a = (a + 0xfd7046c5u) + (a << 3);
    a = (a ^ 0xb55a4f09u) + (a >> 16);
    return a;
}

__device__ __forceinline__ bool is_candidate(int col, int row, int n) {
    return col != row && static_cast<unsigned>(col) < static_cast<unsigned>(n);
}

// Lexicographic max of (weight, column) from (0, -1); NaN weights never win.
__device__ __forceinline__ void best_take(float& bw, int& bc, float w, int col) {
    if (w > bw || (w == bw && col > bc)) {
        bw = w;
        bc = col;
    }
}

__device__ __forceinline__ void count_block(int pred, int* counter) {
    const int n = __syncthreads_count(pred);
    if (threadIdx.x == 0 && n) atomicAdd(counter, n);
}

__global__ void agg_diag_weights_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                        const float* __restrict__ va, float* __restrict__ diag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float d = 0.0f;
    for (int j = rp[i]; j < rp[i + 1]; ++j)
        if (ci[j] == i) {
            d = va[j];
            break;
        }
    diag[i] = d;
}

// w_ij = |a_ij| / max(|a_ii|, |a_jj|), perturbed by a hash of the unordered pair to break ties.
__global__ void agg_edge_weight_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                       const float* __restrict__ va, const float* __restrict__ diag,
                                       float* __restrict__ w) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float di = fabsf(diag[i]);
    for (int j = rp[i]; j < rp[i + 1]; ++j) {
        const int jc = ci[j];
        if (!is_candidate(jc, i, n)) {
            w[j] = -1.0f;
            continue;
        }
        const float den = fmaxf(di, fabsf(diag[jc]));
        const float ed = fabsf(va[j]) / den;
        const unsigned lo = static_cast<unsigned>(min(i, jc));
        const unsigned hi = static_cast<unsigned>(max(i, jc));
        const float frac = 1e-5f * static_cast<float>(agg_hash(lo, hi)) / 4294967295.0f;
        w[j] = __fmaf_rn(frac, ed, ed);
    }
}

__global__ void agg_init_kernel(int n, int* __restrict__ agg, int* __restrict__ partner, int* __restrict__ strongest) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    agg[i] = i;
    partner[i] = -1;
    strongest[i] = -1;
}

__global__ void agg_r1_find_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                   const float* __restrict__ w, const int* __restrict__ partner,
                                   int* __restrict__ strongest) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || partner[t] != -1) return;
    float bw = 0.0f;
    int bc = -1;
    for (int j = rp[t]; j < rp[t + 1]; ++j) {
        const int jc = ci[j];
        if (!is_candidate(jc, t, n) || partner[jc] != -1) continue;
        best_take(bw, bc, w[j], jc);
    }
    if (bc != -1) strongest[t] = bc;
}

__global__ void agg_r1_match_kernel(int n, int* __restrict__ partner, int* __restrict__ agg,
                                    const int* __restrict__ strongest, int* __restrict__ remaining) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    int un = 0;
    if (t < n && partner[t] == -1) {
        const int pm = strongest[t];
        if (pm != -1 && strongest[pm] == t) {
            partner[t] = pm;
            agg[t] = min(pm, t);
        } else {
            un = 1;
        }
    }
    count_block(un, remaining);
}

__global__ void agg_r2_init_kernel(int n, int* __restrict__ partner, float* __restrict__ wsn,
                                   int* __restrict__ aggregated) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    if (partner[t] == -1) partner[t] = t;
    wsn[t] = -1.0f;
    aggregated[t] = -1;
}

__global__ void agg_r2_find_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                   const float* __restrict__ w, const int* __restrict__ aggregated,
                                   const int* __restrict__ agg, const int* __restrict__ partner,
                                   int* __restrict__ strongest, float* __restrict__ wsn) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || aggregated[t] != -1) return;
    const int p = partner[t];
    float bw = 0.0f;
    int bc = -1;
    for (int j = rp[t]; j < rp[t + 1]; ++j) {
        const int jc = ci[j];
        if (!is_candidate(jc, t, n)) continue;
        if (aggregated[jc] != -1 || jc == p) continue;
        best_take(bw, bc, w[j], jc);
    }
    if (bc != -1) {
        wsn[t] = bw;
        strongest[t] = agg[bc];
    }
}

// Both members of a pair adopt one proposal. Row t writes its own slot only, and reads its
// partner's only when the partner's proposal is strictly stronger, in which case the partner
// writes nothing: the read never races a write.
__global__ void agg_r2_agree_kernel(int n, int* __restrict__ aggregated, int* __restrict__ strongest,
                                    const float* __restrict__ wsn, const int* __restrict__ partner) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || aggregated[t] != -1) return;
    const int p = partner[t];
    const float mine = wsn[t];
    const float theirs = (p != -1) ? wsn[p] : -1.0f;
    if (mine < 0.0f && theirs < 0.0f) {
        aggregated[t] = 1;
        strongest[t] = -1;
    } else if (mine < theirs) {
        strongest[t] = strongest[p];
    }
}

__global__ void agg_r2_match_kernel(int n, int* __restrict__ agg, int* __restrict__ aggregated,
                                    const int* __restrict__ strongest, int* __restrict__ remaining) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    int un = 0;
    if (t < n && aggregated[t] == -1) {
        const int pm = strongest[t];
        const int mine = agg[t];
        if (pm != -1 && strongest[pm] == mine) {
            aggregated[t] = 1;
            agg[t] = min(pm, mine);
        } else {
            un = 1;
        }
    }
    count_block(un, remaining);
}

__global__ void agg_merge_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                 const float* __restrict__ w, const int* __restrict__ agg,
                                 const int* __restrict__ aggregated, int* __restrict__ cand) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || aggregated[t] != -1) return;
    float bw = 0.0f;
    int bc = -1;
    for (int j = rp[t]; j < rp[t + 1]; ++j) {
        const int jc = ci[j];
        if (!is_candidate(jc, t, n) || aggregated[jc] == -1) continue;
        best_take(bw, bc, w[j], jc);
    }
    cand[t] = (bc != -1) ? agg[bc] : t;
}

__global__ void agg_join_kernel(int n, int* __restrict__ agg, int* __restrict__ aggregated, const int* __restrict__ cand) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n && aggregated[t] == -1) {
        agg[t] = cand[t];
        aggregated[t] = 1;
    }
}

__global__ void agg_mark_kernel(int n, const int* __restrict__ agg, int* __restrict__ used) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) used[agg[t]] = 1;
}

__global__ void agg_relabel_kernel(int n, int* __restrict__ agg, const int* __restrict__ excl) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) agg[t] = excl[agg[t]];
}

// --- sparse products ----------------------------------------------------------------------

__global__ void row_of_kernel(const int* __restrict__ ptr, int n, int* __restrict__ row_of) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int p = ptr[i]; p < ptr[i + 1]; ++p) row_of[p] = i;
}

__global__ void spgemm_count_kernel(int n, const int* __restrict__ ap, const int* __restrict__ ac,
                                    const int* __restrict__ bp, long long* __restrict__ cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long c = 0;
    for (int p = ap[i]; p < ap[i + 1]; ++p) {
        const int j = ac[p];
        c += bp[j + 1] - bp[j];
    }
    cnt[i] = c;
}

__global__ void spgemm_expand_kernel(int n, const int* __restrict__ ap, const int* __restrict__ ac,
                                     const double* __restrict__ av, const int* __restrict__ bp,
                                     const int* __restrict__ bc, const double* __restrict__ bv,
                                     const long long* __restrict__ off, std::uint64_t* __restrict__ key,
                                     double* __restrict__ val) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long o = off[i];
    const std::uint64_t hi = static_cast<std::uint64_t>(i) << 32;
    for (int p = ap[i]; p < ap[i + 1]; ++p) {
        const int j = ac[p];
        const double a = av[p];
        for (int q = bp[j]; q < bp[j + 1]; ++q) {
            key[o] = hi | static_cast<std::uint32_t>(bc[q]);
            val[o] = a * bv[q];
            ++o;
        }
    }
}

__global__ void head_flags64_kernel(const std::uint64_t* __restrict__ keys, long long len, int* __restrict__ flags) {
    const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q < len) flags[q] = (q == 0 || keys[q] != keys[q - 1]) ? 1 : 0;
}

__global__ void reduce_runs_kernel(const std::uint64_t* __restrict__ keys, const double* __restrict__ vals,
                                   const int* __restrict__ flags, const int* __restrict__ pos, long long len,
                                   int* __restrict__ col, int* __restrict__ row_of, double* __restrict__ out) {
    const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= len || !flags[q]) return;
    const std::uint64_t k = keys[q];
    double acc = 0.0;
    long long e = q;
    while (e < len && keys[e] == k) acc = acc + vals[e++];
    const int p = pos[q];
    col[p] = static_cast<int>(k & 0xffffffffu);
    row_of[p] = static_cast<int>(k >> 32);
    out[p] = acc;
}

__global__ void segment_starts_kernel(const int* __restrict__ sorted_keys, long long len, int n_segments,
                                      int* __restrict__ ptr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n_segments) return;
    long long lo = 0, hi = len;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (sorted_keys[mid] < i) lo = mid + 1;
        else hi = mid;
    }
    ptr[i] = static_cast<int>(lo);
}

__global__ void gather_kernel(const double* __restrict__ src, const int* __restrict__ idx, long n,
                              double* __restrict__ dst) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q < n) dst[q] = src[idx[q]];
}

__global__ void gather_int_kernel(const int* __restrict__ src, const int* __restrict__ idx, long n,
                                  int* __restrict__ dst) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q < n) dst[q] = src[idx[q]];
}

__global__ void iota_kernel(int* out, long n) {
    const long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = static_cast<int>(i);
}

__global__ void l1_dinv_kernel(const int* __restrict__ ptr, const int* __restrict__ col,
                               const double* __restrict__ val, int n, double* __restrict__ dinv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc = 0.0, diag = 0.0;
    for (int p = ptr[i]; p < ptr[i + 1]; ++p) {
        acc = acc + fabs(val[p]);
        if (col[p] == i) diag = val[p];
    }
    if (diag < 0.0) acc = -acc;
    if (acc == 0.0) acc = 1.0;
    dinv[i] = 1.0 / acc;
}

__global__ void agg_count_kernel(const int* __restrict__ agg, int n, int* __restrict__ count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicAdd(count + agg[i], 1);
}

__global__ void tentative_kernel(const int* __restrict__ agg, const int* __restrict__ count, int n,
                                 int* __restrict__ ptr, int* __restrict__ col, double* __restrict__ val) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    ptr[i] = i;
    if (i == n) return;
    col[i] = agg[i];
    val[i] = 1.0 / sqrt(static_cast<double>(count[agg[i]]));
}

// P = (I - 4/3 D^-1 A) P_tent applied to AP_tent in place.
__global__ void smooth_prolongator_kernel(const int* __restrict__ ptr, const int* __restrict__ col,
                                          double* __restrict__ val, const int* __restrict__ agg,
                                          const double* __restrict__ pt, const double* __restrict__ dinv, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double damping = 4.0 / 3.0;
    for (int q = ptr[i]; q < ptr[i + 1]; ++q) {
        const double scaled = damping * (dinv[i] * val[q]);
        val[q] = (col[q] == agg[i]) ? (pt[i] - scaled) : -scaled;
    }
}

__global__ void to_f32_kernel(const double* __restrict__ in, long n, float* __restrict__ out) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q < n) out[q] = static_cast<float>(in[q]);
}

__global__ void compose_kernel(int* __restrict__ agg, const int* __restrict__ step, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) agg[i] = step[agg[i]];
}

// --- coarse Cholesky inverse --------------------------------------------------------------

__global__ void densify_kernel(const int* __restrict__ ptr, const int* __restrict__ col,
                               const double* __restrict__ val, int n, double* __restrict__ m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int p = ptr[i]; p < ptr[i + 1]; ++p) m[static_cast<long>(i) * n + col[p]] = val[p];
}

// Left-looking Cholesky L L^T of a dense SPD matrix in place, one block; column j's diagonal by
// thread 0, then the column below it in parallel. Sums run in ascending k like the CPU restatement.
__global__ void cholesky_kernel(double* __restrict__ m, int n, int* __restrict__ status) {
    __shared__ double d_sh;
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    for (int j = 0; j < n; ++j) {
        if (threadIdx.x == 0) {
            double d = m[static_cast<long>(j) * n + j];
            for (int k = 0; k < j; ++k) d -= m[static_cast<long>(j) * n + k] * m[static_cast<long>(j) * n + k];
            if (!(d > 0.0)) {
                bad = 1;
                d = 1.0;
            }
            d = sqrt(d);
            m[static_cast<long>(j) * n + j] = d;
            d_sh = d;
        }
        __syncthreads();
        const double d = d_sh;
        for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
            double s = m[static_cast<long>(i) * n + j];
            for (int k = 0; k < j; ++k) s -= m[static_cast<long>(i) * n + k] * m[static_cast<long>(j) * n + k];
            m[static_cast<long>(i) * n + j] = s / d;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *status = bad;
}

// inv = L^-T L^-1, one thread per column of the identity.
__global__ void cholesky_inverse_kernel(const double* __restrict__ L, int n, double* __restrict__ y,
                                        double* __restrict__ inv) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    double* yc = y + static_cast<long>(c) * n;
    for (int i = 0; i < n; ++i) {
        double s = (i == c) ? 1.0 : 0.0;
        for (int k = 0; k < i; ++k) s -= L[static_cast<long>(i) * n + k] * yc[k];
        yc[i] = s / L[static_cast<long>(i) * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = yc[i];
        for (int k = i + 1; k < n; ++k) s -= L[static_cast<long>(k) * n + i] * inv[static_cast<long>(k) * n + c];
        inv[static_cast<long>(i) * n + c] = s / L[static_cast<long>(i) * n + i];
    }
}

void tentative(const DevArray<int>& agg, int n, int nc, DevCsr<double>& pt, cudaStream_t s) {
    DevArray<int> count(nc);
    count.zero(s);
    agg_count_kernel<<<grid_for(n), kBlock, 0, s>>>(agg.get(), n, count.get()); count_launch();
    pt.n = n;
    pt.ncol = nc;
    pt.nnz = n;
    pt.ptr.resize(n + 1);
    pt.col.resize(n);
    pt.val.resize(n);
    tentative_kernel<<<grid_for(n + 1), kBlock, 0, s>>>(agg.get(), count.get(), n, pt.ptr.get(), pt.col.get(),
                                                        pt.val.get()); count_launch();
    CUNIBS_LAUNCH_CHECK("tentative prolongator");
}

void galerkin(const DevCsr<double>& a, const DevCsr<double>& p, DevCsr<double>& out, cudaStream_t s) {
    DevCsr<double> ap, r;
    spgemm(a, p, ap, s);
    transpose(p, r, s);
    spgemm(r, ap, out, s);
}

// One level's aggregation: `rounds` composed SIZE_4 passes (fem/solve.py:178-209).
int aggregate_level(const DevCsr<double>& a, const Params& prm, DevArray<int>& agg, cudaStream_t s) {
    DevCsr<double> cur_store;
    const DevCsr<double>* cur = &a;
    bool have = false;
    int n_coarse = a.n;
    for (int round = 0; round < prm.agg_rounds; ++round) {
        if (cur->n <= prm.min_coarse_rows) break;
        DevArray<float> v32(cur->nnz ? cur->nnz : 1);
        to_f32_kernel<<<grid_for(cur->nnz), kBlock, 0, s>>>(cur->val.get(), cur->nnz, v32.get()); count_launch();
        DevArray<int> step(cur->n);
        const int nc = select_size4(cur->n, cur->ptr.get(), cur->col.get(), v32.get(), step.get(), s);
        if (nc == cur->n || nc < prm.min_coarse_rows) break;
        if (!have) {
            agg.resize(a.n);
            CUNIBS_CHECK(cudaMemcpyAsync(agg.get(), step.get(), sizeof(int) * a.n, cudaMemcpyDeviceToDevice, s));
            have = true;
        } else {
            compose_kernel<<<grid_for(a.n), kBlock, 0, s>>>(agg.get(), step.get(), a.n); count_launch();
        }
        n_coarse = nc;
        if (round + 1 < prm.agg_rounds) {
            DevCsr<double> pt, next;
            tentative(step, cur->n, nc, pt, s);
            galerkin(*cur, pt, next, s);
            cur_store = std::move(next);
            cur = &cur_store;
        }
    }
    return have ? n_coarse : -1;
}

void to_f32(const DevArray<double>& in, long n, DevArray<float>& out, cudaStream_t s) {
    out.resize(n ? n : 1);
    to_f32_kernel<<<grid_for(n), kBlock, 0, s>>>(in.get(), n, out.get()); count_launch();
}

}  // namespace

int select_size4(int n, const int* rp, const int* ci, const float* va, int* agg, cudaStream_t s) {
    if (n <= 0) return 0;
    const int nnz = read_scalar(rp + n, s);
    DevArray<float> diag(n), w(nnz > 0 ? nnz : 1), wsn(n);
    DevArray<int> partner(n), strongest(n), aggregated(n), cand(n), counter(1), used(n + 1), excl(n + 1);
    const unsigned blocks = grid_for(n);
    agg_diag_weights_kernel<<<blocks, kBlock, 0, s>>>(n, rp, ci, va, diag.get()); count_launch();
    if (nnz > 0) {
        agg_edge_weight_kernel<<<blocks, kBlock, 0, s>>>(n, rp, ci, va, diag.get(), w.get());
        count_launch();
    }
    agg_init_kernel<<<blocks, kBlock, 0, s>>>(n, agg, partner.get(), strongest.get()); count_launch();
    CUNIBS_LAUNCH_CHECK("aggregation init");
    int unassigned = n;
    for (int iter = 0; iter <= 15; ++iter) {
        counter.zero(s);
        agg_r1_find_kernel<<<blocks, kBlock, 0, s>>>(n, rp, ci, w.get(), partner.get(), strongest.get()); count_launch();
        agg_r1_match_kernel<<<blocks, kBlock, 0, s>>>(n, partner.get(), agg, strongest.get(), counter.get()); count_launch();
        CUNIBS_LAUNCH_CHECK("aggregation round 1");
        const int prev = unassigned;
        unassigned = read_scalar(counter.get(), s);
        if (unassigned == 0 || unassigned == prev) break;
    }
    agg_r2_init_kernel<<<blocks, kBlock, 0, s>>>(n, partner.get(), wsn.get(), aggregated.get()); count_launch();
    unassigned = n;
    for (int iter = 0; iter <= 15; ++iter) {
        counter.zero(s);
        agg_r2_find_kernel<<<blocks, kBlock, 0, s>>>(n, rp, ci, w.get(), aggregated.get(), agg, partner.get(),
                                                    strongest.get(), wsn.get()); count_launch();
        agg_r2_agree_kernel<<<blocks, kBlock, 0, s>>>(n, aggregated.get(), strongest.get(), wsn.get(), partner.get()); count_launch();
        agg_r2_match_kernel<<<blocks, kBlock, 0, s>>>(n, agg, aggregated.get(), strongest.get(), counter.get()); count_launch();
        CUNIBS_LAUNCH_CHECK("aggregation round 2");
        const int prev = unassigned;
        unassigned = read_scalar(counter.get(), s);
        if (unassigned == 0 || unassigned == prev ||
            static_cast<float>(unassigned) / static_cast<float>(n) < 0.05f)
            break;
    }
    if (unassigned != 0) {
        agg_merge_kernel<<<blocks, kBlock, 0, s>>>(n, rp, ci, w.get(), agg, aggregated.get(), cand.get()); count_launch();
        agg_join_kernel<<<blocks, kBlock, 0, s>>>(n, agg, aggregated.get(), cand.get()); count_launch();
    }
    used.zero(s);
    agg_mark_kernel<<<blocks, kBlock, 0, s>>>(n, agg, used.get()); count_launch();
    exclusive_scan(used.get(), excl.get(), n + 1, s);
    agg_relabel_kernel<<<blocks, kBlock, 0, s>>>(n, agg, excl.get()); count_launch();
    CUNIBS_LAUNCH_CHECK("aggregation relabel");
    return read_scalar(excl.get() + n, s);
}

void spgemm(const DevCsr<double>& A, const DevCsr<double>& B, DevCsr<double>& C, cudaStream_t s) {
    const int n = A.n;
    C.n = n;
    C.ncol = B.ncol;
    DevArray<long long> cnt(n + 1), off(n + 1);
    CUNIBS_CHECK(cudaMemsetAsync(cnt.get() + n, 0, sizeof(long long), s));
    spgemm_count_kernel<<<grid_for(n), kBlock, 0, s>>>(n, A.ptr.get(), A.col.get(), B.ptr.get(), cnt.get()); count_launch();
    exclusive_scan(cnt.get(), off.get(), n + 1, s);
    const long long T = read_scalar(off.get() + n, s);
    if (T > 0x7fffffffLL) fail(kENoMem, "sparse product exceeds 2^31 partial products");
    DevArray<std::uint64_t> key(T ? T : 1), key_s(T ? T : 1);
    DevArray<double> val(T ? T : 1), val_s(T ? T : 1);
    spgemm_expand_kernel<<<grid_for(n), kBlock, 0, s>>>(n, A.ptr.get(), A.col.get(), A.val.get(), B.ptr.get(),
                                                        B.col.get(), B.val.get(), off.get(), key.get(), val.get()); count_launch();
    sort_pairs(key.get(), key_s.get(), val.get(), val_s.get(), T, 32 + bits_for(n), s);
    DevArray<int> flags(T + 1), pos(T + 1);
    head_flags64_kernel<<<grid_for(T), kBlock, 0, s>>>(key_s.get(), T, flags.get()); count_launch();
    CUNIBS_CHECK(cudaMemsetAsync(flags.get() + T, 0, sizeof(int), s));
    exclusive_scan(flags.get(), pos.get(), T + 1, s);
    const int nnz = read_scalar(pos.get() + T, s);
    C.nnz = nnz;
    C.col.resize(nnz ? nnz : 1);
    C.val.resize(nnz ? nnz : 1);
    DevArray<int> row_of(nnz ? nnz : 1);
    reduce_runs_kernel<<<grid_for(T), kBlock, 0, s>>>(key_s.get(), val_s.get(), flags.get(), pos.get(), T,
                                                      C.col.get(), row_of.get(), C.val.get()); count_launch();
    C.ptr.resize(n + 1);
    segment_starts_kernel<<<grid_for(n + 1), kBlock, 0, s>>>(row_of.get(), nnz, n, C.ptr.get()); count_launch();
    CUNIBS_LAUNCH_CHECK("spgemm");
}

void transpose(const DevCsr<double>& A, DevCsr<double>& T, cudaStream_t s) {
    const long nnz = A.nnz;
    T.n = A.ncol;
    T.ncol = A.n;
    T.nnz = nnz;
    DevArray<int> row_of(nnz ? nnz : 1), ids(nnz ? nnz : 1), col_s(nnz ? nnz : 1), perm(nnz ? nnz : 1);
    row_of_kernel<<<grid_for(A.n), kBlock, 0, s>>>(A.ptr.get(), A.n, row_of.get()); count_launch();
    iota_kernel<<<grid_for(nnz), kBlock, 0, s>>>(ids.get(), nnz); count_launch();
    sort_pairs(A.col.get(), col_s.get(), ids.get(), perm.get(), nnz, bits_for(A.ncol), s);
    T.ptr.resize(T.n + 1);
    segment_starts_kernel<<<grid_for(T.n + 1), kBlock, 0, s>>>(col_s.get(), nnz, T.n, T.ptr.get()); count_launch();
    T.col.resize(nnz ? nnz : 1);
    T.val.resize(nnz ? nnz : 1);
    gather_int_kernel<<<grid_for(nnz), kBlock, 0, s>>>(row_of.get(), perm.get(), nnz, T.col.get()); count_launch();
    gather_kernel<<<grid_for(nnz), kBlock, 0, s>>>(A.val.get(), perm.get(), nnz, T.val.get()); count_launch();
    CUNIBS_LAUNCH_CHECK("transpose");
}

void l1_dinv(const DevCsr<double>& a, DevArray<double>& dinv, cudaStream_t s) {
    dinv.resize(a.n);
    l1_dinv_kernel<<<grid_for(a.n), kBlock, 0, s>>>(a.ptr.get(), a.col.get(), a.val.get(), a.n, dinv.get()); count_launch();
    CUNIBS_LAUNCH_CHECK("l1 dinv");
}

int choose_tpr(int n_rows, long nnz) {
    if (n_rows <= 0) return 1;
    // Rows alone fill the GPU here; splitting them only adds combine work (measured on the finest
    // level of the 1M-tet head: 22 us per pass at one lane per row against 35 us at two).
    if (n_rows >= 65536) return 1;
    const double per = static_cast<double>(nnz) / n_rows;
    int t = 1;
    while (t < 32 && per / t > 8.0) t *= 2;
    return t;
}

Cheby make_cheby(int degree, double lower_ratio) {
    if (degree < 1 || degree > 8) fail(kEInval, "Chebyshev degree must be in [1, 8]");
    if (!(lower_ratio > 1.0)) fail(kEInval, "Chebyshev lower_ratio must exceed 1");
    Cheby c;
    const double hi = 1.0, lo = hi / lower_ratio;
    const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo);
    const double sigma = theta / delta;
    c.alpha0 = 1.0 / theta;
    double rho = 1.0 / sigma;
    for (int j = 0; j + 1 < degree; ++j) {
        const double rho_next = 1.0 / (2.0 * sigma - rho);
        const double beta = rho_next * rho;
        c.c_cur[j] = 1.0 + beta;
        c.c_prev[j] = -beta;
        c.alpha[j] = 2.0 * rho_next / delta;
        rho = rho_next;
    }
    c.degree = degree;
    return c;
}

// inv (and its FP32 copy) = the dense inverse of the SPD operator a, through a Cholesky factorisation.
static void dense_inverse(const DevCsr<double>& a, DevArray<double>& inv, DevArray<float>& inv32, const char* what,
                   cudaStream_t s) {
    const int n = a.n;
    DevArray<double> dense(static_cast<std::size_t>(n) * n), y(static_cast<std::size_t>(n) * n);
    dense.zero(s);
    densify_kernel<<<grid_for(n), kBlock, 0, s>>>(a.ptr.get(), a.col.get(), a.val.get(), n, dense.get());
    count_launch();
    DevArray<int> status(1);
    cholesky_kernel<<<1, 1024, 0, s>>>(dense.get(), n, status.get()); count_launch();
    if (read_scalar(status.get(), s)) fail(kEInternal, std::string(what) + " is not positive definite");
    inv.resize(static_cast<std::size_t>(n) * n);
    cholesky_inverse_kernel<<<grid_for(n, 64), 64, 0, s>>>(dense.get(), n, y.get(), inv.get()); count_launch();
    to_f32(inv, static_cast<long>(n) * n, inv32, s);
    CUNIBS_LAUNCH_CHECK("dense inverse");
    CUNIBS_CHECK(cudaStreamSynchronize(s));
}

// The finest level's smoother weights and FP32 copies after new values were written into it (the
// same pattern: conductivity changes only values); every coarser level, prolongator and the dense
// bottom are kept.
void refresh_finest_derived(Hierarchy& h, cudaStream_t s) {
    Level& L = h.levels[0];
    l1_dinv(L.a, L.dinv, s);
    to_f32(L.a.val, L.a.nnz, L.a32, s);
    to_f32(L.dinv, L.n, L.dinv32, s);
    CUNIBS_LAUNCH_CHECK("refresh finest level");
}

void build_hierarchy(Hierarchy& h, DevCsr<double>& a0, const Params& prm, cudaStream_t s) {
    h.levels.clear();
    h.sizes.assign(1, a0.n);
    h.cheby = make_cheby(prm.cheby_degree, prm.cheby_lower_ratio);
    DevCsr<double> a = std::move(a0);
    for (int lev = 0; lev < prm.max_levels; ++lev) {
        if (a.n <= prm.min_coarse_rows) break;
        DevArray<int> agg;
        const int nc = aggregate_level(a, prm, agg, s);
        if (nc < 0 || nc == a.n || nc < prm.min_coarse_rows) break;
        Level L;
        L.n = a.n;
        L.n_coarse = nc;
        l1_dinv(a, L.dinv, s);
        DevCsr<double> pt;
        tentative(agg, a.n, nc, pt, s);
        spgemm(a, pt, L.p, s);
        smooth_prolongator_kernel<<<grid_for(a.n), kBlock, 0, s>>>(L.p.ptr.get(), L.p.col.get(), L.p.val.get(),
                                                                   agg.get(), pt.val.get(), L.dinv.get(), a.n); count_launch();
        CUNIBS_LAUNCH_CHECK("smooth prolongator");
        transpose(L.p, L.r, s);
        DevCsr<double> next;
        DevCsr<double> ap;
        spgemm(a, L.p, ap, s);
        spgemm(L.r, ap, next, s);
        L.agg = std::move(agg);
        L.a = std::move(a);
        to_f32(L.a.val, L.a.nnz, L.a32, s);
        to_f32(L.dinv, L.n, L.dinv32, s);
        to_f32(L.p.val, L.p.nnz, L.p32, s);
        to_f32(L.r.val, L.r.nnz, L.r32, s);
        L.tpr_a = choose_tpr(L.n, L.a.nnz);
        L.tpr_p = choose_tpr(L.n, L.p.nnz);
        L.tpr_r = choose_tpr(L.n_coarse, L.r.nnz);
        h.levels.push_back(std::move(L));
        a = std::move(next);
        h.sizes.push_back(a.n);
    }
    h.nc = a.n;
    h.coarse = std::move(a);
    dense_inverse(h.coarse, h.coarse_inv, h.coarse_inv32, "coarsest AMG operator", s);
    // The V-cycle's bottom: the first level below the finest small enough for a dense solve. Its
    // exact inverse replaces the smoothing, restriction and prolongation of every level under it
    // (a few latency-bound launches each per V-cycle) with one dense product.
    h.vcycle_levels = static_cast<int>(h.levels.size());
    h.bottom_n = h.nc;
    for (int l = 1; l < static_cast<int>(h.levels.size()); ++l) {
        if (prm.dense_max_rows > 0 && h.levels[l].n <= prm.dense_max_rows) {
            h.vcycle_levels = l;
            h.bottom_n = h.levels[l].n;
            dense_inverse(h.levels[l].a, h.level_inv, h.level_inv32, "AMG level operator", s);
            break;
        }
    }
    CUNIBS_CHECK(cudaStreamSynchronize(s));
}

}  // namespace cunibs
