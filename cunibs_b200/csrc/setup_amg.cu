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
//
// The matching rules are the AMGx SIZE_4 selector's as the reference applies them (aggregate.cu):
// edge weight |a_ij| / max(|a_ii|, |a_jj|) perturbed by a hash of the unordered pair; round 1
// pairs rows with their strongest unpaired neighbour on a mutual choice, round 2 merges pairs
// into quads the same way, leftovers join their strongest aggregated neighbour, and labels are
// renumbered in order. What is this project's own is how it runs on the GPU:
//
// * Edge keys. Every CSR entry carries one 64-bit key, (bits of its weight) << 32 | (column + 1),
//   or 0 when the entry can never be chosen (the diagonal, a column outside the level, a NaN
//   weight). Weights are >= 0, whose IEEE bit patterns order like the values, so "strongest
//   neighbour, highest column on equal weight" is the plain maximum of the eligible keys, and
//   key 0 is "no neighbour". A scan reads one word per entry.
// * Group-per-row scans. G lanes (G from the level's mean row length) stride over a row's keys
//   and combine their maxima with shuffles; the maximum of a set does not depend on the order it
//   is taken in, so the result equals a sequential fold over the row.
// * Device-side loop control. Each matching round is queued as its full schedule of iterations
//   up front. The last block of an iteration's final kernel (ticket counter) adds up the rows
//   left unmatched and sets the round's `done` word when the round's exit rule holds; every
//   later kernel of the round reads `done` first and returns at once. The host waits only once,
//   for the number of aggregates.

// One step of the hash: x = (x op c) + (x shift s), op add or xor, shift left or right.
struct HashStep {
    bool use_xor;
    unsigned c;
    bool left;
    int shift;
};

// Robert Jenkins' 32-bit integer hash (six add/xor-shift steps), seeded by xor: the perturbation
// AMGx applies to edge weights, which the bit-exact partition requires as is.
__device__ __forceinline__ unsigned pair_hash(unsigned lo, unsigned hi) {
    constexpr HashStep steps[6] = {{false, 0x7ed55d16u, true, 12}, {true, 0xc761c23cu, false, 19},
                                   {false, 0x165667b1u, true, 5},  {true, 0xd3a2646cu, true, 9},
                                   {false, 0xfd7046c5u, true, 3},  {true, 0xb55a4f09u, false, 16}};
    unsigned x = lo ^ hi;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const unsigned mixed = steps[k].use_xor ? (x ^ steps[k].c) : (x + steps[k].c);
        x = mixed + (steps[k].left ? (x << steps[k].shift) : (x >> steps[k].shift));
    }
    return x;
}

__device__ __forceinline__ unsigned long long edge_key(float w, int col) {
    return (static_cast<unsigned long long>(__float_as_uint(w)) << 32) | static_cast<unsigned>(col + 1);
}
__device__ __forceinline__ int key_col(unsigned long long k) { return static_cast<int>(k & 0xffffffffu) - 1; }
__device__ __forceinline__ float key_weight(unsigned long long k) { return __uint_as_float(static_cast<unsigned>(k >> 32)); }

// The lanes of this thread's row group (G consecutive lanes; the groups tile the warp). A group
// leaves or stays as a whole, so its mask names exactly the lanes that take part.
template <int G>
__device__ __forceinline__ unsigned group_mask() {
    if constexpr (G == 32) {
        return 0xffffffffu;
    } else {
        return ((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1));
    }
}

// Maximum over the G lanes of a row group.
template <int G>
__device__ __forceinline__ unsigned long long group_max(unsigned long long v) {
    const unsigned m = group_mask<G>();
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
        const unsigned long long u = __shfl_xor_sync(m, v, o, G);
        v = u > v ? u : v;
    }
    return v;
}

// Loop control shared by the kernels of one matching round.
struct MatchCtl {
    int unmatched;  // rows left unmatched by the current iteration (summed by its blocks)
    int arrived;    // blocks of the current iteration's final kernel that have added their count
    int previous;   // rows left unmatched by the previous iteration (n before the first)
    int done;       // 1 once the round's exit rule held
};

// Which rule ends a round: round 1 stops when every row is paired or an iteration pairs none;
// round 2 also stops once fewer than 5% of the rows are left.
enum class ExitRule { kPairs, kQuads };

// Called by every thread of a block of a round's final kernel, `left` its row's "still unmatched".
template <ExitRule R>
__device__ void close_iteration(int left, int n, MatchCtl* ctl) {
    __shared__ int block_left;
    __shared__ bool last;
    if (threadIdx.x == 0) block_left = 0;
    __syncthreads();
    if (left) atomicAdd(&block_left, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (block_left) atomicAdd(&ctl->unmatched, block_left);
        __threadfence();
        last = atomicAdd(&ctl->arrived, 1) == static_cast<int>(gridDim.x) - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        const int now = atomicAdd(&ctl->unmatched, 0);
        bool stop = now == 0 || now == ctl->previous;
        if (R == ExitRule::kQuads) stop = stop || static_cast<float>(now) / static_cast<float>(n) < 0.05f;
        ctl->previous = now;
        ctl->unmatched = 0;
        ctl->arrived = 0;
        if (stop) ctl->done = 1;
    }
}

__global__ void match_ctl_reset_kernel(MatchCtl* ctl, int n) {
    ctl->unmatched = 0;
    ctl->arrived = 0;
    ctl->previous = n;
    ctl->done = 0;
}

// |diagonal| of every row (0 when the row stores none): the first diagonal entry the row holds.
template <int G>
__global__ void row_diag_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                const float* __restrict__ va, float* __restrict__ adiag) {
    const int lane = threadIdx.x % G;
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    const unsigned gmask = group_mask<G>();
    if (row >= n) return;  // whole groups leave together (n rows x G lanes)
    float d = 0.0f;
    for (int base = rp[row]; base < rp[row + 1]; base += G) {
        const int j = base + lane;
        const bool hit = j < rp[row + 1] && ci[j] == row;
        const unsigned m = __ballot_sync(gmask, hit) & gmask;
        if (m) {
            const int first = __ffs(m) - 1;  // lowest lane: the first such entry of the row
            d = __shfl_sync(gmask, hit ? va[j] : 0.0f, first & (G - 1), G);
            break;
        }
    }
    if (lane == 0) adiag[row] = fabsf(d);
}

// The edge keys of every entry of a row.
__global__ void edge_keys_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                 const float* __restrict__ va, const float* __restrict__ adiag,
                                 unsigned long long* __restrict__ key) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    const float di = adiag[row];
    for (int j = rp[row]; j < rp[row + 1]; ++j) {
        const int c = ci[j];
        unsigned long long k = 0;
        if (c != row && static_cast<unsigned>(c) < static_cast<unsigned>(n)) {
            const float ed = fabsf(va[j]) / fmaxf(di, adiag[c]);
            const unsigned h = pair_hash(static_cast<unsigned>(min(row, c)), static_cast<unsigned>(max(row, c)));
            const float frac = 1e-5f * static_cast<float>(h) / 4294967295.0f;
            const float w = __fmaf_rn(frac, ed, ed);
            if (!(w != w)) k = edge_key(w, c);  // a NaN weight never wins
        }
        key[j] = k;
    }
}

__global__ void match_init_kernel(int n, int* __restrict__ agg, int* __restrict__ partner, int* __restrict__ choice) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    agg[t] = t;
    partner[t] = -1;
    choice[t] = -1;
}

// Round 1, propose: an unpaired row names its strongest unpaired neighbour. A row that sees none
// keeps its earlier proposal (the reference's behaviour, which gives a coarser hierarchy).
template <int G>
__global__ void pair_propose_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                    const unsigned long long* __restrict__ key, const int* __restrict__ partner,
                                    int* __restrict__ choice, const MatchCtl* __restrict__ ctl) {
    if (ctl->done) return;
    const int lane = threadIdx.x % G;
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    if (row >= n || partner[row] != -1) return;  // whole groups leave together
    unsigned long long best = 0;
    for (int j = rp[row] + lane; j < rp[row + 1]; j += G) {
        const unsigned long long k = key[j];
        if (k > best && partner[key_col(k)] == -1) best = k;
    }
    best = group_max<G>(best);
    if (lane == 0 && best) choice[row] = key_col(best);
}

// Round 1, accept: two rows that named each other become a pair labelled by the smaller index.
__global__ void pair_accept_kernel(int n, int* __restrict__ partner, int* __restrict__ agg,
                                   const int* __restrict__ choice, MatchCtl* __restrict__ ctl) {
    if (ctl->done) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    int left = 0;
    if (t < n && partner[t] == -1) {
        const int c = choice[t];
        if (c != -1 && choice[c] == t) {
            partner[t] = c;
            agg[t] = min(t, c);
        } else {
            left = 1;
        }
    }
    close_iteration<ExitRule::kPairs>(left, n, ctl);
}

// Between the rounds: unpaired rows pair with themselves; nothing is merged yet.
__global__ void quad_init_kernel(int n, int* __restrict__ partner, float* __restrict__ offer,
                                 int* __restrict__ merged) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    if (partner[t] == -1) partner[t] = t;
    offer[t] = -1.0f;
    merged[t] = -1;
}

// Round 2, propose: a row of an unmerged pair names the pair of its strongest unmerged neighbour
// outside its own pair, and records that edge's weight as its offer.
template <int G>
__global__ void quad_propose_kernel(int n, const int* __restrict__ rp, const unsigned long long* __restrict__ key,
                                    const int* __restrict__ merged, const int* __restrict__ agg,
                                    const int* __restrict__ partner, int* __restrict__ choice,
                                    float* __restrict__ offer, const MatchCtl* __restrict__ ctl) {
    if (ctl->done) return;
    const int lane = threadIdx.x % G;
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    if (row >= n || merged[row] != -1) return;  // whole groups leave together
    const int mate = partner[row];
    unsigned long long best = 0;
    for (int j = rp[row] + lane; j < rp[row + 1]; j += G) {
        const unsigned long long k = key[j];
        if (k <= best) continue;
        const int c = key_col(k);
        if (c != mate && merged[c] == -1) best = k;
    }
    best = group_max<G>(best);
    if (lane == 0 && best) {
        offer[row] = key_weight(best);
        choice[row] = agg[key_col(best)];
    }
}

// Round 2, settle: the two rows of a pair adopt the stronger of their two proposals; a pair whose
// rows both have no offer stops here as a pair. A row reads its mate's choice only when the
// mate's offer is strictly stronger, and then the mate writes nothing, so no read races a write.
__global__ void quad_settle_kernel(int n, int* __restrict__ merged, int* __restrict__ choice,
                                   const float* __restrict__ offer, const int* __restrict__ partner,
                                   const MatchCtl* __restrict__ ctl) {
    if (ctl->done) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || merged[t] != -1) return;
    const int mate = partner[t];
    const float own = offer[t];
    const float other = mate != -1 ? offer[mate] : -1.0f;
    if (own < 0.0f && other < 0.0f) {
        merged[t] = 1;
        choice[t] = -1;
    } else if (own < other) {
        choice[t] = choice[mate];
    }
}

// Round 2, accept: two pairs that named each other merge, labelled by the smaller label.
__global__ void quad_accept_kernel(int n, int* __restrict__ agg, int* __restrict__ merged,
                                   const int* __restrict__ choice, MatchCtl* __restrict__ ctl) {
    if (ctl->done) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    int left = 0;
    if (t < n && merged[t] == -1) {
        const int c = choice[t];
        const int label = agg[t];
        if (c != -1 && choice[c] == label) {
            merged[t] = 1;
            agg[t] = min(c, label);
        } else {
            left = 1;
        }
    }
    close_iteration<ExitRule::kQuads>(left, n, ctl);
}

// Leftovers (rows still unmerged when round 2 ended): each picks the label of its strongest merged
// neighbour, or its own index when it has none; the picks are applied in a second kernel so every
// row sees the same merged set.
template <int G>
__global__ void leftover_pick_kernel(int n, const int* __restrict__ rp, const unsigned long long* __restrict__ key,
                                     const int* __restrict__ agg, const int* __restrict__ merged,
                                     int* __restrict__ pick) {
    const int lane = threadIdx.x % G;
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    if (row >= n || merged[row] != -1) return;  // whole groups leave together
    unsigned long long best = 0;
    for (int j = rp[row] + lane; j < rp[row + 1]; j += G) {
        const unsigned long long k = key[j];
        if (k > best && merged[key_col(k)] != -1) best = k;
    }
    best = group_max<G>(best);
    if (lane == 0) pick[row] = best ? agg[key_col(best)] : row;
}

__global__ void leftover_apply_kernel(int n, int* __restrict__ agg, int* __restrict__ merged,
                                      const int* __restrict__ pick) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n && merged[t] == -1) {
        agg[t] = pick[t];
        merged[t] = 1;
    }
}

// Labels in use, then each row's label replaced by the number of used labels below it.
__global__ void label_used_kernel(int n, const int* __restrict__ agg, int* __restrict__ used) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) used[agg[t]] = 1;
}

__global__ void label_renumber_kernel(int n, int* __restrict__ agg, const int* __restrict__ below) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) agg[t] = below[agg[t]];
}

// Lanes per row of the scanning kernels, from the level's mean row length.
int group_lanes(int n, long nnz) {
    const double per = n > 0 ? static_cast<double>(nnz) / n : 0.0;
    return per <= 12.0 ? 4 : per <= 24.0 ? 8 : per <= 48.0 ? 16 : 32;
}

unsigned group_grid(int n, int G) {
    const long threads = static_cast<long>(n) * G;
    return static_cast<unsigned>((threads + kBlock - 1) / kBlock);
}

// Runs the whole selection on `s` and returns the number of aggregates (the one host wait).
template <int G>
int run_matching(int n, long nnz, const int* rp, const int* ci, const float* va, int* agg, cudaStream_t s) {
    constexpr int kMaxIterations = 16;  // per round, as the reference's selector
    const unsigned rows = grid_for(n), groups = group_grid(n, G);
    DevArray<float> adiag(n), offer(n);
    DevArray<unsigned long long> key(nnz > 0 ? nnz : 1);
    DevArray<int> partner(n), choice(n), merged(n), pick(n), used(n + 1), below(n + 1);
    DevArray<MatchCtl> ctl(1);
    row_diag_kernel<G><<<groups, kBlock, 0, s>>>(n, rp, ci, va, adiag.get()); count_launch();
    edge_keys_kernel<<<rows, kBlock, 0, s>>>(n, rp, ci, va, adiag.get(), key.get()); count_launch();
    match_init_kernel<<<rows, kBlock, 0, s>>>(n, agg, partner.get(), choice.get()); count_launch();
    match_ctl_reset_kernel<<<1, 1, 0, s>>>(ctl.get(), n); count_launch();
    CUNIBS_LAUNCH_CHECK("aggregation set-up");
    for (int it = 0; it < kMaxIterations; ++it) {
        pair_propose_kernel<G><<<groups, kBlock, 0, s>>>(n, rp, ci, key.get(), partner.get(), choice.get(), ctl.get());
        pair_accept_kernel<<<rows, kBlock, 0, s>>>(n, partner.get(), agg, choice.get(), ctl.get());
        count_launch(2);
    }
    CUNIBS_LAUNCH_CHECK("aggregation pairs");
    quad_init_kernel<<<rows, kBlock, 0, s>>>(n, partner.get(), offer.get(), merged.get()); count_launch();
    match_ctl_reset_kernel<<<1, 1, 0, s>>>(ctl.get(), n); count_launch();
    for (int it = 0; it < kMaxIterations; ++it) {
        quad_propose_kernel<G><<<groups, kBlock, 0, s>>>(n, rp, key.get(), merged.get(), agg, partner.get(),
                                                          choice.get(), offer.get(), ctl.get());
        quad_settle_kernel<<<rows, kBlock, 0, s>>>(n, merged.get(), choice.get(), offer.get(), partner.get(), ctl.get());
        quad_accept_kernel<<<rows, kBlock, 0, s>>>(n, agg, merged.get(), choice.get(), ctl.get());
        count_launch(3);
    }
    CUNIBS_LAUNCH_CHECK("aggregation quads");
    // With no row left unmerged both kernels find nothing to do.
    leftover_pick_kernel<G><<<groups, kBlock, 0, s>>>(n, rp, key.get(), agg, merged.get(), pick.get());
    leftover_apply_kernel<<<rows, kBlock, 0, s>>>(n, agg, merged.get(), pick.get());
    count_launch(2);
    used.zero(s);
    label_used_kernel<<<rows, kBlock, 0, s>>>(n, agg, used.get()); count_launch();
    exclusive_scan(used.get(), below.get(), n + 1, s);
    label_renumber_kernel<<<rows, kBlock, 0, s>>>(n, agg, below.get()); count_launch();
    CUNIBS_LAUNCH_CHECK("aggregation labels");
    return read_scalar(below.get() + n, s);
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

// --- dense inverse of the V-cycle's bottom operator ----------------------------------------
//
// A blocked sweep (Gauss-Jordan elimination without pivoting, which an SPD matrix never needs) on
// the lower triangle of the matrix padded to a multiple of kSweepB with an identity block. Sweeping
// pivot block k with P = A_kk^-1 maps
//   A_kk -> -P,  A_ik -> C_i = A_ik P,  A_ij -> A_ij - C_i A_kj   (i, j != k),
// and after every block has been swept the matrix holds -A^-1. Only tiles on or below the block
// diagonal are stored and updated (A_kj for j > k is read as A_jk^T), so a step is one SYRK-shaped
// product of about n^2 kSweepB multiply-adds; the whole inverse costs n^3 of them, on every SM.

constexpr int kSweepB = 64;

__global__ void densify_lower_kernel(const int* __restrict__ ptr, const int* __restrict__ col,
                                     const double* __restrict__ val, int n, int N, double* __restrict__ m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    if (i >= n) {
        m[static_cast<long>(i) * N + i] = 1.0;  // identity padding
        return;
    }
    for (int p = ptr[i]; p < ptr[i + 1]; ++p) m[static_cast<long>(i) * N + col[p]] = val[p];
}

// Tile (I, J) of the symmetric matrix as stored (lower triangle): element (r, c) of the tile.
__device__ __forceinline__ double sym_tile(const double* __restrict__ m, int N, int I, int J, int r, int c) {
    const long row = static_cast<long>(I) * kSweepB + r, col = static_cast<long>(J) * kSweepB + c;
    return (I > J || (I == J && r >= c)) ? m[row * N + col] : m[col * N + row];
}

// acc (per thread a 4 x 4 patch of a 64 x 64 tile) = X (64 x 64, rows ldx apart) * Y (64 x 64, rows
// ldy apart); the reduction dimension in chunks of 32 staged (coalesced loads) in `stage`, a
// shared-memory buffer of kStageDoubles.
constexpr int kStageDoubles = kSweepB * 33 + 32 * kSweepB;

__device__ __forceinline__ void tile_product(const double* X, long ldx, const double* Y, long ldy, double acc[4][4],
                                             double* stage) {
    double (*xs)[33] = reinterpret_cast<double (*)[33]>(stage);
    double (*ys)[kSweepB] = reinterpret_cast<double (*)[kSweepB]>(stage + kSweepB * 33);
    const int t = threadIdx.x, ty = t / 16, tx = t % 16;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
    for (int k0 = 0; k0 < kSweepB; k0 += 32) {
        for (int q = t; q < kSweepB * 32; q += blockDim.x) {
            xs[q / 32][q % 32] = X[(q / 32) * ldx + k0 + q % 32];
            ys[q / kSweepB][q % kSweepB] = Y[(k0 + q / kSweepB) * ldy + q % kSweepB];
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < 32; ++kk) {
            double xa[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) xa[a] = xs[ty * 4 + a][kk];
            const double2 y0 = *reinterpret_cast<const double2*>(&ys[kk][tx * 4]);
            const double2 y1 = *reinterpret_cast<const double2*>(&ys[kk][tx * 4 + 2]);
            const double yb[4] = {y0.x, y0.y, y1.x, y1.y};
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] = fma(xa[a], yb[b], acc[a][b]);
        }
        __syncthreads();
    }
}

// P = A_kk^-1 of the current pivot block, by a scalar sweep of its 64 pivots in shared memory
// (which leaves -A_kk^-1). status = 1 when a pivot is not positive (not SPD).
__global__ void __launch_bounds__(256) sweep_pivot_kernel(const double* __restrict__ m, int N, int k,
                                                          double* __restrict__ pinv, int* __restrict__ status) {
    __shared__ double b[kSweepB][kSweepB + 1];
    __shared__ double dsh;
    for (int q = threadIdx.x; q < kSweepB * kSweepB; q += blockDim.x)
        b[q / kSweepB][q % kSweepB] = sym_tile(m, N, k, k, q / kSweepB, q % kSweepB);
    __syncthreads();
    for (int p = 0; p < kSweepB; ++p) {
        if (threadIdx.x == 0) {
            double d = b[p][p];
            if (!(d > 0.0)) {
                *status = 1;
                d = 1.0;
            }
            dsh = d;
        }
        __syncthreads();
        const double d = dsh;
        for (int q = threadIdx.x; q < kSweepB * kSweepB; q += blockDim.x) {
            const int i = q / kSweepB, j = q % kSweepB;
            if (i != p && j != p) b[i][j] -= b[i][p] * b[p][j] / d;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < kSweepB; i += blockDim.x) {
            if (i != p) {
                b[i][p] /= d;
                b[p][i] /= d;
            }
        }
        if (threadIdx.x == 0) b[p][p] = -1.0 / d;
        __syncthreads();
    }
    // P is symmetric; its two rounded halves are averaged so that it is so exactly.
    for (int q = threadIdx.x; q < kSweepB * kSweepB; q += blockDim.x) {
        const int i = q / kSweepB, j = q % kSweepB;
        pinv[q] = -0.5 * (b[i][j] + b[j][i]);
    }
}

// For every block row I != k (blockIdx.x = I): the old row panel rbuf[:, I] = A_kI (64 x N, rows N
// apart) and C_I = A_Ik P into cbuf (N x 64), formed as C_I^T = P A_kI (P is symmetric).
__global__ void __launch_bounds__(256) sweep_panel_kernel(const double* __restrict__ m, int N, int k,
                                                          const double* __restrict__ pinv, double* __restrict__ cbuf,
                                                          double* __restrict__ rbuf) {
    __shared__ __align__(16) double buf[kStageDoubles];
    static_assert(kStageDoubles >= kSweepB * (kSweepB + 1), "the staging buffer holds one padded tile");
    double (*tile)[kSweepB + 1] = reinterpret_cast<double (*)[kSweepB + 1]>(buf);  // A_kI
    const int I = blockIdx.x;
    if (I == k) return;
    for (int q = threadIdx.x; q < kSweepB * kSweepB; q += blockDim.x) {
        // Read along the stored rows: A_kI itself above the diagonal block, A_Ik below it.
        if (I < k) {
            const int r = q / kSweepB, c = q % kSweepB;
            tile[r][c] = m[(static_cast<long>(k) * kSweepB + r) * N + static_cast<long>(I) * kSweepB + c];
        } else {
            const int c = q / kSweepB, r = q % kSweepB;
            tile[r][c] = m[(static_cast<long>(I) * kSweepB + c) * N + static_cast<long>(k) * kSweepB + r];
        }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < kSweepB * kSweepB; q += blockDim.x) {
        const int r = q / kSweepB, c = q % kSweepB;
        rbuf[static_cast<long>(r) * N + static_cast<long>(I) * kSweepB + c] = tile[r][c];
    }
    __syncthreads();
    double acc[4][4];
    tile_product(pinv, kSweepB, rbuf + static_cast<long>(I) * kSweepB, N, acc, buf);
    const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
            cbuf[(static_cast<long>(I) * kSweepB + tx * 4 + b) * kSweepB + ty * 4 + a] = acc[a][b];
}

// A_IJ -= C_I A_kJ for the stored tiles I >= J with I, J != k (blockIdx = (J, I)).
__global__ void __launch_bounds__(256) sweep_update_kernel(double* __restrict__ m, int N, int k,
                                                           const double* __restrict__ cbuf,
                                                           const double* __restrict__ rbuf) {
    __shared__ __align__(16) double buf[kStageDoubles];
    const int J = blockIdx.x, I = blockIdx.y;
    if (I < J || I == k || J == k) return;
    double acc[4][4];
    tile_product(cbuf + static_cast<long>(I) * kSweepB * kSweepB, kSweepB, rbuf + static_cast<long>(J) * kSweepB, N,
                 acc, buf);
    const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        double* row = m + (static_cast<long>(I) * kSweepB + ty * 4 + a) * N + static_cast<long>(J) * kSweepB + tx * 4;
        double2 v0 = *reinterpret_cast<double2*>(row), v1 = *reinterpret_cast<double2*>(row + 2);
        v0.x -= acc[a][0];
        v0.y -= acc[a][1];
        v1.x -= acc[a][2];
        v1.y -= acc[a][3];
        *reinterpret_cast<double2*>(row) = v0;
        *reinterpret_cast<double2*>(row + 2) = v1;
    }
}

// The swept pivot row and column: A_Ik = C_I (stored as A_kI = C_I^T above the diagonal), A_kk = -P.
__global__ void __launch_bounds__(256) sweep_finish_kernel(double* __restrict__ m, int N, int k,
                                                           const double* __restrict__ pinv,
                                                           const double* __restrict__ cbuf) {
    const int I = blockIdx.x;
    for (int q = threadIdx.x; q < kSweepB * kSweepB; q += blockDim.x) {
        const int r = q / kSweepB, c = q % kSweepB;
        if (I == k) {
            m[(static_cast<long>(k) * kSweepB + r) * N + static_cast<long>(k) * kSweepB + c] = -pinv[q];
        } else if (I > k) {
            m[(static_cast<long>(I) * kSweepB + r) * N + static_cast<long>(k) * kSweepB + c] =
                cbuf[(static_cast<long>(I) * kSweepB + r) * kSweepB + c];
        } else {
            m[(static_cast<long>(k) * kSweepB + c) * N + static_cast<long>(I) * kSweepB + r] =
                cbuf[(static_cast<long>(I) * kSweepB + r) * kSweepB + c];
        }
    }
}

// inv = A^-1 (n x n, rows of ld entries, zero past column n) and its FP32 copy, from the swept
// lower triangle (-A^-1).
__global__ void sweep_extract_kernel(const double* __restrict__ m, int N, int n, int ld, double* __restrict__ inv,
                                     float* __restrict__ inv32) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<long>(n) * ld) return;
    const int i = static_cast<int>(q / ld), j = static_cast<int>(q % ld);
    const double v = j < n ? -m[static_cast<long>(i >= j ? i : j) * N + (i >= j ? j : i)] : 0.0;
    inv[q] = v;
    inv32[q] = static_cast<float>(v);
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
        const int nc = select_size4(cur->n, cur->nnz, cur->ptr.get(), cur->col.get(), v32.get(), step.get(), s);
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

int select_size4(int n, long nnz, const int* rp, const int* ci, const float* va, int* agg, cudaStream_t s) {
    if (n <= 0) return 0;
    switch (group_lanes(n, nnz)) {
        case 4: return run_matching<4>(n, nnz, rp, ci, va, agg, s);
        case 8: return run_matching<8>(n, nnz, rp, ci, va, agg, s);
        case 16: return run_matching<16>(n, nnz, rp, ci, va, agg, s);
        default: return run_matching<32>(n, nnz, rp, ci, va, agg, s);
    }
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
    // About sixteen entries per sub-lane (two batches of eight loads in flight): measured on the
    // 1M-tet head's level 1 (10k rows of 57 entries, 4 sub-lanes) and restriction (8 sub-lanes),
    // split solve stage 3.87 ms per block of 8 against 4.01 ms at eight entries and 4.05 at 32.
    while (t < 32 && per / t > 16.0) t *= 2;
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

// inv (and its FP32 copy) = the dense inverse of the SPD operator a, by the blocked sweep; rows of
// dense_ld(a.n) entries.
static void dense_inverse(const DevCsr<double>& a, DevArray<double>& inv, DevArray<float>& inv32, const char* what,
                          cudaStream_t s) {
    const int n = a.n;
    const int T = (n + kSweepB - 1) / kSweepB;
    const int N = T * kSweepB;
    DevArray<double> m(static_cast<std::size_t>(N) * N), pinv(kSweepB * kSweepB),
        cbuf(static_cast<std::size_t>(N) * kSweepB), rbuf(static_cast<std::size_t>(N) * kSweepB);
    m.zero(s);
    densify_lower_kernel<<<grid_for(N), kBlock, 0, s>>>(a.ptr.get(), a.col.get(), a.val.get(), n, N, m.get());
    count_launch();
    DevArray<int> status(1);
    status.zero(s);
    for (int k = 0; k < T; ++k) {
        sweep_pivot_kernel<<<1, 256, 0, s>>>(m.get(), N, k, pinv.get(), status.get());
        sweep_panel_kernel<<<T, 256, 0, s>>>(m.get(), N, k, pinv.get(), cbuf.get(), rbuf.get());
        sweep_update_kernel<<<dim3(T, T), 256, 0, s>>>(m.get(), N, k, cbuf.get(), rbuf.get());
        sweep_finish_kernel<<<T, 256, 0, s>>>(m.get(), N, k, pinv.get(), cbuf.get());
        count_launch(4);
    }
    CUNIBS_LAUNCH_CHECK("dense inverse");
    if (read_scalar(status.get(), s)) fail(kEInternal, std::string(what) + " is not positive definite");
    const int ld = dense_ld(n);
    inv.resize(static_cast<std::size_t>(n) * ld);
    inv32.resize(static_cast<std::size_t>(n) * ld);
    sweep_extract_kernel<<<grid_for(static_cast<std::int64_t>(n) * ld), kBlock, 0, s>>>(m.get(), N, n, ld, inv.get(),
                                                                                      inv32.get());
    count_launch();
    CUNIBS_LAUNCH_CHECK("dense inverse extract");
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
