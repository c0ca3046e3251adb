// Post-processing of a solved block: E = -grad v - dA/dt per tetrahedron, the potential on the full
// node set, and the gray-matter summary metrics.
//
// Reference behaviour restated: reconstruct.cu:36-76 (FP64 accumulation of grad v, FP32 output),
// fem/solve.py:939-941 (grounded node carries v = 0), metrics.py:58-243 (volume-weighted
// peak/location, centre of gravity, mean/std, p50/p95/p99/p99.9 at midpoint positions with linear
// interpolation, focality at 0.5 and 0.75 of p99.9). The reference sorts each placement's
// gray-matter |E| (stable) and prefix-sums the sorted volumes; here the percentiles come from a
// weighted radix select over the same order (below), with exact fixed-point volume sums, so the
// ranks are integer-exact and every metric reproduces run to run.
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

// --- gray-matter percentiles by weighted radix select -----------------------------------------
//
// Order: gray-matter element i of a placement has the key (bits(|E|) << 32) | i. |E| >= 0, so its
// IEEE bits order like its value, and equal values keep element order: the order of the
// reference's stable sort. Weights: each element's FP32 volume as an int64 fixed-point number
// (one power-of-two scale per mesh, chosen so the total stays below 2^52), so every sum of weights
// is exact, needs no fixed order and is the same run to run.
//
// With B_e the weight ordered before e and W the total, the weighted quantile at q interpolates
// linearly between the two elements whose midpoint positions pos = (B + w/2) / W bracket q
// (numpy.interp). That needs only the element e whose weight interval [B_e, B_e + w_e) holds
// T = q W and its neighbour on q's side. e's value is found by a radix descent over the 32 value
// bits (11, 11, 10 bits per level, one launch each): every block histograms (count, weight) of its
// elements inside the current range in shared memory (lanes of a warp on one bucket add together)
// and adds the non-empty buckets to integer counters; the last block of each placement scans them
// and narrows the range to the bucket that holds T. Then one pass gathers each range's keys (at
// most kCand of them) and, by integer max/min, the range's first and last key and the nearest keys
// on either side of it; one block per quantile finds e by counting (each candidate's B is the
// weight of the smaller keys). A range that still holds more than kCand elements after the last
// level is one value repeated (ties): there only its first and last element can bracket q with an
// element outside it, and every other bracket interpolates between two equal values.

constexpr int kQ = 4;  // p50, p95, p99, p99.9 (focality is measured against p99.9)
constexpr int kSelBuckets = 2048;
constexpr int kSelLevels = 3;  // 11 + 11 + 10 bits of |E|
constexpr int kCand = 512;
constexpr int kSelThreads = 256;
constexpr int kResolveThreads = kCand;

__host__ __device__ constexpr int level_width(int level) { return level == 2 ? 10 : 11; }

// q as the reference passes it: FP32 constants widened.
__device__ __forceinline__ double sel_q(int q) {
    return q == 0 ? static_cast<double>(0.5f) : q == 1 ? static_cast<double>(0.95f)
         : q == 2 ? static_cast<double>(0.99f) : static_cast<double>(0.999f);
}

struct SelState {
    unsigned long long prefix;  // key bits above `shift` that every key of the range shares
    long long before;           // weight of the elements ordered below the range
    long long weight;           // weight of the range
    int shift;                  // key bits below the prefix (64: the whole key space)
    int count;                  // elements in the range
    int phase;                  // 0 narrowing, 1 settled (gather, resolve)
    int pad;
};

// The range's extremes and its outside neighbours, found by the gather pass.
struct SelEdges {
    unsigned long long first;  // smallest key in the range
    unsigned long long last;   // largest key in the range
    unsigned long long pred;   // largest key below the range, plus one (0: none)
    unsigned long long succ;   // smallest key above the range (~0: none)
};

// Shared per-mesh quantities of the fixed-point weights.
struct SelMesh {
    unsigned wmax_bits;  // largest gray-matter FP32 volume, as bits
    int exp2;            // weight = volume * 2^exp2 (rounded to the nearest integer)
    long long total;     // sum of the weights
};

__device__ __forceinline__ bool in_range(unsigned long long key, const SelState& st) {
    return st.shift >= 64 || (key >> st.shift) == st.prefix;
}

__device__ __forceinline__ unsigned long long sel_key(float v, int i) {
    return (static_cast<unsigned long long>(__float_as_uint(v)) << 32) | static_cast<unsigned>(i);
}

__global__ void gm_wmax_kernel(const float* __restrict__ vols32, const int* __restrict__ gm, int n_gm,
                               SelMesh* __restrict__ sm) {
    unsigned m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_gm; i += gridDim.x * blockDim.x)
        m = max(m, __float_as_uint(vols32[gm[i]]));
    m = __reduce_max_sync(0xffffffffu, m);
    if ((threadIdx.x & 31) == 0) atomicMax(&sm->wmax_bits, m);
}

__device__ __forceinline__ int sel_exp2(const SelMesh* sm, int n_gm) {
    // The largest volume lies in [2^e, 2^(e+1)); n_gm of them stay below 2^52 at 2^(51 - e - ceil(log2 n)).
    const int e = static_cast<int>((sm->wmax_bits >> 23) & 0xffu) - 127;
    const int lg = n_gm > 1 ? 32 - __clz(static_cast<unsigned>(n_gm - 1)) : 0;
    return 51 - e - lg;
}

__global__ void gm_wfix_kernel(const float* __restrict__ vols32, const int* __restrict__ gm, int n_gm,
                               SelMesh* __restrict__ sm, long long* __restrict__ wfix) {
    const int s = sel_exp2(sm, n_gm);
    long long part = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_gm; i += gridDim.x * blockDim.x) {
        const long long w = llrint(ldexp(static_cast<double>(vols32[gm[i]]), s));
        wfix[i] = w;
        part += w;
    }
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(reinterpret_cast<unsigned long long*>(&sm->total),
                                           static_cast<unsigned long long>(part));
    if (blockIdx.x == 0 && threadIdx.x == 0) sm->exp2 = s;
}

__global__ void sel_init_kernel(int k, int n_gm, const SelMesh* __restrict__ sm, SelState* __restrict__ st,
                                int* __restrict__ cand_n, SelEdges* __restrict__ edges, int* __restrict__ ticket,
                                long long* __restrict__ foc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < k * kQ) {
        SelState s0;
        s0.prefix = 0;
        s0.before = 0;
        s0.weight = sm->total;
        s0.shift = 64;
        s0.count = n_gm;
        s0.phase = n_gm <= kCand ? 1 : 0;
        s0.pad = 0;
        st[t] = s0;
        cand_n[t] = 0;
        edges[t] = SelEdges{~0ull, 0ull, 0ull, ~0ull};
    }
    if (t < k) ticket[t] = 0;
    if (t < 2 * k) foc[t] = 0;
}

// One narrowing level for every placement (blockIdx.y) and every quantile still narrowing. On
// the first level all quantiles share the whole key range, so one histogram serves them all, and
// the placement's gray-matter values are written out contiguously (gv) for the later passes.
__global__ void __launch_bounds__(kSelThreads) sel_level_kernel(
    int level, const float* __restrict__ magn, const int* __restrict__ gm, int n_gm, int n_tets,
    const long long* __restrict__ wfix, const SelMesh* __restrict__ sm, float* __restrict__ gv,
    SelState* __restrict__ states, unsigned* __restrict__ hcnt, unsigned long long* __restrict__ hw,
    int* __restrict__ ticket) {
    extern __shared__ unsigned char sel_smem[];
    // [slots][buckets] weights (8-byte aligned first), then [slots][buckets] counts.
    const int slots = level == 0 ? 1 : kQ;
    unsigned long long* sw = reinterpret_cast<unsigned long long*>(sel_smem);
    unsigned* scnt = reinterpret_cast<unsigned*>(sw + slots * kSelBuckets);
    __shared__ SelState st[kQ];
    __shared__ bool last;
    const int c = blockIdx.y;
    if (threadIdx.x < kQ) st[threadIdx.x] = states[c * kQ + threadIdx.x];
    __syncthreads();
    const bool first = level == 0;
    bool active[kQ];
    bool any = false;
#pragma unroll
    for (int q = 0; q < kQ; ++q) {
        active[q] = st[q].phase == 0;
        any = any || active[q];
    }
    if (!any && !first) return;  // every quantile has settled: nothing to do (all blocks agree)
    const int width = level_width(level);
    for (int b = threadIdx.x; b < slots * kSelBuckets; b += blockDim.x) {
        scnt[b] = 0;
        sw[b] = 0;
    }
    __syncthreads();
    const long chunk = (static_cast<long>(n_gm) + gridDim.x - 1) / gridDim.x;
    const int i0 = static_cast<int>(min(static_cast<long>(n_gm), blockIdx.x * chunk));
    const int i1 = static_cast<int>(min(static_cast<long>(n_gm), i0 + chunk));
    float* gvc = gv + static_cast<long>(c) * n_gm;
    const int lane = threadIdx.x & 31;
    // Whole warps walk the chunk together (i past the end is idle), so the warp-wide intrinsics
    // below always see all 32 lanes.
    for (int base = i0 + (threadIdx.x & ~31); base < i1; base += blockDim.x) {
        const int i = base + lane;
        const bool ok = i < i1;
        float v = 0.0f;
        if (ok) {
            if (first) {
                v = magn[static_cast<long>(c) * n_tets + gm[i]];
                gvc[i] = v;
            } else {
                v = gvc[i];
            }
        }
        if (!any) continue;
        const unsigned long long key = sel_key(v, i);
        int dig[kQ];
        bool hit = false;
#pragma unroll
        for (int q = 0; q < kQ; ++q) {
            dig[q] = -1;
            if (q < slots && ok && (first || (active[q] && in_range(key, st[q])))) {
                dig[q] = static_cast<int>((key >> (st[q].shift - width)) & ((1ull << width) - 1));
                hit = true;
            }
        }
        if (!first) {
            // Past the first level few elements fall in a range, and those spread over the range's
            // buckets: plain shared-memory atomics.
            if (!hit) continue;
            const unsigned long long w = static_cast<unsigned long long>(wfix[i]);
#pragma unroll
            for (int q = 0; q < kQ; ++q) {
                if (dig[q] < 0) continue;
                atomicAdd(&scnt[q * kSelBuckets + dig[q]], 1u);
                atomicAdd(&sw[q * kSelBuckets + dig[q]], w);
            }
            continue;
        }
        if (!__any_sync(0xffffffffu, hit)) continue;  // nothing of this warp's 32 is in a range
        const unsigned long long w = hit ? static_cast<unsigned long long>(wfix[i]) : 0ull;
#pragma unroll
        for (int q = 0; q < kQ; ++q) {
            if (q >= slots) break;
            const int d = dig[q];
            // Lanes on the same bucket add together: one shared-memory atomic per bucket per warp. A
            // weight is below 2^52, so its two 26-bit halves sum over 32 lanes without overflow.
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            if (d < 0) continue;
            const unsigned lo = __reduce_add_sync(peers, static_cast<unsigned>(w & 0x3ffffffull));
            const unsigned hi = __reduce_add_sync(peers, static_cast<unsigned>(w >> 26));
            if (lane == __ffs(peers) - 1) {
                atomicAdd(&scnt[q * kSelBuckets + d], static_cast<unsigned>(__popc(peers)));
                atomicAdd(&sw[q * kSelBuckets + d], (static_cast<unsigned long long>(hi) << 26) + lo);
            }
        }
    }
    if (!any) return;  // first level with nothing to narrow: the values are written, that is all
    __syncthreads();
    unsigned* gcnt = hcnt + static_cast<long>(c) * kQ * kSelBuckets;
    unsigned long long* gw = hw + static_cast<long>(c) * kQ * kSelBuckets;
    for (int b = threadIdx.x; b < slots * kSelBuckets; b += blockDim.x) {
        if (scnt[b]) {
            atomicAdd(&gcnt[b], scnt[b]);
            atomicAdd(&gw[b], sw[b]);
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&ticket[c], 1) == static_cast<int>(gridDim.x) - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    // The placement's last block: narrow each quantile's range to the bucket that holds T.
    constexpr int kPer = kSelBuckets / kSelThreads;
    __shared__ long long scan[kSelThreads];
    __shared__ int pick;
    __shared__ long long pick_below, pick_weight;
    __shared__ unsigned pick_count;
    const double total = static_cast<double>(sm->total);
    for (int q = 0; q < kQ; ++q) {
        if (!active[q]) continue;
        const int slot = first ? 0 : q;
        const unsigned* hc = gcnt + slot * kSelBuckets;
        const unsigned long long* hwq = gw + slot * kSelBuckets;
        const double T = sel_q(q) * total;
        long long mine[kPer];
        long long run = 0;
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            mine[u] = static_cast<long long>(__ldcg(hwq + threadIdx.x * kPer + u));
            run += mine[u];
        }
        scan[threadIdx.x] = run;
        if (threadIdx.x == 0) pick = kSelBuckets;
        __syncthreads();
        for (int off = 1; off < kSelThreads; off <<= 1) {
            const long long add = threadIdx.x >= off ? scan[threadIdx.x - off] : 0;
            __syncthreads();
            scan[threadIdx.x] += add;
            __syncthreads();
        }
        // Inclusive cumulative weight at the end of each bucket; the first bucket whose end passes
        // T holds it (with T at or past the range's end, by rounding of q W: its last non-empty
        // bucket).
        const long long excl = scan[threadIdx.x] - run;
        long long cum = st[q].before + excl;
        int found = kSelBuckets, last_nz = -1;
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            cum += mine[u];
            if (found == kSelBuckets && mine[u] > 0 && static_cast<double>(cum) > T) found = threadIdx.x * kPer + u;
            if (mine[u] > 0) last_nz = threadIdx.x * kPer + u;
        }
        if (found < kSelBuckets) atomicMin(&pick, found);
        __syncthreads();
        if (pick == kSelBuckets) {
            if (threadIdx.x == 0) pick = -1;
            __syncthreads();
            if (last_nz >= 0) atomicMax(&pick, last_nz);
            __syncthreads();
        }
        const int b = pick;
        if (b >= threadIdx.x * kPer && b < (threadIdx.x + 1) * kPer) {
            // The bucket's owner: its weight-before from its own scan share.
            long long below = excl;
            for (int u = 0; u < b - threadIdx.x * kPer; ++u) below += mine[u];
            pick_below = below;
            pick_weight = mine[b - threadIdx.x * kPer];
            pick_count = __ldcg(hc + b);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            SelState s = st[q];
            s.before += pick_below;
            s.weight = pick_weight;
            s.prefix = (s.shift >= 64 ? 0ull : (s.prefix << width)) | static_cast<unsigned long long>(b);
            s.shift -= width;
            s.count = static_cast<int>(pick_count);
            s.phase = (s.count <= kCand || s.shift <= 32) ? 1 : 0;
            states[c * kQ + q] = s;
        }
        __syncthreads();
    }
    // Clear this placement's histograms for the next level.
    for (int b = threadIdx.x; b < kQ * kSelBuckets; b += blockDim.x) {
        gcnt[b] = 0;
        gw[b] = 0;
    }
    if (threadIdx.x == 0) ticket[c] = 0;
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long u = __shfl_xor_sync(0xffffffffu, v, o);
        v = u > v ? u : v;
    }
    return v;
}
__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long u = __shfl_xor_sync(0xffffffffu, v, o);
        v = u < v ? u : v;
    }
    return v;
}

// Each quantile's range: its keys (when it holds at most kCand), its first and last key, and the
// nearest keys below and above it.
__global__ void __launch_bounds__(kSelThreads) sel_gather_kernel(const float* __restrict__ gv, int n_gm,
                                                                 const SelState* __restrict__ states,
                                                                 unsigned long long* __restrict__ cand,
                                                                 int* __restrict__ cand_n,
                                                                 SelEdges* __restrict__ edges) {
    const int c = blockIdx.y;
    SelState st[kQ];
#pragma unroll
    for (int q = 0; q < kQ; ++q) st[q] = states[c * kQ + q];
    unsigned long long lo[kQ], hi[kQ], below[kQ], above[kQ];
#pragma unroll
    for (int q = 0; q < kQ; ++q) {
        lo[q] = ~0ull;
        hi[q] = 0;
        below[q] = 0;
        above[q] = ~0ull;
    }
    const long chunk = (static_cast<long>(n_gm) + gridDim.x - 1) / gridDim.x;
    const int i0 = static_cast<int>(min(static_cast<long>(n_gm), blockIdx.x * chunk));
    const int i1 = static_cast<int>(min(static_cast<long>(n_gm), i0 + chunk));
    const float* gvc = gv + static_cast<long>(c) * n_gm;
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        const unsigned long long key = sel_key(gvc[i], i);
#pragma unroll
        for (int q = 0; q < kQ; ++q) {
            if (in_range(key, st[q])) {
                lo[q] = min(lo[q], key);
                hi[q] = max(hi[q], key);
                if (st[q].count <= kCand) {
                    const int slot = atomicAdd(&cand_n[c * kQ + q], 1);
                    if (slot < kCand) cand[(static_cast<long>(c) * kQ + q) * kCand + slot] = key;
                }
            } else if ((key >> st[q].shift) < st[q].prefix) {  // shift < 64 here: a full range has no outside
                below[q] = max(below[q], key + 1);
            } else {
                above[q] = min(above[q], key);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < kQ; ++q) {
        const unsigned long long a = warp_min_u64(lo[q]), b = warp_max_u64(hi[q]);
        const unsigned long long p = warp_max_u64(below[q]), s = warp_min_u64(above[q]);
        if ((threadIdx.x & 31) == 0) {
            SelEdges* e = edges + c * kQ + q;
            if (a != ~0ull) atomicMin(&e->first, a);
            if (b) atomicMax(&e->last, b);
            if (p) atomicMax(&e->pred, p);
            if (s != ~0ull) atomicMin(&e->succ, s);
        }
    }
}

// Linear interpolation between (x0, v0) and (x1, v1) at q, as numpy.interp evaluates it.
__device__ __forceinline__ double interp2(double q, double x0, double v0, double x1, double v1) {
    const double slope = (v1 - v0) / (x1 - x0);
    return slope * (q - x0) + v0;
}

// One block per (quantile, placement). Candidates: each one's B is the weight of the range's
// smaller keys plus the range's `before`; the candidate whose [B, B + w) holds T is e, bracketed
// with its neighbour on q's side (the next candidate, or the nearest key outside the range). A
// range of ties: only its first and last element can bracket q with an element outside it.
__global__ void __launch_bounds__(kResolveThreads) sel_resolve_kernel(
    const long long* __restrict__ wfix, const SelMesh* __restrict__ sm, const SelState* __restrict__ states,
    const unsigned long long* __restrict__ cand, const int* __restrict__ cand_n,
    const SelEdges* __restrict__ edges, double* __restrict__ qval) {
    __shared__ unsigned long long key[kCand];
    __shared__ long long wt[kCand];
    __shared__ int hit;
    const int q = blockIdx.x, c = blockIdx.y;
    const SelState st = states[c * kQ + q];
    const SelEdges ed = edges[c * kQ + q];
    const double total = static_cast<double>(sm->total);
    const double qv = sel_q(q);
    const double T = qv * total;
    const double two_w = 2.0 * total;
    auto w_of = [&](unsigned long long k) { return wfix[static_cast<unsigned>(k & 0xffffffffu)]; };
    auto v_of = [&](unsigned long long k) { return static_cast<double>(__uint_as_float(static_cast<unsigned>(k >> 32))); };
    auto pos_of = [&](long long b, long long w) { return static_cast<double>(2 * b + w) / two_w; };
    double* out = qval + c * kQ + q;
    if (st.count > kCand) {
        // One value repeated over the whole range (every value bit is fixed).
        if (threadIdx.x != 0) return;
        const double v = v_of(ed.first);
        const long long wf = w_of(ed.first), wl = w_of(ed.last);
        const double p_first = pos_of(st.before, wf);
        const double p_last = pos_of(st.before + st.weight - wl, wl);
        if (p_first > qv) {
            if (ed.pred == 0) *out = v;
            else {
                const unsigned long long pk = ed.pred - 1;
                const long long wp = w_of(pk);
                *out = interp2(qv, pos_of(st.before - wp, wp), v_of(pk), p_first, v);
            }
        } else if (p_last <= qv) {
            if (ed.succ == ~0ull) *out = v;
            else *out = interp2(qv, p_last, v, pos_of(st.before + st.weight, w_of(ed.succ)), v_of(ed.succ));
        } else {
            *out = v;  // two elements of the range bracket q
        }
        return;
    }
    const int n = min(cand_n[c * kQ + q], kCand);
    if (n == 0) {  // cannot happen for a range chosen by weight; reported as NaN rather than read
        if (threadIdx.x == 0) *out = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    const unsigned long long* src = cand + (static_cast<long>(c) * kQ + q) * kCand;
    __shared__ long long hit_before;
    __shared__ unsigned long long e_key, prev_key, next_key;
    const int j = threadIdx.x;  // one candidate per thread (kResolveThreads == kCand)
    unsigned long long kj = ~0ull;
    if (j < n) {
        kj = src[j];
        key[j] = kj;
        wt[j] = w_of(kj);
    }
    if (threadIdx.x == 0) {
        hit = -1;
        prev_key = 0;
        next_key = ~0ull;
    }
    __syncthreads();
    // Each candidate's weight-before (keys are distinct); exact integer sums, any order.
    if (j < n) {
        long long b = st.before;
        for (int u = 0; u < n; ++u) b += key[u] < kj ? wt[u] : 0;
        if (static_cast<double>(b) <= T && T < static_cast<double>(b + wt[j])) {
            hit = j;
            hit_before = b;
        }
    }
    __syncthreads();
    if (hit < 0) {  // T at or past the range's end (rounding of q W): the range's last key
        if (threadIdx.x == 0) e_key = 0;
        __syncthreads();
        if (j < n) atomicMax(&e_key, kj);
        __syncthreads();
        if (j < n && kj == e_key) {
            long long b = st.before;
            for (int u = 0; u < n; ++u) b += key[u] < kj ? wt[u] : 0;
            hit = j;
            hit_before = b;
        }
        __syncthreads();
    }
    const unsigned long long ke = key[hit];
    if (j < n) {  // the candidates just below and above e (prev as key + 1, 0: none)
        if (kj < ke) atomicMax(&prev_key, kj + 1);
        if (kj > ke) atomicMin(&next_key, kj);
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const long long we = wt[hit];
    const long long be = hit_before;
    const unsigned long long prev = prev_key ? prev_key : ed.pred;
    const unsigned long long next = next_key != ~0ull ? next_key : ed.succ;
    const double pe = pos_of(be, we);
    if (pe <= qv) {
        if (next == ~0ull) *out = v_of(ke);
        else *out = interp2(qv, pe, v_of(ke), pos_of(be + we, w_of(next)), v_of(next));
    } else {
        if (prev == 0) {
            *out = v_of(ke);
        } else {
            const unsigned long long pk = prev - 1;
            const long long wp = w_of(pk);
            *out = interp2(qv, pos_of(be - wp, wp), v_of(pk), pe, v_of(ke));
        }
    }
}

// Focality: the weight of the elements with |E| >= 0.5 p99.9 and >= 0.75 p99.9.
__global__ void __launch_bounds__(kSelThreads) sel_focality_kernel(const float* __restrict__ gv, int n_gm,
                                                                   const long long* __restrict__ wfix,
                                                                   const double* __restrict__ qval,
                                                                   long long* __restrict__ foc) {
    const int c = blockIdx.y;
    const double p999 = qval[c * kQ + 3];
    const double t0 = 0.5 * p999, t1 = 0.75 * p999;
    const long chunk = (static_cast<long>(n_gm) + gridDim.x - 1) / gridDim.x;
    const int i0 = static_cast<int>(min(static_cast<long>(n_gm), blockIdx.x * chunk));
    const int i1 = static_cast<int>(min(static_cast<long>(n_gm), i0 + chunk));
    const float* gvc = gv + static_cast<long>(c) * n_gm;
    long long s0 = 0, s1 = 0;
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        const double v = gvc[i];
        if (v >= t0) s0 += wfix[i];
        if (v >= t1) s1 += wfix[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (s0) atomicAdd(reinterpret_cast<unsigned long long*>(&foc[2 * c]), static_cast<unsigned long long>(s0));
        if (s1) atomicAdd(reinterpret_cast<unsigned long long*>(&foc[2 * c + 1]), static_cast<unsigned long long>(s1));
    }
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

// One warp per placement: partials combined in a fixed order (lane l takes blocks l and l + 32,
// then a butterfly); the percentiles and the focality weights come from the radix select.
__global__ void __launch_bounds__(kWarp) summary_final_kernel(
    int k, const int* __restrict__ gm, const double* __restrict__ bary, const double* __restrict__ part,
    const int* __restrict__ part_i, const double* __restrict__ var_part, const double* __restrict__ qval,
    const long long* __restrict__ foc, const SelMesh* __restrict__ sm, double* __restrict__ out) {
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
    if (lane != 0) return;
    double* o = out + static_cast<long>(c) * kSummaryLen;
    const double w_s = f[1], wm_s = f[2];
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
    for (int j = 0; j < kQ; ++j) o[10 + j] = qval[c * kQ + j];
    for (int g = 0; g < 2; ++g) o[14 + g] = ldexp(static_cast<double>(foc[2 * c + g]), -sm->exp2);
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
    // Fixed-point gray-matter weights: once per mesh (volumes do not change with conductivity).
    if (w.wfix_n != n) {
        w.wfix.resize(n);
        w.sel_mesh.resize(sizeof(SelMesh));
        w.sel_mesh.zero(s);
        SelMesh* sm = reinterpret_cast<SelMesh*>(w.sel_mesh.get());
        gm_wmax_kernel<<<std::min(grid_for(n), 592u), kBlock, 0, s>>>(m.vols32.get(), m.gm_index.get(), n, sm);
        gm_wfix_kernel<<<std::min(grid_for(n), 592u), kBlock, 0, s>>>(m.vols32.get(), m.gm_index.get(), n, sm,
                                                                   w.wfix.get());
        count_launch(2);
        CUNIBS_LAUNCH_CHECK("gray-matter weights");
        w.wfix_n = n;
    }
    const SelMesh* sm = reinterpret_cast<const SelMesh*>(w.sel_mesh.get());
    static_assert(sizeof(SelState) % 8 == 0, "state alignment");
    w.gv.reserve(static_cast<std::size_t>(n) * k);
    w.sel_state.reserve(sizeof(SelState) * k * kQ);
    w.hcnt.reserve(static_cast<std::size_t>(k) * kQ * kSelBuckets);
    w.hw.reserve(static_cast<std::size_t>(k) * kQ * kSelBuckets);
    w.cand.reserve(static_cast<std::size_t>(k) * kQ * kCand);
    w.edges.reserve(sizeof(SelEdges) * k * kQ);
    w.cand_n.reserve(static_cast<std::size_t>(k) * kQ);
    w.ticket.reserve(k);
    w.qval.reserve(static_cast<std::size_t>(k) * kQ);
    w.foc.reserve(2 * static_cast<std::size_t>(k));
    SelState* st = reinterpret_cast<SelState*>(w.sel_state.get());
    // The histograms start clear and each level's last blocks clear them again for the next.
    if (!w.hist_clear || w.hist_k < k) {
        w.hcnt.zero(s);
        w.hw.zero(s);
        w.hist_clear = true;
        w.hist_k = k;
    }
    SelEdges* edges = reinterpret_cast<SelEdges*>(w.edges.get());
    sel_init_kernel<<<1, 256, 0, s>>>(k, n, sm, st, w.cand_n.get(), edges, w.ticket.get(), w.foc.get());
    count_launch();
    // Blocks per placement: about two waves over the GPU for the whole block of placements.
    const unsigned chunks = static_cast<unsigned>(std::max(1, std::min(64, (2 * 148 + k - 1) / k)));
    // Shared histograms: one slot on the first level (every quantile shares the whole range), kQ after.
    const std::size_t slot_bytes = static_cast<std::size_t>(kSelBuckets) * (sizeof(unsigned) + sizeof(unsigned long long));
    static bool opted = false;  // per process: the attribute is per kernel, the same on every device
    if (!opted) {
        CUNIBS_CHECK(cudaFuncSetAttribute(sel_level_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(kQ * slot_bytes)));
        opted = true;
    }
    for (int level = 0; level < kSelLevels; ++level) {
        const std::size_t smem = (level == 0 ? 1 : kQ) * slot_bytes;
        sel_level_kernel<<<dim3(chunks, k), kSelThreads, smem, s>>>(level, magnE, m.gm_index.get(), n, m.n_tets,
                                                                    w.wfix.get(), sm, w.gv.get(), st, w.hcnt.get(),
                                                                    w.hw.get(), w.ticket.get());
        count_launch();
    }
    sel_gather_kernel<<<dim3(chunks, k), kSelThreads, 0, s>>>(w.gv.get(), n, st, w.cand.get(), w.cand_n.get(), edges);
    sel_resolve_kernel<<<dim3(kQ, k), kResolveThreads, 0, s>>>(w.wfix.get(), sm, st, w.cand.get(), w.cand_n.get(),
                                                                edges, w.qval.get());
    sel_focality_kernel<<<dim3(chunks, k), kSelThreads, 0, s>>>(w.gv.get(), n, w.wfix.get(), w.qval.get(),
                                                                w.foc.get());
    count_launch(3);
    CUNIBS_LAUNCH_CHECK("gm percentiles");
    w.part.reserve(static_cast<std::size_t>(k) * kSumBlocks * (kSumFields + 1));
    w.part_i.reserve(static_cast<std::size_t>(k) * kSumBlocks);
    double* part = w.part.get();
    double* var_part = part + static_cast<std::size_t>(k) * kSumBlocks * kSumFields;
    summary_stats_kernel<<<dim3(kSumBlocks, k), kSumT, 0, s>>>(magnE, m.gm_index.get(), n, m.n_tets, m.vols32.get(),
                                                               m.bary.get(), part, w.part_i.get());
    summary_var_kernel<<<dim3(kSumBlocks, k), kSumT, 0, s>>>(magnE, m.gm_index.get(), n, m.n_tets, m.vols32.get(),
                                                             part, var_part);
    summary_final_kernel<<<k, kWarp, 0, s>>>(k, m.gm_index.get(), m.bary.get(), part, w.part_i.get(), var_part,
                                          w.qval.get(), w.foc.get(), sm, out);
    count_launch(3);
    CUNIBS_LAUNCH_CHECK("gm summary");
}

void gm_summary(const Mesh& m, const float* magnE, int k, double* summary_dev, SummaryWork& w, cudaStream_t s) {
    gm_summary_impl(m, magnE, k, summary_dev, w, s);
}

}  // namespace cunibs
