// BF16 tensor-core GEMM for sm_100a (B200): C[M,N] = A[M,K] . B[N,K]^T, FP32 accumulation in TMEM.
//
// The GEMMs of the learned warm start (forward, both backward products, and the prolongation of the
// predicted coefficients) all take this one "both operands K-major" form; the network keeps the
// transposed copies it needs (the epilogue writes them for free) instead of switching operand
// majorness.
//
// One CTA per BM x BN output tile, 6 warps:
//   warp 4       TMA producer: 128-byte-swizzled K-major tiles of A and B into a STAGES-deep ring,
//                each stage guarded by a full/empty mbarrier pair (cp.async.bulk.tensor, no multicast);
//   warp 5       allocates TMEM, and one elected lane issues tcgen05.mma (kind::f16, BF16 in, FP32
//                accumulate) per 16-wide K step, releasing each stage with tcgen05.commit;
//   warps 0..3   epilogue: tcgen05.ld of their 32 TMEM lanes (one output row per thread), then the
//                fused tail (bias, SiLU or SiLU' gating) and the stores: FP32 and/or BF16 row-major and
//                a BF16 transposed copy (coalesced: a warp's lanes are 32 consecutive rows).
// Every mbarrier wait is bounded; on expiry the kernel records an error flag and winds down (the
// TMEM allocation is always released).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <atomic>
#include <cstdlib>
#include <mutex>

#include "internal.hpp"

namespace cunibs {
namespace {

constexpr int BM = 128;
constexpr int BK = 64;  // one 128-byte swizzle atom of BF16 per row
constexpr int STAGES = 4;
constexpr int kThreads = 192;
// Every mbarrier wait gives up after this many polls or this much %globaltimer time, whichever
// comes first (a stage's loads land within microseconds; these only bound a failure).
constexpr long long kSpinLimit = 1LL << 24;
constexpr unsigned long long kWaitLimitNs = 2000000000ULL;

__device__ __forceinline__ std::uint32_t smem_u32(const void* p) {
    return static_cast<std::uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(std::uint64_t* bar, std::uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(std::uint64_t* bar, std::uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(std::uint64_t* bar, std::uint32_t parity) {
    std::uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for the phase with the given parity to complete: at most `polls` polls and at most
// `limit_ns` of global time.
__device__ __forceinline__ bool mbar_wait(std::uint64_t* bar, std::uint32_t parity, long long polls,
                                          unsigned long long limit_ns) {
    const unsigned long long t0 = global_ns();
    for (long long i = 0; i < polls; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 255) == 255 && global_ns() - t0 > limit_ns) return false;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(const CUtensorMap* map, std::uint64_t* bar, void* dst, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<std::uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Shared-memory matrix descriptor of a K-major, 128-byte-swizzled tile: rows 128 B apart, 8-row
// groups 1024 B apart (SBO), descriptor version 1, layout type 2 (SWIZZLE_128B).
__device__ __forceinline__ std::uint64_t sw128_desc(const void* tile) {
    const std::uint64_t addr = smem_u32(tile);
    std::uint64_t d = (addr & 0x3FFFF) >> 4;
    d |= std::uint64_t{1} << 16;
    d |= std::uint64_t{1024 >> 4} << 32;
    d |= std::uint64_t{1} << 46;
    d |= std::uint64_t{2} << 61;
    return d;
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, M x N.
template <int BN>
__host__ __device__ constexpr std::uint32_t idesc_bf16() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<std::uint32_t>(BN >> 3) << 17) |
           (static_cast<std::uint32_t>(BM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(std::uint32_t tmem_d, std::uint64_t adesc, std::uint64_t bdesc,
                                          std::uint32_t idesc, std::uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(
            tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(std::uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(std::uint32_t taddr, float (&v)[16]) {
    std::uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }

// d silu / dz = s (1 + z (1 - s)), s = sigmoid(z)
__device__ __forceinline__ float silu_grad(float z) {
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

template <int BN>
__global__ void __launch_bounds__(kThreads, 1)
    gemm_bf16_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                     GemmEpilogue ep, int M, int N, int K) {
    constexpr std::uint32_t kABytes = BM * BK * 2;
    constexpr std::uint32_t kBBytes = BN * BK * 2;
    constexpr std::uint32_t kStageBytes = kABytes + kBBytes;
    constexpr std::uint32_t kTmemCols = BN < 32 ? 32 : BN;
    extern __shared__ unsigned char dyn_smem[];
    // SWIZZLE_128B tiles want 1024-byte alignment.
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<std::uintptr_t>(dyn_smem) + 1023) &
                                                          ~std::uintptr_t{1023});
    std::uint64_t* full = reinterpret_cast<std::uint64_t*>(smem + STAGES * kStageBytes);
    std::uint64_t* empty = full + STAGES;
    std::uint64_t* accum = empty + STAGES;
    std::uint32_t* tmem_slot = reinterpret_cast<std::uint32_t*>(accum + 1);
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int num_kb = (K + BK - 1) / BK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(accum, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 5) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const std::uint32_t tmem = *tmem_slot;

    if (warp == 4 && lane == 0) {
        // Producer.
        // ep.withhold_loads (a test of the timeout path) issues no loads: the MMA warp's first wait
        // can then only run out.
        for (int kb = 0; kb < num_kb && !ep.withhold_loads; ++kb) {
            const int s = kb % STAGES;
            if (kb >= STAGES && !mbar_wait(&empty[s], ((kb / STAGES) & 1) ^ 1, ep.wait_polls, ep.wait_ns)) {
                *abort_flag = 1;
                break;
            }
            unsigned char* st = smem + s * kStageBytes;
            mbar_expect_tx(&full[s], kStageBytes);
            tma_load_2d(&map_a, &full[s], st, kb * BK, m0);
            tma_load_2d(&map_b, &full[s], st + kABytes, kb * BK, n0);
        }
    } else if (warp == 5 && lane == 0) {
        // MMA issuer.
        constexpr std::uint32_t idesc = idesc_bf16<BN>();
        bool ok = true;
        for (int kb = 0; kb < num_kb && ok; ++kb) {
            const int s = kb % STAGES;
            if (!mbar_wait(&full[s], (kb / STAGES) & 1, ep.wait_polls, ep.wait_ns)) {
                ok = false;
                break;
            }
            tc_fence_after();
            unsigned char* st = smem + s * kStageBytes;
            const std::uint64_t adesc = sw128_desc(st), bdesc = sw128_desc(st + kABytes);
#pragma unroll
            for (int k = 0; k < BK / 16; ++k)
                umma_bf16(tmem, adesc + 2 * k, bdesc + 2 * k, idesc, (kb > 0 || k > 0) ? 1u : 0u);
            umma_commit(&empty[s]);
        }
        if (!ok) *abort_flag = 1;
        umma_commit(accum);  // arrives once every MMA issued above has completed
    } else if (warp < 4) {
        // Epilogue: thread (warp, lane) owns output row m0 + 32 warp + lane.
        const bool ready = mbar_wait(accum, 0, ep.wait_polls, ep.wait_ns);
        tc_fence_after();
        const int row = m0 + warp * 32 + lane;
        if (ready) {
#pragma unroll 1
            for (int c = 0; c < BN; c += 16) {
                float v[16];
                tmem_ld16(tmem + (static_cast<std::uint32_t>(warp * 32) << 16) + static_cast<std::uint32_t>(c), v);
                const bool row_ok = row < M;
                const int col0 = n0 + c;
                float z[16], h[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = col0 + j;
                    float t = v[j];
                    if (row_ok && col < N) {
                        if (ep.bias) t += ep.bias[col];
                        if (ep.gate) t *= silu_grad(ep.gate[static_cast<std::int64_t>(row) * ep.ld_gate + col]);
                    }
                    z[j] = t;
                    h[j] = ep.act == 1 ? silu(t) : t;
                }
                if (!row_ok) continue;
                const std::int64_t at = static_cast<std::int64_t>(row) * ep.ld_out + col0;
                // A full, aligned 16-column run goes out as 16-byte vector stores; the ragged edge
                // (or an unaligned leading dimension) element by element.
                const bool full = col0 + 16 <= N && (ep.ld_out % 8) == 0;
                if (ep.out32) {
                    if (full && (reinterpret_cast<std::uintptr_t>(ep.out32) & 15) == 0) {
#pragma unroll
                        for (int j = 0; j < 16; j += 4)
                            *reinterpret_cast<float4*>(ep.out32 + at + j) = make_float4(z[j], z[j + 1], z[j + 2], z[j + 3]);
                    } else {
                        for (int j = 0; j < 16 && col0 + j < N; ++j) ep.out32[at + j] = z[j];
                    }
                }
                if (ep.out16) {
                    if (full && (reinterpret_cast<std::uintptr_t>(ep.out16) & 15) == 0) {
#pragma unroll
                        for (int j = 0; j < 16; j += 8) {
                            __nv_bfloat162 q[4];
#pragma unroll
                            for (int u = 0; u < 4; ++u) q[u] = __floats2bfloat162_rn(h[j + 2 * u], h[j + 2 * u + 1]);
                            *reinterpret_cast<uint4*>(ep.out16 + at + j) = *reinterpret_cast<uint4*>(q);
                        }
                    } else {
                        for (int j = 0; j < 16 && col0 + j < N; ++j) ep.out16[at + j] = __float2bfloat16_rn(h[j]);
                    }
                }
                if (ep.out16t) {
                    for (int j = 0; j < 16 && col0 + j < N; ++j)
                        ep.out16t[static_cast<std::int64_t>(col0 + j) * ep.ld_t + row] = __float2bfloat16_rn(h[j]);
                }
            }
        } else {
            *abort_flag = 1;
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x == 0 && *abort_flag && ep.error) atomicExch(ep.error, 1);
    if (warp == 5)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

// Tall, narrow products streamed by persistent CTAs: C[M, BN] = A[M, K] . B[BN, K]^T with K at most
// kStreamMaxKB * BK and only an FP32 output (the prolongation of the network's coefficients through
// the basis: M = nodes, K = 2 x rank, a 183 MB A read once). One CTA per SM walks the M tiles
// tile = blockIdx.x, + gridDim.x, ...:
//   warp 4   loads B once (it stays in shared memory), then streams A's 128 x 64 tiles through a
//            kStreamStages-deep ring without a break between M tiles;
//   warp 5   issues the MMAs of tile t into one of two TMEM accumulators (t & 1), so tile t + 1
//            accumulates while the epilogue drains tile t;
//   warps 0-3 read a finished accumulator, release it (one arrive per warp) and store its rows.
// Every wait is bounded; an expired wait sets the abort word, every role leaves its loop at its next
// check, and before TMEM is freed the MMA issuer waits (bounded) for its issued MMAs and the producer
// for its last issued loads.
constexpr int kStreamStages = 8;
constexpr int kStreamMaxKB = 8;

template <int BN>
__global__ void __launch_bounds__(kThreads, 1)
    gemm_stream_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                       float* __restrict__ out32, int ld_out, int M, int N, int K, int* error, long long wait_polls,
                       unsigned long long wait_ns, int withhold_loads) {
    constexpr std::uint32_t kABytes = BM * BK * 2;
    constexpr std::uint32_t kBBytes = BN * BK * 2;
    constexpr std::uint32_t kTmemCols = 2 * BN < 32 ? 32 : 2 * BN;
    extern __shared__ unsigned char dyn_smem[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<std::uintptr_t>(dyn_smem) + 1023) &
                                                          ~std::uintptr_t{1023});
    unsigned char* a_ring = smem;                                    // kStreamStages x kABytes
    unsigned char* b_res = smem + kStreamStages * kABytes;           // kStreamMaxKB x kBBytes
    std::uint64_t* full = reinterpret_cast<std::uint64_t*>(b_res + kStreamMaxKB * kBBytes);
    std::uint64_t* empty = full + kStreamStages;
    std::uint64_t* acc_full = empty + kStreamStages;  // [2]
    std::uint64_t* acc_empty = acc_full + 2;          // [2]
    std::uint64_t* b_full = acc_empty + 2;
    std::uint64_t* drain = b_full + 1;
    std::uint32_t* tmem_slot = reinterpret_cast<std::uint32_t*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int num_kb = (K + BK - 1) / BK;
    const int n_tiles = (M + BM - 1) / BM;
    if (threadIdx.x == 0) {
        for (int i = 0; i < kStreamStages; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&acc_full[a], 1);
            mbar_init(&acc_empty[a], 4);  // one arrive per epilogue warp
        }
        mbar_init(b_full, 1);
        mbar_init(drain, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 5) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const std::uint32_t tmem = *tmem_slot;

    if (warp == 4 && lane == 0) {
        // Producer.
        long long issued = 0;  // A k-blocks issued over all tiles
        if (!withhold_loads) {
            mbar_expect_tx(b_full, kBBytes * num_kb);
            for (int kb = 0; kb < num_kb; ++kb) tma_load_2d(&map_b, b_full, b_res + kb * kBBytes, kb * BK, 0);
            for (int tile = blockIdx.x; tile < n_tiles && !*abort_flag; tile += gridDim.x) {
                for (int kb = 0; kb < num_kb; ++kb, ++issued) {
                    const int sidx = static_cast<int>(issued % kStreamStages);
                    if (issued >= kStreamStages &&
                        !mbar_wait(&empty[sidx], static_cast<std::uint32_t>(((issued / kStreamStages) & 1) ^ 1),
                                   wait_polls, wait_ns)) {
                        *abort_flag = 1;
                        break;
                    }
                    mbar_expect_tx(&full[sidx], kABytes);
                    tma_load_2d(&map_a, &full[sidx], a_ring + sidx * kABytes, kb * BK, tile * BM);
                }
            }
            // Before the shared memory goes: the last loads issued into each stage have landed.
            for (long long g = issued > kStreamStages ? issued - kStreamStages : 0; g < issued; ++g)
                (void)mbar_wait(&full[g % kStreamStages], static_cast<std::uint32_t>((g / kStreamStages) & 1),
                                wait_polls, wait_ns);
            (void)mbar_wait(b_full, 0, wait_polls, wait_ns);
        }
    } else if (warp == 5 && lane == 0) {
        // MMA issuer.
        constexpr std::uint32_t idesc = idesc_bf16<BN>();
        bool ok = mbar_wait(b_full, 0, wait_polls, wait_ns);
        long long used = 0;  // A k-blocks consumed over all tiles
        int t = 0;           // this CTA's tile count
        for (int tile = blockIdx.x; ok && tile < n_tiles; tile += gridDim.x, ++t) {
            const int a = t & 1;
            if (t >= 2 && !mbar_wait(&acc_empty[a], static_cast<std::uint32_t>(((t >> 1) & 1) ^ 1), wait_polls, wait_ns)) {
                ok = false;
                break;
            }
            tc_fence_after();
            for (int kb = 0; kb < num_kb; ++kb, ++used) {
                const int sidx = static_cast<int>(used % kStreamStages);
                if (*abort_flag || !mbar_wait(&full[sidx], static_cast<std::uint32_t>((used / kStreamStages) & 1),
                                              wait_polls, wait_ns)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const std::uint64_t adesc = sw128_desc(a_ring + sidx * kABytes);
                const std::uint64_t bdesc = sw128_desc(b_res + kb * kBBytes);
#pragma unroll
                for (int k = 0; k < BK / 16; ++k)
                    umma_bf16(tmem + static_cast<std::uint32_t>(a * BN), adesc + 2 * k, bdesc + 2 * k, idesc,
                              (kb > 0 || k > 0) ? 1u : 0u);
                umma_commit(&empty[sidx]);
            }
            if (!ok) break;
            umma_commit(&acc_full[a]);
        }
        if (!ok) *abort_flag = 1;
        // Every MMA issued above has completed before the final barrier frees TMEM.
        umma_commit(drain);
        (void)mbar_wait(drain, 0, wait_polls, wait_ns);
    } else if (warp < 4) {
        // Epilogue: thread (warp, lane) owns row 32 warp + lane of each tile.
        int t = 0;
        for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, ++t) {
            const int a = t & 1;
            if (*abort_flag || !mbar_wait(&acc_full[a], static_cast<std::uint32_t>((t >> 1) & 1), wait_polls, wait_ns)) {
                *abort_flag = 1;
                break;
            }
            tc_fence_after();
            float v[BN];
#pragma unroll
            for (int c = 0; c < BN; c += 16) {
                float part[16];
                tmem_ld16(tmem + (static_cast<std::uint32_t>(warp * 32) << 16) + static_cast<std::uint32_t>(a * BN + c),
                          part);
#pragma unroll
                for (int j = 0; j < 16; ++j) v[c + j] = part[j];
            }
            // The accumulator is in registers: hand it back to the MMA issuer.
            tc_fence_before();
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[a])) : "memory");
            const int row = tile * BM + warp * 32 + lane;
            if (row < M) {
                float* o = out32 + static_cast<std::int64_t>(row) * ld_out;
                if (N == BN && (ld_out % 4) == 0 && (reinterpret_cast<std::uintptr_t>(out32) & 15) == 0) {
#pragma unroll
                    for (int j = 0; j < BN; j += 4)
                        *reinterpret_cast<float4*>(o + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
                } else {
#pragma unroll
                    for (int j = 0; j < BN; ++j)
                        if (j < N) o[j] = v[j];
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x == 0 && *abort_flag && error) atomicExch(error, 1);
    if (warp == 5)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    if (!fn) fail(kECuda, "cuTensorMapEncodeTiled is unavailable");
    return fn;
}

// Row-major [rows, cols] BF16 with leading dimension ld (elements), boxes of box_rows x 64.
CUtensorMap make_map(const void* base, int rows, int cols, int ld, int box_rows) {
    if (reinterpret_cast<std::uintptr_t>(base) % 16 != 0) fail(kEInval, "GEMM operand is not 16-byte aligned");
    if (ld % 8 != 0) fail(kEInval, "GEMM leading dimension must be a multiple of 8 elements");
    CUtensorMap map;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld) * 2};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(BK), static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult rc = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides,
                                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (rc != CUDA_SUCCESS) fail(kEInval, "cuTensorMapEncodeTiled rejected a GEMM operand");
    return map;
}

template <int BN>
void launch(const GemmProblem& p, cudaStream_t s) {
    const CUtensorMap ma = make_map(p.a, p.M, p.K, p.lda, BM);
    const CUtensorMap mb = make_map(p.b, p.N, p.K, p.ldb, BN);
    constexpr std::size_t smem = STAGES * (BM + BN) * BK * 2 + 1024 + 256;
    // The shared-memory opt-in is set once per device (a host call per launch costs more than a
    // small GEMM's tiles).
    static std::atomic<std::uint64_t> opted{0};
    int dev = 0;
    CUNIBS_CHECK(cudaGetDevice(&dev));
    const std::uint64_t bit = std::uint64_t{1} << (dev & 63);
    if (!(opted.load(std::memory_order_acquire) & bit)) {
        CUNIBS_CHECK(cudaFuncSetAttribute(gemm_bf16_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(smem)));
        opted.fetch_or(bit, std::memory_order_acq_rel);
    }
    const dim3 grid((p.N + BN - 1) / BN, (p.M + BM - 1) / BM);
    gemm_bf16_kernel<BN><<<grid, kThreads, smem, s>>>(ma, mb, p.ep, p.M, p.N, p.K);
    count_launch();
    CUNIBS_LAUNCH_CHECK("gemm_bf16");
}

// The wait bounds every launch gets (cunibs_debug_gemm_waits changes them for tests of the
// timeout path), and the per-device word that launches without an error flag of their own report
// an expired wait to (read and cleared by gemm_status).
std::atomic<long long> g_wait_polls{kSpinLimit};
std::atomic<unsigned long long> g_wait_ns{kWaitLimitNs};
std::atomic<int> g_withhold{0};
constexpr int kMaxDevices = 64;
std::mutex g_status_mu;
int* g_status[kMaxDevices] = {};

int* status_word(int dev) {
    if (dev < 0 || dev >= kMaxDevices) fail(kEInval, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_status_mu);
    if (!g_status[dev]) {
        int* p = nullptr;
        CUNIBS_CHECK(cudaMalloc(&p, sizeof(int)));
        CUNIBS_CHECK(cudaMemset(p, 0, sizeof(int)));
        g_status[dev] = p;
    }
    return g_status[dev];
}

// The streamed form of a tall, narrow product with an FP32 output only: one persistent CTA per SM.
void launch_stream(const GemmProblem& p, cudaStream_t s) {
    constexpr int BN = 32;
    const CUtensorMap ma = make_map(p.a, p.M, p.K, p.lda, BM);
    const CUtensorMap mb = make_map(p.b, p.N, p.K, p.ldb, BN);
    constexpr std::size_t smem = kStreamStages * BM * BK * 2 + kStreamMaxKB * BN * BK * 2 + 1024 + 256;
    static std::atomic<std::uint64_t> opted{0};
    int dev = 0;
    CUNIBS_CHECK(cudaGetDevice(&dev));
    const std::uint64_t bit = std::uint64_t{1} << (dev & 63);
    if (!(opted.load(std::memory_order_acquire) & bit)) {
        CUNIBS_CHECK(cudaFuncSetAttribute(gemm_stream_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(smem)));
        opted.fetch_or(bit, std::memory_order_acq_rel);
    }
    int sms = 0;
    CUNIBS_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int n_tiles = (p.M + BM - 1) / BM;
    gemm_stream_kernel<BN><<<std::min(n_tiles, sms), kThreads, smem, s>>>(
        ma, mb, p.ep.out32, p.ep.ld_out, p.M, p.N, p.K, p.ep.error, p.ep.wait_polls, p.ep.wait_ns,
        p.ep.withhold_loads);
    count_launch();
    CUNIBS_LAUNCH_CHECK("gemm_bf16 stream");
}

bool streams(const GemmProblem& p) {
    const GemmEpilogue& e = p.ep;
    const bool plain = e.out32 && !e.out16 && !e.out16t && !e.bias && !e.gate && e.act == 0;
    return plain && p.N <= 32 && p.K <= kStreamMaxKB * BK && p.M >= 64 * BM;
}

}  // namespace

void gemm_bf16(const GemmProblem& p_in, cudaStream_t s) {
    if (p_in.M <= 0 || p_in.N <= 0 || p_in.K <= 0) fail(kEInval, "GEMM sizes must be positive");
    if (p_in.K % 8 != 0) fail(kEInval, "GEMM K must be a multiple of 8");
    if (p_in.ep.out16t && p_in.ep.ld_t < p_in.M) fail(kEInval, "transposed output leading dimension is below M");
    GemmProblem p = p_in;
    p.ep.wait_polls = g_wait_polls.load(std::memory_order_relaxed);
    p.ep.wait_ns = g_wait_ns.load(std::memory_order_relaxed);
    p.ep.withhold_loads = g_withhold.load(std::memory_order_relaxed);
    if (!p.ep.error) {
        int dev = 0;
        CUNIBS_CHECK(cudaGetDevice(&dev));
        p.ep.error = status_word(dev);
    }
    // A tall, narrow product with a plain FP32 output streams through persistent CTAs.
    if (streams(p) && std::getenv("CUNIBS_GEMM_TILED") == nullptr) {
        launch_stream(p, s);
        return;
    }
    // One row of tiles (M <= 128, the warm start's network at inference) is latency-bound: 32-wide
    // tiles give 4x the CTAs and smaller stages (measured 20.5 -> 10.4 us for 16 x 512 x 512).
    if (p.N <= 16) launch<16>(p, s);
    else if (p.N <= 32 || p.M <= BM) launch<32>(p, s);
    else launch<128>(p, s);
}

bool gemm_status(cudaStream_t s) {
    int dev = 0;
    CUNIBS_CHECK(cudaGetDevice(&dev));
    int* w = status_word(dev);
    int h = 0;
    CUNIBS_CHECK(cudaMemcpyAsync(&h, w, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUNIBS_CHECK(cudaStreamSynchronize(s));
    if (h) {
        CUNIBS_CHECK(cudaMemsetAsync(w, 0, sizeof(int), s));
        CUNIBS_CHECK(cudaStreamSynchronize(s));
    }
    return h != 0;
}

void gemm_set_waits(long long polls, unsigned long long limit_ns, int withhold_loads) {
    g_wait_polls.store(polls > 0 ? polls : kSpinLimit, std::memory_order_relaxed);
    g_wait_ns.store(limit_ns > 0 ? limit_ns : kWaitLimitNs, std::memory_order_relaxed);
    g_withhold.store(withhold_loads ? 1 : 0, std::memory_order_relaxed);
}

}  // namespace cunibs
