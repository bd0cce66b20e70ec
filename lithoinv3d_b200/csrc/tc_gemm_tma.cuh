// BF16 GEMM on the 5th-generation tensor cores fed by the tensor-memory
// accelerator: C[M x N] = A[M x K] . B[K x N], operand layouts, epilogues and
// size rules of k_gemm_bf16 (mlp_kernels.cuh), FP32 accumulation in tensor
// memory.
//
// CTA: 128 threads, tile 128 x BN x 64 (BN = 256 when N allows, else 128),
// a ring of four shared-memory stages, warp-specialised:
//  * warp 0, one lane: producer.  Per K block it waits for the stage to be
//    free, arms the stage's `full` mbarrier with the stage's byte count and
//    issues 2-D bulk tensor loads (cp.async.bulk.tensor, 128-byte swizzle, no
//    multicast) of the A and B tiles;
//  * warp 1, one lane: MMA issuer.  It waits for `full`, issues four
//    tcgen05.mma (M 128, N BN, K 16) from shared-memory descriptors into a
//    BN-column FP32 accumulator in tensor memory, and commits them to the
//    stage's `empty` mbarrier, which frees the stage for the producer; after
//    the last K block it commits to `done`;
//  * all four warps: epilogue.  After `done` each warp reads its 32 TMEM lanes
//    (rows) with tcgen05.ld, applies bias / ReLU and stores.
// Tile layouts in shared memory (the tensor cores' canonical 128-byte swizzled
// layouts, which the bulk tensor loads produce):
//  * K-major operand (K contiguous in global memory): rows of 64 K values
//    (128 bytes), 8-row groups 1024 bytes apart (stride byte offset); the
//    k-th 16-wide K slice starts 32 k bytes into the tile;
//  * MN-major operand (M or N contiguous): 64-wide M/N groups of 64 K rows,
//    groups 8192 bytes apart (leading byte offset), 8-row K groups 1024 bytes
//    apart (stride byte offset); the k-th K slice starts 2048 k bytes in.
// Every mbarrier wait is bounded: on expiry the role stops issuing, the block
// still waits (bounded) for its own loads and MMAs, frees its tensor memory
// and raises g_tc_gemm_error.
#pragma once
#include <cuda.h>

#include "tc_gemm.cuh"

namespace litho_b200 {
namespace mlp {

constexpr int kTmaStages = 4;
constexpr int kTmaThreads = 128;

template <int BN>
struct TmaShape {
    static constexpr int kStageA = kBM * kTcBK * 2;   // 16 KB
    static constexpr int kStageB = BN * kTcBK * 2;    // 16 or 32 KB
    static constexpr int kStage = kStageA + kStageB;
    // tiles + 1 KB to align the ring to 1024 bytes + barriers
    static constexpr int kSmem = kTmaStages * kStage + 1024 + 256;
};

// 128-byte-swizzle shared-memory matrix descriptor: start address, leading and
// stride byte offsets (all >> 4), version 1 [46,48), swizzle mode 2 [61,64).
__device__ __forceinline__ uint64_t tma_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(mbar)
        : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

// A is [M][K] (A_T = false, K-major) or [K][M] (MN-major); B is [K][N]
// (B_T = false, MN-major) or [N][K] (K-major).  Tensor maps: K-major operands
// map (K, rows) with boxes of 64 x rows-of-the-tile; MN-major ones map
// (M or N, K) with boxes of 64 x 64.
template <bool A_T, bool B_T, int EPI, int BN>
__global__ void __launch_bounds__(kTmaThreads) k_gemm_tma(int M, int N, int K, const __grid_constant__ CUtensorMap mapA,
                                                         const __grid_constant__ CUtensorMap mapB,
                                                         const float* __restrict__ bias, float* __restrict__ Cf,
                                                         __nv_bfloat16* __restrict__ Cb, int ldc) {
    using Sh = TmaShape<BN>;
    extern __shared__ uint8_t tma_smem_raw[];
    const uint32_t raw = smem_addr(tma_smem_raw);
    const uint32_t ring = (raw + 1023u) & ~1023u;  // 1024-byte aligned tiles (swizzle atoms)
    uint8_t* ringPtr = tma_smem_raw + (ring - raw);
    uint64_t* bars = reinterpret_cast<uint64_t*>(ringPtr + kTmaStages * Sh::kStage);  // full[4], empty[4], done
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(bars + 2 * kTmaStages + 1);
    int* flags = reinterpret_cast<int*>(tmemSlot + 1);  // [0] abort, [1] loads issued, [2] loads consumed
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * BN;
    auto full = [&](int s) { return smem_addr(&bars[s]); };
    auto empty = [&](int s) { return smem_addr(&bars[kTmaStages + s]); };
    const uint32_t done = smem_addr(&bars[2 * kTmaStages]);
    auto stageA = [&](int s) { return ring + s * Sh::kStage; };
    auto stageB = [&](int s) { return ring + s * Sh::kStage + Sh::kStageA; };

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmemSlot)),
                     "r"((uint32_t)BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < 2 * kTmaStages + 1; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bars[s])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        flags[0] = 0; flags[1] = 0; flags[2] = 0;
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapA)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapB)) : "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
    const uint32_t tmem = *tmemSlot;
    const int nk = K / kTcBK;
    volatile int* vflags = flags;

    if (warp == 0 && lane == 0) {  // producer
        int kt = 0;
        for (; kt < nk; ++kt) {
            const int s = kt % kTmaStages;
            if (vflags[0]) break;
            if (kt >= kTmaStages && !tc_wait(empty(s), ((kt / kTmaStages) - 1) & 1, g_tc_stage_wait_limit)) {
                vflags[0] = 1;
                break;
            }
            mbar_arrive_tx(full(s), (uint32_t)Sh::kStage);
            const int k0 = kt * kTcBK;
            if (!A_T) {
                tma_load_2d(stageA(s), &mapA, k0, m0, full(s));
            } else {
#pragma unroll
                for (int h = 0; h < kBM / 64; ++h) tma_load_2d(stageA(s) + h * 8192, &mapA, m0 + 64 * h, k0, full(s));
            }
            if (B_T) {
                tma_load_2d(stageB(s), &mapB, k0, n0, full(s));
            } else {
#pragma unroll
                for (int h = 0; h < BN / 64; ++h) tma_load_2d(stageB(s) + h * 8192, &mapB, n0 + 64 * h, k0, full(s));
            }
        }
        vflags[1] = kt;
    } else if (warp == 1 && lane == 0) {  // MMA issuer
        constexpr uint32_t idesc = tc_idesc(A_T ? 1 : 0, B_T ? 0 : 1, BN);
        int kt = 0;
        for (; kt < nk; ++kt) {
            const int s = kt % kTmaStages;
            if (vflags[0]) break;
            if (!tc_wait(full(s), (kt / kTmaStages) & 1, g_tc_stage_wait_limit)) {
                vflags[0] = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::);
#pragma unroll
            for (int j = 0; j < kTcBK / 16; ++j) {
                const uint64_t ad = A_T ? tma_smem_desc(stageA(s) + 2048u * j, 8192u, 1024u)
                                        : tma_smem_desc(stageA(s) + 32u * j, 16u, 1024u);
                const uint64_t bd = B_T ? tma_smem_desc(stageB(s) + 32u * j, 16u, 1024u)
                                        : tma_smem_desc(stageB(s) + 2048u * j, 8192u, 1024u);
                const uint32_t acc = (kt > 0 || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(empty(s))
                         : "memory");
        }
        vflags[2] = kt;
        // every MMA issued above is complete once `done` fires
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(done)
                     : "memory");
    }
    __syncthreads();
    bool ok = tc_wait(done, 0);  // full limit: the accumulator is read (or freed) only after the MMAs
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
    if (threadIdx.x == 0) {
        // loads issued but never consumed must land before the block exits
        const int issued = vflags[1], consumed = vflags[2];
        for (int kt = consumed; kt < issued; ++kt)
            if (!tc_wait(full(kt % kTmaStages), (kt / kTmaStages) & 1)) ok = false;
    }
    const bool good = __syncthreads_and(ok && vflags[0] == 0 && vflags[2] == nk);
    if (!good) {
        if (threadIdx.x == 0) atomicExch(&g_tc_gemm_error, 1u);
    } else {
        const int row = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 32) {
            uint32_t v[32];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                  "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                  "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            const int col0 = n0 + c0;
#pragma unroll
            for (int j = 0; j < 32; j += 2) {
                float v0 = __uint_as_float(v[j]), v1 = __uint_as_float(v[j + 1]);
                if (EPI == EPI_BIAS_RELU || EPI == EPI_BIAS_F32) {
                    v0 += bias[col0 + j];
                    v1 += bias[col0 + j + 1];
                }
                if (EPI == EPI_BIAS_RELU || EPI == EPI_BF16) {
                    __nv_bfloat162 o;
                    o.x = __float2bfloat16(EPI == EPI_BIAS_RELU ? fmaxf(v0, 0.f) : v0);
                    o.y = __float2bfloat16(EPI == EPI_BIAS_RELU ? fmaxf(v1, 0.f) : v1);
                    *reinterpret_cast<__nv_bfloat162*>(Cb + (size_t)row * ldc + col0 + j) = o;
                } else {
                    *reinterpret_cast<float2*>(Cf + (size_t)row * ldc + col0 + j) = make_float2(v0, v1);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN));
    (void)M;
    (void)N;
}

}  // namespace mlp
}  // namespace litho_b200
