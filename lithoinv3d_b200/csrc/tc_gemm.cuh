// BF16 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a) for the
// warm-start MLP: C[M x N] = A[M x K] . B[K x N] with the operand layouts,
// epilogues and size rules of k_gemm_bf16 (mlp_kernels.cuh), FP32
// accumulation in tensor memory.
//
// CTA: 128 threads, tile 128 x BN x 64 (BN = 256 when N allows, else 128),
// a ring of four (three) shared-memory stages filled by cp.async (16-byte
// chunks).  Each stage holds an operand tile in the
// tensor cores' no-swizzle canonical layout: 8-row x 16-byte core matrices,
// core matrices of consecutive 8-row (or 8-column) groups 128 bytes apart
// (stride byte offset), K blocks of 8 elements 16 x rows bytes apart
// (leading byte offset).  A K-contiguous operand is read K-major, an M- or
// N-contiguous one MN-major (the instruction descriptor's major bits), so no
// transposition is done in software.  One thread issues four
// tcgen05.mma (M = 128, N = BN, K = 16) per stage into a BN-column TMEM
// accumulator and commits them to the stage's mbarrier; the stage is
// refilled only after that mbarrier completes.  The epilogue reads the
// accumulator with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = rows),
// applies bias / ReLU and stores.  Every mbarrier wait is bounded: on
// expiry the kernel records an error flag, still waits (bounded) for its own
// MMAs and frees its tensor memory.
#pragma once
#include "mlp_kernels.cuh"

namespace litho_b200 {
namespace mlp {

constexpr int kTcBK = 64;
constexpr int kTcThreads = 128;
// Tile 128 x BN x 64 (BN = 128 or 256): operand tiles of 128 x 64 (A) and
// BN x 64 (B) bf16; stages and the TMEM accumulator sized by BN.
template <int BN>
struct TcShape {
    static constexpr int kStageA = kBM * kTcBK * 2;         // 16 KB
    static constexpr int kStageB = BN * kTcBK * 2;          // 16 or 32 KB
    static constexpr int kStages = BN == 128 ? 3 : 4;
    static constexpr int kSmem = kStages * (kStageA + kStageB);  // 96 KB (2 CTAs / SM) or 192 KB (1 CTA / SM)
    static constexpr uint32_t kTmemCols = BN;
};
constexpr long long kTcWaitLimit = 1ll << 24;   // mbarrier polls before a wait is abandoned

// Error flag set by a tensor-core GEMM whose mbarrier wait expired.
__device__ unsigned int g_tc_gemm_error = 0;
// Poll limit of the main loop's waits (a stage's MMAs done before the stage
// is refilled).  Host-settable (lf_set_device_wait_limit) so that the expiry
// path can be exercised: with 0 every such wait gives up at once.  The final
// wait for the CTA's own MMAs always uses kTcWaitLimit, so tensor memory is
// never freed while an MMA of the CTA may still write it.
__device__ long long g_tc_stage_wait_limit = kTcWaitLimit;

__device__ __forceinline__ uint64_t tc_smem_desc(uint32_t saddr, uint32_t lbo) {
    // start address >> 4 [0,14), leading byte offset >> 4 [16,30) (the K
    // step between 8-element blocks: 16 x the tile's rows), stride byte
    // offset 128 >> 4 [32,46), descriptor version 1 [46,48), base offset 0,
    // layout type 0 (no swizzle) [61,64)
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)(128u >> 4) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, major
// modes (0 K-major, 1 MN-major), N = BN, M = 128.
__host__ __device__ constexpr uint32_t tc_idesc(int a_mn_major, int b_mn_major, int bn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn_major << 15) | ((uint32_t)b_mn_major << 16) |
           ((uint32_t)(bn >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
}

// Non-blocking test of the mbarrier phase, polled with a short sleep: the
// wait gives up after kTcWaitLimit polls (well under a second).
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity, long long limit = kTcWaitLimit) {
    for (long long i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if (i > 64) __nanosleep(32);
    }
    return false;
}

// One operand tile (ROWS of the output dimension x 64 of K) into a stage.
// Chunk c (16 bytes) lands at byte 16 c of the stage, so the cp.async
// writes of a warp are contiguous (no bank conflicts):
//   K_CONTIG (stored [rows][K], K-major tile): c = kc * ROWS + r, i.e. K
//     chunk kc of row r at kc * 16 ROWS + (r / 8) * 128 + (r % 8) * 16;
//   else (stored [K][rows], MN-major tile): c = ((k / 8) * G + g) * 8 + k % 8
//     with G = ROWS / 8 groups, i.e. group g at depth k at
//     (k / 8) * 16 ROWS + g * 128 + (k % 8) * 16.
template <bool K_CONTIG, int ROWS>
__device__ __forceinline__ void tc_load_tile(uint8_t* stage, const __nv_bfloat16* __restrict__ g, int ld, int r0,
                                             int k0) {
    constexpr int G = ROWS / 8;
#pragma unroll
    for (int i = 0; i < ROWS * 8 / kTcThreads; ++i) {
        const int c = i * kTcThreads + (int)threadIdx.x;
        if (K_CONTIG) {
            const int kc = c / ROWS, r = c % ROWS;
            cp_async16(stage + c * 16, g + (size_t)(r0 + r) * ld + k0 + kc * 8);
        } else {
            const int k = ((c / (8 * G)) << 3) | (c & 7), grp = (c >> 3) % G;
            cp_async16(stage + c * 16, g + (size_t)(k0 + k) * ld + r0 + grp * 8);
        }
    }
}

template <bool A_T, bool B_T, int EPI, int BN>
__global__ void __launch_bounds__(kTcThreads) k_gemm_tc(int M, int N, int K, const __nv_bfloat16* __restrict__ A,
                                                       int lda, const __nv_bfloat16* __restrict__ B, int ldb,
                                                       const float* __restrict__ bias, float* __restrict__ Cf,
                                                       __nv_bfloat16* __restrict__ Cb, int ldc) {
    using Sh = TcShape<BN>;
    constexpr int kTcStages = Sh::kStages;
    constexpr uint32_t kTcTmemCols = Sh::kTmemCols;
    // stage s: A tile then B tile
    extern __shared__ __align__(1024) uint8_t tc_smem[];
    __shared__ __align__(8) uint64_t mbar[kTcStages];
    __shared__ uint32_t tmem_slot;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * BN;
    auto stageA = [&](int st) { return tc_smem + st * (Sh::kStageA + Sh::kStageB); };
    auto stageB = [&](int st) { return tc_smem + st * (Sh::kStageA + Sh::kStageB) + Sh::kStageA; };
    auto bar = [&](int st) { return smem_addr(&mbar[st]); };

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(kTcTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (threadIdx.x == 0) {
        for (int st = 0; st < kTcStages; ++st) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar(st)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
    const uint32_t tmem = tmem_slot;
    constexpr uint32_t idesc = tc_idesc(A_T ? 1 : 0, B_T ? 0 : 1, BN);
    constexpr uint32_t lboA = kBM * 16, lboB = BN * 16;

    const int nk = K / kTcBK;
    bool ok = true;
    int last = -1;  // last iteration whose MMAs were committed (block-uniform)
    // prologue: the first kTcStages - 1 stages
    for (int p = 0; p < kTcStages - 1; ++p) {
        if (p < nk) {
            tc_load_tile<!A_T, kBM>(stageA(p), A, lda, m0, p * kTcBK);
            tc_load_tile<B_T, BN>(stageB(p), B, ldb, n0, p * kTcBK);
        }
        cp_async_commit();
    }
    for (int kt = 0; kt < nk; ++kt) {
        const int cur = kt % kTcStages;
        asm volatile("cp.async.wait_group %0;\n" ::"n"(kTcStages - 2));  // stage kt has landed
        // this thread's shared-memory writes -> the tensor cores' (async) proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::);
            const uint32_t a0 = smem_addr(stageA(cur)), b0 = smem_addr(stageB(cur));
#pragma unroll
            for (int s = 0; s < kTcBK / 16; ++s) {
                const uint64_t ad = tc_smem_desc(a0 + s * 2 * lboA, lboA), bd = tc_smem_desc(b0 + s * 2 * lboB, lboB);
                const uint32_t acc = (kt > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                    ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar(cur))
                         : "memory");
        }
        last = kt;
        // refill the stage the MMAs of iteration kt - 1 read, once they are done
        const int nxt = kt + kTcStages - 1;
        if (nxt < nk) {
            if (kt >= 1) {
                const int prev = (kt - 1) % kTcStages;
                if (ok && !tc_wait(bar(prev), ((kt - 1) / kTcStages) & 1, g_tc_stage_wait_limit)) ok = false;
            }
            if (!__syncthreads_and(ok)) {
                ok = false;
                break;
            }
            tc_load_tile<!A_T, kBM>(stageA(nxt % kTcStages), A, lda, m0, nxt * kTcBK);
            tc_load_tile<B_T, BN>(stageB(nxt % kTcStages), B, ldb, n0, nxt * kTcBK);
        }
        cp_async_commit();
    }
    cp_async_wait_all();  // no copy may land after an early exit
    // every MMA of this CTA has completed once the last commit has
    if (last >= 0 && !tc_wait(bar(last % kTcStages), (last / kTcStages) & 1)) ok = false;
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
    if (!__syncthreads_and(ok)) {
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
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols));
    (void)M;
    (void)N;
}



}  // namespace mlp
}  // namespace litho_b200
