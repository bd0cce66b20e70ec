// BF16 tensor-core kernels of the warm-start MLP (training and inference),
// FP32 accumulation.  No reference counterpart: the reference has no learned
// component.
//
// GEMM: C[M x N] = A[M x K] . B[K x N], bf16 operands, fp32 accumulators,
// mma.sync m16n8k16.  A is stored row-major [M][K] (A_T = false) or as its
// transpose [K][M] (A_T = true); B row-major [K][N] (B_T = false) or as [N][K]
// (B_T = true).  Tiles stay in the stored layout in shared memory and the
// fragments are read with ldmatrix, transposing on the fly where the stored
// layout differs from the fragment's -- so the forward Y = X W^T, the input
// gradient dX = dY W and the weight gradient dW = dY^T X use one kernel.
// CTA tile 128 x 128 x 32, 8 warps of 64 x 32, cp.async double buffering.
// M and N must be multiples of 128 and K of 32 (the network pads its
// layers); every operand row starts on a 16-byte boundary.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace litho_b200 {
namespace mlp {

constexpr int kBM = 128, kBN = 128, kBK = 32;
constexpr int kGemmThreads = 256;
// padded shared-memory row lengths (bf16 elements): +8 keeps ldmatrix rows
// on different banks and 16-byte aligned
constexpr int kRowMK = kBK + 8;    // tiles stored [128][32]
constexpr int kRowKM = kBM + 8;    // tiles stored [32][128]
constexpr int kTileElems = (kBM * kRowMK > kBK * kRowKM) ? kBM * kRowMK : kBK * kRowKM;

enum Epilogue {
    EPI_F32 = 0,        // C fp32
    EPI_BIAS_RELU = 1,  // bf16 relu(C + bias[n])
    EPI_BIAS_F32 = 2,   // fp32 C + bias[n]
    EPI_BF16 = 3,       // bf16 C
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(smem)), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::); }

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_addr(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_addr(p)));
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Loads one operand tile (128 rows of the M or N side x 32 of K) into shared
// memory in its stored layout.  TRANS = stored [K][MN]: 32 rows of 128.
template <bool TRANS>
__device__ __forceinline__ void load_tile(__nv_bfloat16* sm, const __nv_bfloat16* __restrict__ g, int ld, int mn0,
                                          int k0) {
    const int t = threadIdx.x;
    if (!TRANS) {  // [mn][k]: 128 rows x 4 chunks of 8
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int c = t + i * kGemmThreads, row = c >> 2, col = (c & 3) * 8;
            cp_async16(sm + row * kRowMK + col, g + (size_t)(mn0 + row) * ld + k0 + col);
        }
    } else {  // [k][mn]: 32 rows x 16 chunks of 8
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int c = t + i * kGemmThreads, row = c >> 4, col = (c & 15) * 8;
            cp_async16(sm + row * kRowKM + col, g + (size_t)(k0 + row) * ld + mn0 + col);
        }
    }
}

// lda / ldb: row lengths (elements) of A and B as stored.
template <bool A_T, bool B_T, int EPI>
__global__ void __launch_bounds__(kGemmThreads) k_gemm_bf16(int M, int N, int K, const __nv_bfloat16* __restrict__ A,
                                                            int lda, const __nv_bfloat16* __restrict__ B, int ldb,
                                                            const float* __restrict__ bias, float* __restrict__ Cf,
                                                            __nv_bfloat16* __restrict__ Cb, int ldc) {
    __shared__ __align__(16) __nv_bfloat16 sA[2][kTileElems];
    __shared__ __align__(16) __nv_bfloat16 sB[2][kTileElems];
    const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = (warp >> 2) * 64, wn = (warp & 3) * 32;  // warp tile origin in the CTA tile
    float acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[i][j][k] = 0.f;
    const int nk = K / kBK;
    load_tile<A_T>(sA[0], A, lda, m0, 0);
    load_tile<!B_T>(sB[0], B, ldb, n0, 0);
    cp_async_commit();
    const int r = lane & 7, mat = lane >> 3;  // ldmatrix: row within 8x8 matrix, matrix index
    for (int kt = 0; kt < nk; ++kt) {
        const int cur = kt & 1;
        if (kt + 1 < nk) {
            load_tile<A_T>(sA[cur ^ 1], A, lda, m0, (kt + 1) * kBK);
            load_tile<!B_T>(sB[cur ^ 1], B, ldb, n0, (kt + 1) * kBK);
            cp_async_commit();
            cp_async_wait_one();
        } else {
            cp_async_wait_all();
        }
        __syncthreads();
        const __nv_bfloat16* a = sA[cur];
        const __nv_bfloat16* b = sB[cur];
#pragma unroll
        for (int kk = 0; kk < kBK; kk += 16) {
            uint32_t af[4][4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int mrow = wm + i * 16;
                if (!A_T)  // stored [m][k]: matrices (m+0,k+0) (m+8,k+0) (m+0,k+8) (m+8,k+8)
                    ldsm_x4(af[i], a + (mrow + r + 8 * (mat & 1)) * kRowMK + kk + 8 * (mat >> 1));
                else  // stored [k][m], transposed on load
                    ldsm_x4_t(af[i], a + (kk + r + 8 * (mat >> 1)) * kRowKM + mrow + 8 * (mat & 1));
            }
            uint32_t bf[4][2];
#pragma unroll
            for (int j = 0; j < 4; j += 2) {
                const int ncol = wn + j * 8;
                uint32_t t4[4];
                if (B_T)  // stored [n][k]: matrices (n+0,k+0) (n+0,k+8) (n+8,k+0) (n+8,k+8)
                    ldsm_x4(t4, b + (ncol + r + 8 * (mat >> 1)) * kRowMK + kk + 8 * (mat & 1));
                else  // stored [k][n], transposed on load
                    ldsm_x4_t(t4, b + (kk + r + 8 * (mat & 1)) * kRowKM + ncol + 8 * (mat >> 1));
                bf[j][0] = t4[0]; bf[j][1] = t4[1];
                bf[j + 1][0] = t4[2]; bf[j + 1][1] = t4[3];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bf[j][0], bf[j][1]);
        }
        __syncthreads();
    }
    // epilogue: c0,c1 at (row g, cols 2q, 2q+1), c2,c3 at row g + 8
    const int g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int row = m0 + wm + i * 16 + g + 8 * h;
                const int col = n0 + wn + j * 8 + 2 * q;
                float v0 = acc[i][j][2 * h], v1 = acc[i][j][2 * h + 1];
                if (EPI == EPI_BIAS_RELU || EPI == EPI_BIAS_F32) {
                    v0 += bias[col];
                    v1 += bias[col + 1];
                }
                if (EPI == EPI_BIAS_RELU || EPI == EPI_BF16) {
                    __nv_bfloat162 o;
                    o.x = __float2bfloat16(EPI == EPI_BIAS_RELU ? fmaxf(v0, 0.f) : v0);
                    o.y = __float2bfloat16(EPI == EPI_BIAS_RELU ? fmaxf(v1, 0.f) : v1);
                    *reinterpret_cast<__nv_bfloat162*>(Cb + (size_t)row * ldc + col) = o;
                } else {
                    *reinterpret_cast<float2*>(Cf + (size_t)row * ldc + col) = make_float2(v0, v1);
                }
            }
    (void)M;
    (void)N;
}

// fp32 -> bf16, n elements.
__global__ void k_to_bf16(size_t n, const float* __restrict__ x, __nv_bfloat16* __restrict__ y) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16(x[i]);
}

// Loss: 0.5 * mean over (row, col < n_valid) of (pred - target)^2 with the
// gradient w.r.t. pred (bf16, padding columns zero) and per-block sums.
__global__ void k_mse(int rows, int cols, int n_valid, const float* __restrict__ pred, const float* __restrict__ target,
                      int ld_target, __nv_bfloat16* __restrict__ dpred, float* __restrict__ block_loss) {
    __shared__ float red[256];
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const float inv = 1.f / ((float)rows * (float)n_valid);
    float l = 0.f;
    if (i < (size_t)rows * cols) {
        const int r = (int)(i / cols), c = (int)(i % cols);
        float d = 0.f;
        if (c < n_valid) {
            d = pred[i] - target[(size_t)r * ld_target + c];
            l = 0.5f * d * d * inv;
        }
        dpred[i] = __float2bfloat16(d * inv);
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) block_loss[blockIdx.x] = red[0];
}

// ReLU backward in place on the bf16 gradient: dz = dy * (y > 0).
__global__ void k_relu_bwd(size_t n, const __nv_bfloat16* __restrict__ y, __nv_bfloat16* __restrict__ dy) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n && !(__bfloat162float(y[i]) > 0.f)) dy[i] = __float2bfloat16(0.f);
}

// Bias gradient: column sums of dY [rows][cols] (bf16), fp32 out.
__global__ void k_colsum(int rows, int cols, const __nv_bfloat16* __restrict__ dy, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.f;
    for (int r = 0; r < rows; ++r) s += __bfloat162float(dy[(size_t)r * cols + c]);
    out[c] = s;
}

// Adam on fp32 master weights (Kingma & Ba, 2015, with bias correction
// c1 = 1 - b1^t, c2 = 1 - b2^t); refreshes the bf16 copy wb when given.
__global__ void k_adam(size_t n, float* __restrict__ w, const float* __restrict__ gw, float* __restrict__ m1,
                       float* __restrict__ m2, float lr, float b1, float b2, float eps, float c1, float c2,
                       __nv_bfloat16* __restrict__ wb) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = gw[i];
    const float a = b1 * m1[i] + (1.f - b1) * g, b = b2 * m2[i] + (1.f - b2) * g * g;
    m1[i] = a;
    m2[i] = b;
    const float v = w[i] - lr * (a / c1) / (sqrtf(b / c2) + eps);
    w[i] = v;
    if (wb) wb[i] = __float2bfloat16(v);
}

}  // namespace mlp
}  // namespace litho_b200
