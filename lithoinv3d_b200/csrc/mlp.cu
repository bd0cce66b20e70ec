// Warm-start MLP: training and inference on the device with the BF16
// tensor-core kernels of mlp_kernels.cuh.  No reference counterpart (the
// reference's L-BFGS-B starts from the model's own parameters with a
// steepest-descent first step, lbfgsb_optimizer.cpp:35-38, 162).
//
// Network: n_in -> width (ReLU) x depth -> n_out, fp32 master weights with
// Adam, bf16 copies for the GEMMs, fp32 accumulation.  Layer widths are
// padded to multiples of 128 (the GEMM tile); padded output columns carry
// zero targets and are masked out of the loss.
#include "../../include/litho_gpu.h"
#include "mlp_kernels.cuh"
#include "tc_gemm.cuh"
#include "tc_gemm_tma.cuh"

#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

using namespace litho_b200::mlp;

namespace {

int cdiv_i(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }
int pad128(int n) { return cdiv_i(n, 128) * 128; }

template <typename T>
struct Buf {
    T* p = nullptr;
    size_t n = 0;
    Buf() = default;
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
    Buf(Buf&& o) noexcept : p(o.p), n(o.n) {
        o.p = nullptr;
        o.n = 0;
    }
    ~Buf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t count) {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) {
            n = count;
            e = cudaMemset(p, 0, std::max<size_t>(count, 1) * sizeof(T));
        }
        return e;
    }
};

struct Layer {
    int in = 0, out = 0;  // padded dims
    Buf<float> w, b, gw, gb, mw, vw, mb, vb;
    Buf<__nv_bfloat16> wb;  // bf16 copy [out][in]
    Buf<__nv_bfloat16> act;  // bf16 output activation [batch][out] (hidden layers)
};

}  // namespace

struct lf_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    int n_in = 0, n_in_pad = 0, width = 0, depth = 0, n_out = 0, n_out_pad = 0, batch = 0;
    std::vector<Layer> layers;  // depth hidden + 1 output
    Buf<__nv_bfloat16> xb, dz, dh;  // input, gradient buffers (bf16)
    Buf<float> pred, loss_blocks;
    int step = 0;
    int engine = LF_GEMM_AUTO;  // lf_mlp_set_engine: per GEMM, TMA-fed tcgen05 for deep K, mma.sync otherwise
    std::string err;
};

#define MLP_TRY(m, expr)                                                       \
    do {                                                                       \
        cudaError_t e_ = (expr);                                               \
        if (e_ != cudaSuccess) {                                               \
            (m)->err = std::string(#expr) + ": " + cudaGetErrorString(e_);     \
            return LF_ECUDA;                                                   \
        }                                                                      \
    } while (0)

static lf_status mlp_check_launch(lf_mlp* m) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        m->err = std::string("kernel launch: ") + cudaGetErrorString(e);
        return LF_ECUDA;
    }
    return LF_OK;
}

// One GEMM on `stream`: the tcgen05 kernel (K a multiple of 64; 128 x 256
// tiles when N allows, else 128 x 128) or the warp-level mma.sync kernel
// (K a multiple of 32).
template <bool A_T, bool B_T, int EPI, int BN>
static cudaError_t gemm_tc(cudaStream_t stream, int M, int N, int K, const __nv_bfloat16* A, int lda,
                           const __nv_bfloat16* B, int ldb, const float* bias, float* Cf, __nv_bfloat16* Cb, int ldc) {
    static bool attr = false;  // per instantiation, per process (the attribute is per function)
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_gemm_tc<A_T, B_T, EPI, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             TcShape<BN>::kSmem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    dim3 grid(N / BN, M / kBM);
    k_gemm_tc<A_T, B_T, EPI, BN><<<grid, kTcThreads, TcShape<BN>::kSmem, stream>>>(M, N, K, A, lda, B, ldb, bias, Cf,
                                                                                  Cb, ldc);
    return cudaPeekAtLastError();  // left for the caller's launch check
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library does not link the driver library itself).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// 2-D tensor map of a row-major bf16 array [rows][cols] with row length ld
// (elements): boxes of 64 columns x box_rows rows, 128-byte swizzle.
static bool bf16_map(CUtensorMap* map, const void* base, int rows, int cols, int ld, int box_rows) {
    const auto encode = tensor_map_encoder();
    if (!encode) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {64u, (cuuint32_t)box_rows};
    const cuuint32_t elem[2] = {1u, 1u};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, elem,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// One GEMM on the TMA-fed, warp-specialised tcgen05 kernel (tc_gemm_tma.cuh).
template <bool A_T, bool B_T, int EPI, int BN>
static cudaError_t gemm_tma(cudaStream_t stream, int M, int N, int K, const __nv_bfloat16* A, int lda,
                            const __nv_bfloat16* B, int ldb, const float* bias, float* Cf, __nv_bfloat16* Cb, int ldc) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_gemm_tma<A_T, B_T, EPI, BN>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, TmaShape<BN>::kSmem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    CUtensorMap mapA, mapB;
    const bool okA = A_T ? bf16_map(&mapA, A, K, M, lda, 64) : bf16_map(&mapA, A, M, K, lda, kBM);
    const bool okB = B_T ? bf16_map(&mapB, B, N, K, ldb, BN) : bf16_map(&mapB, B, K, N, ldb, 64);
    if (!okA || !okB) return cudaErrorInvalidValue;
    dim3 grid(N / BN, M / kBM);
    k_gemm_tma<A_T, B_T, EPI, BN><<<grid, kTmaThreads, TmaShape<BN>::kSmem, stream>>>(M, N, K, mapA, mapB, bias, Cf,
                                                                                     Cb, ldc);
    return cudaPeekAtLastError();
}

// LF_GEMM_AUTO: the TMA-fed tcgen05 kernel for deep reductions, where its
// pipeline pays (measured on B200: 24.7 against 12.2 TFLOP/s at K = 8192 on
// the network's 256 x 512 first layer, 757 against 290 at 4096^3), the
// mma.sync kernel for the shallow ones (81 against 52 TFLOP/s at K = 256,
// 14.0 against 8.9 at K = 512).
constexpr int kAutoTmaMinK = 2048;
static int auto_engine(int K) { return K >= kAutoTmaMinK && K % kTcBK == 0 ? LF_GEMM_TCGEN05_TMA : LF_GEMM_MMA_SYNC; }

template <bool A_T, bool B_T, int EPI>
static cudaError_t gemm_on(int engine, cudaStream_t stream, int M, int N, int K, const __nv_bfloat16* A, int lda,
                           const __nv_bfloat16* B, int ldb, const float* bias, float* Cf, __nv_bfloat16* Cb, int ldc) {
    if (engine == LF_GEMM_AUTO) engine = auto_engine(K);
    if (engine == LF_GEMM_TCGEN05_TMA) {
        if (N % 256 == 0)
            return gemm_tma<A_T, B_T, EPI, 256>(stream, M, N, K, A, lda, B, ldb, bias, Cf, Cb, ldc);
        return gemm_tma<A_T, B_T, EPI, 128>(stream, M, N, K, A, lda, B, ldb, bias, Cf, Cb, ldc);
    }
    if (engine == LF_GEMM_TCGEN05) {
        if (N % 256 == 0)
            return gemm_tc<A_T, B_T, EPI, 256>(stream, M, N, K, A, lda, B, ldb, bias, Cf, Cb, ldc);
        return gemm_tc<A_T, B_T, EPI, 128>(stream, M, N, K, A, lda, B, ldb, bias, Cf, Cb, ldc);
    }
    dim3 grid(N / kBN, M / kBM);
    k_gemm_bf16<A_T, B_T, EPI><<<grid, kGemmThreads, 0, stream>>>(M, N, K, A, lda, B, ldb, bias, Cf, Cb, ldc);
    return cudaPeekAtLastError();  // left for the caller's launch check
}

template <bool A_T, bool B_T, int EPI>
static void gemm(lf_mlp* m, int M, int N, int K, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb,
                 const float* bias, float* Cf, __nv_bfloat16* Cb, int ldc) {
    cudaError_t e = gemm_on<A_T, B_T, EPI>(m->engine, m->stream, M, N, K, A, lda, B, ldb, bias, Cf, Cb, ldc);
    if (e != cudaSuccess && m->err.empty()) m->err = std::string("gemm launch: ") + cudaGetErrorString(e);
}

// Reads and clears the tensor-core GEMM error flag (an mbarrier wait that
// expired); synchronises the stream.
static lf_status tc_check(lf_mlp* m) {
    unsigned int flag = 0;
    MLP_TRY(m, cudaMemcpyFromSymbolAsync(&flag, g_tc_gemm_error, sizeof(flag), 0, cudaMemcpyDeviceToHost, m->stream));
    MLP_TRY(m, cudaStreamSynchronize(m->stream));
    if (flag) {
        const unsigned int zero = 0;
        MLP_TRY(m, cudaMemcpyToSymbol(g_tc_gemm_error, &zero, sizeof(zero)));
        m->err = "tensor-core GEMM: an mbarrier wait expired";
        return LF_ETIMEOUT;
    }
    return LF_OK;
}

extern "C" lf_status lf_mlp_create(int device, int n_in, int width, int depth, int n_out, int batch, unsigned seed,
                                   lf_mlp** out) {
    if (!out) return LF_EINVAL;
    *out = nullptr;
    if (n_in <= 0 || width <= 0 || width % 128 != 0 || depth < 1 || n_out <= 0 || batch <= 0 || batch % 128 != 0)
        return LF_EINVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return LF_ECUDA;
    }
    auto* m = new (std::nothrow) lf_mlp();
    if (!m) return LF_ENOMEM;
    m->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete m;
        return LF_ECUDA;
    }
    m->n_in = n_in;
    m->n_in_pad = pad128(n_in);
    m->width = pad128(width);
    m->depth = depth;
    m->n_out = n_out;
    m->n_out_pad = pad128(n_out);
    m->batch = batch;
    m->layers.resize(depth + 1);
    std::mt19937_64 rng(seed);
    lf_status st = LF_OK;
    for (int l = 0; l <= depth && st == LF_OK; ++l) {
        Layer& L = m->layers[l];
        L.in = l == 0 ? m->n_in_pad : m->width;
        L.out = l == depth ? m->n_out_pad : m->width;
        const int in_real = l == 0 ? n_in : width, out_real = l == depth ? n_out : width;
        const size_t nw = (size_t)L.in * L.out;
        // He initialisation for ReLU layers (N(0, 2/fan_in)); the output layer
        // starts small; padded rows/columns stay zero
        std::vector<float> w(nw, 0.f);
        std::normal_distribution<float> nd(0.f, std::sqrt(2.f / in_real) * (l == depth ? 0.1f : 1.f));
        for (int o = 0; o < out_real; ++o)
            for (int i = 0; i < in_real; ++i) w[(size_t)o * L.in + i] = nd(rng);
        std::vector<__nv_bfloat16> wb(nw);
        for (size_t i = 0; i < nw; ++i) wb[i] = __float2bfloat16(w[i]);
        cudaError_t e = cudaSuccess;
        for (Buf<float>* b : {&L.w, &L.gw, &L.mw, &L.vw})
            if (e == cudaSuccess) e = b->alloc(nw);
        for (Buf<float>* b : {&L.b, &L.gb, &L.mb, &L.vb})
            if (e == cudaSuccess) e = b->alloc(L.out);
        if (e == cudaSuccess) e = L.wb.alloc(nw);
        if (e == cudaSuccess && l < depth) e = L.act.alloc((size_t)batch * L.out);
        if (e == cudaSuccess) e = cudaMemcpy(L.w.p, w.data(), nw * sizeof(float), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(L.wb.p, wb.data(), nw * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) st = LF_ECUDA;
    }
    if (st == LF_OK) {
        const int widest = std::max(std::max(m->n_in_pad, m->width), m->n_out_pad);
        if (m->xb.alloc((size_t)batch * m->n_in_pad) != cudaSuccess ||
            m->dz.alloc((size_t)batch * widest) != cudaSuccess || m->dh.alloc((size_t)batch * widest) != cudaSuccess ||
            m->pred.alloc((size_t)batch * m->n_out_pad) != cudaSuccess ||
            m->loss_blocks.alloc(cdiv_i((long long)batch * m->n_out_pad, 256)) != cudaSuccess)
            st = LF_ECUDA;
    }
    if (st != LF_OK) {
        cudaStreamDestroy(m->stream);
        delete m;
        return st;
    }
    *out = m;
    return LF_OK;
}

extern "C" void lf_mlp_destroy(lf_mlp* m) {
    if (!m) return;
    cudaSetDevice(m->device);
    cudaStreamSynchronize(m->stream);
    cudaStreamDestroy(m->stream);
    delete m;
}

extern "C" const char* lf_mlp_last_error(lf_mlp* m) { return m ? m->err.c_str() : "null network"; }

// Input rows [rows][n_in] fp32 (device) -> padded bf16 [batch][n_in_pad].
static lf_status load_input(lf_mlp* m, const float* d_x, int rows) {
    MLP_TRY(m, cudaMemsetAsync(m->xb.p, 0, sizeof(__nv_bfloat16) * m->xb.n, m->stream));
    if (m->n_in == m->n_in_pad) {
        const size_t n = (size_t)rows * m->n_in;
        k_to_bf16<<<cdiv_i(n, 256), 256, 0, m->stream>>>(n, d_x, m->xb.p);
    } else {
        for (int r = 0; r < rows; ++r)
            k_to_bf16<<<cdiv_i(m->n_in, 256), 256, 0, m->stream>>>(m->n_in, d_x + (size_t)r * m->n_in,
                                                                    m->xb.p + (size_t)r * m->n_in_pad);
    }
    return mlp_check_launch(m);
}

static lf_status forward(lf_mlp* m) {
    const __nv_bfloat16* x = m->xb.p;
    for (int l = 0; l <= m->depth; ++l) {
        Layer& L = m->layers[l];
        if (l < m->depth) {
            gemm<false, true, EPI_BIAS_RELU>(m, m->batch, L.out, L.in, x, L.in, L.wb.p, L.in, L.b.p, nullptr, L.act.p,
                                            L.out);
            x = L.act.p;
        } else {
            gemm<false, true, EPI_BIAS_F32>(m, m->batch, L.out, L.in, x, L.in, L.wb.p, L.in, L.b.p, m->pred.p, nullptr,
                                           L.out);
        }
    }
    return mlp_check_launch(m);
}

// Loss and parameter gradients for one batch (targets [batch][n_out] fp32).
static lf_status backward(lf_mlp* m, const float* d_y, float* loss) {
    const size_t np = (size_t)m->batch * m->n_out_pad;
    const int nb = cdiv_i(np, 256);
    k_mse<<<nb, 256, 0, m->stream>>>(m->batch, m->n_out_pad, m->n_out, m->pred.p, d_y, m->n_out, m->dz.p,
                                     m->loss_blocks.p);
    for (int l = m->depth; l >= 0; --l) {
        Layer& L = m->layers[l];
        const __nv_bfloat16* xin = l == 0 ? m->xb.p : m->layers[l - 1].act.p;
        // dW [out][in] = dZ^T X: A = dZ stored [batch][out] = [K][M]; B = X [batch][in] = [K][N]
        gemm<true, false, EPI_F32>(m, L.out, L.in, m->batch, m->dz.p, L.out, xin, L.in, nullptr, L.gw.p, nullptr, L.in);
        k_colsum<<<cdiv_i(L.out, 128), 128, 0, m->stream>>>(m->batch, L.out, m->dz.p, L.gb.p);
        if (l > 0) {
            // dH [batch][in] = dZ W: A = dZ [batch][out], B = W [out][in] = [K][N]
            gemm<false, false, EPI_BF16>(m, m->batch, L.in, L.out, m->dz.p, L.out, L.wb.p, L.in, nullptr, nullptr,
                                         m->dh.p, L.in);
            const size_t n = (size_t)m->batch * L.in;
            k_relu_bwd<<<cdiv_i(n, 256), 256, 0, m->stream>>>(n, xin, m->dh.p);
            std::swap(m->dz.p, m->dh.p);
            std::swap(m->dz.n, m->dh.n);
        }
    }
    lf_status st = mlp_check_launch(m);
    if (st != LF_OK) return st;
    if (loss) {
        std::vector<float> lb(nb);
        MLP_TRY(m, cudaMemcpyAsync(lb.data(), m->loss_blocks.p, sizeof(float) * nb, cudaMemcpyDeviceToHost, m->stream));
        MLP_TRY(m, cudaStreamSynchronize(m->stream));
        double s = 0.0;
        for (float v : lb) s += v;
        *loss = static_cast<float>(s);
    }
    return LF_OK;
}

extern "C" lf_status lf_mlp_train_step(lf_mlp* m, const float* d_x, const float* d_y, float lr, float* loss) {
    if (!m || !d_x || !d_y || !(lr > 0.f)) return LF_EINVAL;
    cudaSetDevice(m->device);
    lf_status st = load_input(m, d_x, m->batch);
    if (st == LF_OK) st = forward(m);
    if (st == LF_OK) st = backward(m, d_y, loss);
    if (st != LF_OK) return st;
    ++m->step;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
    for (Layer& L : m->layers) {
        const size_t nw = (size_t)L.in * L.out;
        k_adam<<<cdiv_i(nw, 256), 256, 0, m->stream>>>(nw, L.w.p, L.gw.p, L.mw.p, L.vw.p, lr, b1, b2, eps, c1, c2,
                                                        L.wb.p);
        k_adam<<<cdiv_i(L.out, 256), 256, 0, m->stream>>>(L.out, L.b.p, L.gb.p, L.mb.p, L.vb.p, lr, b1, b2, eps, c1, c2,
                                                           nullptr);
    }
    st = mlp_check_launch(m);
    if (st == LF_OK && m->engine != LF_GEMM_MMA_SYNC) st = tc_check(m);
    return st;
}

extern "C" lf_status lf_mlp_predict(lf_mlp* m, const float* d_x, int rows, float* d_y) {
    if (!m || rows < 0 || (rows > 0 && (!d_x || !d_y))) return LF_EINVAL;
    cudaSetDevice(m->device);
    for (int r0 = 0; r0 < rows; r0 += m->batch) {
        const int nr = std::min(m->batch, rows - r0);
        lf_status st = load_input(m, d_x + (size_t)r0 * m->n_in, nr);
        if (st == LF_OK) st = forward(m);
        if (st != LF_OK) return st;
        MLP_TRY(m, cudaMemcpy2DAsync(d_y + (size_t)r0 * m->n_out, sizeof(float) * m->n_out, m->pred.p,
                                     sizeof(float) * m->n_out_pad, sizeof(float) * m->n_out, nr,
                                     cudaMemcpyDeviceToDevice, m->stream));
    }
    MLP_TRY(m, cudaStreamSynchronize(m->stream));
    return m->engine != LF_GEMM_MMA_SYNC ? tc_check(m) : LF_OK;
}

// Parameters in the unpadded order: for each layer W [out][in] then b [out].
static size_t param_count(const lf_mlp* m) {
    size_t n = 0;
    for (int l = 0; l <= m->depth; ++l) {
        const int in = l == 0 ? m->n_in : (m->width), out = l == m->depth ? m->n_out : m->width;
        n += (size_t)in * out + out;
    }
    return n;
}

extern "C" lf_status lf_mlp_param_count(lf_mlp* m, size_t* n) {
    if (!m || !n) return LF_EINVAL;
    *n = param_count(m);
    return LF_OK;
}

// which: 0 weights, 1 gradients of the last lf_mlp_gradients / train step.
static lf_status copy_params(lf_mlp* m, int which, float* host) {
    size_t k = 0;
    for (int l = 0; l <= m->depth; ++l) {
        Layer& L = m->layers[l];
        const int in = l == 0 ? m->n_in : m->width, out = l == m->depth ? m->n_out : m->width;
        const float* w = which == 0 ? L.w.p : L.gw.p;
        const float* b = which == 0 ? L.b.p : L.gb.p;
        MLP_TRY(m, cudaMemcpy2DAsync(host + k, sizeof(float) * in, w, sizeof(float) * L.in, sizeof(float) * in, out,
                                     cudaMemcpyDeviceToHost, m->stream));
        k += (size_t)in * out;
        MLP_TRY(m, cudaMemcpyAsync(host + k, b, sizeof(float) * out, cudaMemcpyDeviceToHost, m->stream));
        k += out;
    }
    MLP_TRY(m, cudaStreamSynchronize(m->stream));
    return LF_OK;
}

extern "C" lf_status lf_mlp_get_params(lf_mlp* m, float* host) {
    if (!m || !host) return LF_EINVAL;
    cudaSetDevice(m->device);
    return copy_params(m, 0, host);
}

extern "C" lf_status lf_mlp_set_params(lf_mlp* m, const float* host) {
    if (!m || !host) return LF_EINVAL;
    cudaSetDevice(m->device);
    size_t k = 0;
    for (int l = 0; l <= m->depth; ++l) {
        Layer& L = m->layers[l];
        const int in = l == 0 ? m->n_in : m->width, out = l == m->depth ? m->n_out : m->width;
        std::vector<float> w((size_t)L.in * L.out, 0.f);
        for (int o = 0; o < out; ++o)
            std::memcpy(&w[(size_t)o * L.in], host + k + (size_t)o * in, sizeof(float) * in);
        k += (size_t)in * out;
        std::vector<__nv_bfloat16> wb(w.size());
        for (size_t i = 0; i < w.size(); ++i) wb[i] = __float2bfloat16(w[i]);
        std::vector<float> b(L.out, 0.f);
        std::memcpy(b.data(), host + k, sizeof(float) * out);
        k += out;
        MLP_TRY(m, cudaMemcpy(L.w.p, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice));
        MLP_TRY(m, cudaMemcpy(L.wb.p, wb.data(), sizeof(__nv_bfloat16) * wb.size(), cudaMemcpyHostToDevice));
        MLP_TRY(m, cudaMemcpy(L.b.p, b.data(), sizeof(float) * b.size(), cudaMemcpyHostToDevice));
        for (Buf<float>* z : {&L.mw, &L.vw, &L.mb, &L.vb})
            MLP_TRY(m, cudaMemset(z->p, 0, sizeof(float) * z->n));
    }
    m->step = 0;
    return LF_OK;
}

// Loss and parameter gradients (no update) of one batch, gradients in the
// parameter order of lf_mlp_get_params.
extern "C" lf_status lf_mlp_gradients(lf_mlp* m, const float* d_x, const float* d_y, float* loss, float* host_grads) {
    if (!m || !d_x || !d_y) return LF_EINVAL;
    cudaSetDevice(m->device);
    lf_status st = load_input(m, d_x, m->batch);
    if (st == LF_OK) st = forward(m);
    if (st == LF_OK) st = backward(m, d_y, loss);
    if (st == LF_OK && m->engine != LF_GEMM_MMA_SYNC) st = tc_check(m);
    if (st == LF_OK && host_grads) st = copy_params(m, 1, host_grads);
    return st;
}

extern "C" lf_status lf_set_device_wait_limit(long long polls) {
    const long long v = polls < 0 ? kTcWaitLimit : polls;
    return cudaMemcpyToSymbol(g_tc_stage_wait_limit, &v, sizeof(v)) == cudaSuccess ? LF_OK : LF_ECUDA;
}

extern "C" lf_status lf_mlp_set_engine(lf_mlp* m, int engine) {
    if (!m || (engine != LF_GEMM_TCGEN05 && engine != LF_GEMM_MMA_SYNC && engine != LF_GEMM_TCGEN05_TMA &&
               engine != LF_GEMM_AUTO))
        return LF_EINVAL;
    m->engine = engine;
    return LF_OK;
}

extern "C" lf_status lf_gemm_bf16(int engine, int a_trans, int b_trans, int epilogue, int M, int N, int K,
                                  const void* A, int lda, const void* B, int ldb, const float* bias, void* C, int ldc,
                                  void* stream) {
    if (engine == LF_GEMM_AUTO && K > 0) engine = auto_engine(K);
    const bool tc = engine == LF_GEMM_TCGEN05 || engine == LF_GEMM_TCGEN05_TMA;
    if ((!tc && engine != LF_GEMM_MMA_SYNC) || M <= 0 || N <= 0 || K <= 0 || M % kBM ||
        N % kBN || K % (tc ? kTcBK : kBK) || !A || !B || !C ||
        (epilogue != EPI_F32 && epilogue != EPI_BF16 && epilogue != EPI_BIAS_RELU && epilogue != EPI_BIAS_F32) ||
        ((epilogue == EPI_BIAS_RELU || epilogue == EPI_BIAS_F32) && !bias) || lda % 8 || ldb % 8 || ldc % 2 ||
        (reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) % 16)
        return LF_EINVAL;
    // minimum row lengths of the stored operands
    if (lda < (a_trans ? M : K) || ldb < (b_trans ? K : N) || ldc < N) return LF_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const auto* a = static_cast<const __nv_bfloat16*>(A);
    const auto* b = static_cast<const __nv_bfloat16*>(B);
    float* cf = static_cast<float*>(C);
    __nv_bfloat16* cb = static_cast<__nv_bfloat16*>(C);
    cudaError_t e = cudaSuccess;
#define LF_GEMM_CASE(AT, BT)                                                                                          \
    if (!!a_trans == AT && !!b_trans == BT) {                                                                        \
        switch (epilogue) {                                                                                          \
        case EPI_F32: e = gemm_on<AT, BT, EPI_F32>(engine, st, M, N, K, a, lda, b, ldb, bias, cf, nullptr, ldc); break; \
        case EPI_BF16: e = gemm_on<AT, BT, EPI_BF16>(engine, st, M, N, K, a, lda, b, ldb, bias, nullptr, cb, ldc); break; \
        case EPI_BIAS_RELU:                                                                                          \
            e = gemm_on<AT, BT, EPI_BIAS_RELU>(engine, st, M, N, K, a, lda, b, ldb, bias, nullptr, cb, ldc);          \
            break;                                                                                                   \
        default: e = gemm_on<AT, BT, EPI_BIAS_F32>(engine, st, M, N, K, a, lda, b, ldb, bias, cf, nullptr, ldc); break; \
        }                                                                                                            \
    }
    LF_GEMM_CASE(false, false)
    LF_GEMM_CASE(false, true)
    LF_GEMM_CASE(true, false)
    LF_GEMM_CASE(true, true)
#undef LF_GEMM_CASE
    if (e != cudaSuccess) return LF_ECUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return LF_ECUDA;
    if (tc) {
        unsigned int flag = 0;
        if (cudaMemcpyFromSymbol(&flag, g_tc_gemm_error, sizeof(flag)) != cudaSuccess) return LF_ECUDA;
        if (flag) {
            const unsigned int zero = 0;
            cudaMemcpyToSymbol(g_tc_gemm_error, &zero, sizeof(zero));
            return LF_ETIMEOUT;
        }
    }
    return LF_OK;
}
