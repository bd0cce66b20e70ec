"""The warm-start network's GEMM on the 5th-generation tensor cores
(tcgen05.mma, accumulator in tensor memory) against an FP32 product of the
same BF16 operands and against the warp-level mma.sync kernel, for every
operand layout and epilogue the network uses.  Products of BF16 values are
exact in FP32, so the FP32 outputs differ from the reference product only by
the order of the FP32 sums (tolerance 2e-5 relative to the largest entry);
BF16 outputs by at most one BF16 rounding (tolerance 1e-2)."""
import ctypes as C

import numpy as np
import pytest

from lithoinv3d_b200 import _native

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TC, SYNC, TMA = 0, 1, 2
EPI_F32, EPI_BIAS_RELU, EPI_BIAS_F32, EPI_BF16 = 0, 1, 2, 3


def run(lib, engine, a_t, b_t, epi, A, B, bias, M, N, K):
    out_dtype = torch.bfloat16 if epi in (EPI_BIAS_RELU, EPI_BF16) else torch.float32
    Cm = torch.full((M, N), float("nan"), dtype=out_dtype, device="cuda")
    st = lib.lf_gemm_bf16(engine, a_t, b_t, epi, M, N, K, C.c_void_p(A.data_ptr()), A.shape[1],
                          C.c_void_p(B.data_ptr()), B.shape[1], C.cast(C.c_void_p(bias.data_ptr()), _native._dp),
                          C.c_void_p(Cm.data_ptr()), N, None)
    assert st == 0, _native.STATUS.get(st, st)
    return Cm.float()


@pytest.mark.parametrize("engine", [TC, TMA])
@pytest.mark.parametrize("a_t,b_t", [(0, 1), (1, 0), (0, 0), (1, 1)])
@pytest.mark.parametrize("epi", [EPI_F32, EPI_BIAS_RELU, EPI_BIAS_F32, EPI_BF16])
def test_tcgen05_gemm_matches_fp32_product(a_t, b_t, epi, engine):
    lib = _native.load()
    # N = 512 runs the 128 x 256 tiles, N = 384 the 128 x 128 ones
    M, N, K = 256, (512 if epi in (EPI_F32, EPI_BIAS_RELU) else 384), 576
    g = torch.Generator(device="cuda").manual_seed(17 + 4 * a_t + 2 * b_t + epi)
    Am = torch.randn(M, K, generator=g, device="cuda").bfloat16()
    Bm = torch.randn(K, N, generator=g, device="cuda").bfloat16()
    bias = torch.randn(N, generator=g, device="cuda")
    A = Am.t().contiguous() if a_t else Am
    B = Bm.t().contiguous() if b_t else Bm
    want = Am.float() @ Bm.float()
    if epi in (EPI_BIAS_RELU, EPI_BIAS_F32):
        want = want + bias
    if epi == EPI_BIAS_RELU:
        want = torch.relu(want)
    got = run(lib, engine, a_t, b_t, epi, A, B, bias, M, N, K)
    legacy = run(lib, SYNC, a_t, b_t, epi, A, B, bias, M, N, K)
    scale = float(want.abs().max())
    tol = 2e-5 if epi in (EPI_F32, EPI_BIAS_F32) else 1e-2
    assert torch.isfinite(got).all()
    assert float((got - want).abs().max()) <= tol * scale
    assert float((got - legacy).abs().max()) <= tol * scale


def test_tcgen05_gemm_rejects_bad_shapes():
    lib = _native.load()
    A = torch.zeros(128, 96, dtype=torch.bfloat16, device="cuda")  # K = 96: not a multiple of 64
    B = torch.zeros(96, 128, dtype=torch.bfloat16, device="cuda")
    Cm = torch.zeros(128, 128, device="cuda")
    st = lib.lf_gemm_bf16(TC, 0, 0, EPI_F32, 128, 128, 96, C.c_void_p(A.data_ptr()), 96, C.c_void_p(B.data_ptr()),
                          128, None, C.c_void_p(Cm.data_ptr()), 128, None)
    assert _native.STATUS[st] == "LF_EINVAL"


@pytest.mark.parametrize("engine", [TC, TMA])
def test_tcgen05_gemm_wait_expiry_reports_timeout_and_recovers(engine):
    """Failure detection without a fault: with the main-loop wait limit at 0
    every stage wait gives up at once, so the kernel abandons the product,
    drains its own MMAs, frees its tensor memory and raises the error flag;
    lf_gemm_bf16 returns LF_ETIMEOUT.  With the default limit restored the
    same call on the same device succeeds and is correct."""
    lib = _native.load()
    M, N, K = 256, 512, 576  # 9 K-blocks: more than the stage ring, so refill waits happen
    g = torch.Generator(device="cuda").manual_seed(5)
    Am = torch.randn(M, K, generator=g, device="cuda").bfloat16()
    Bm = torch.randn(K, N, generator=g, device="cuda").bfloat16()
    bias = torch.zeros(N, device="cuda")
    Cm = torch.full((M, N), float("nan"), dtype=torch.float32, device="cuda")

    def call():
        return lib.lf_gemm_bf16(engine, 0, 0, EPI_F32, M, N, K, C.c_void_p(Am.data_ptr()), K, C.c_void_p(Bm.data_ptr()),
                                N, C.cast(C.c_void_p(bias.data_ptr()), _native._dp), C.c_void_p(Cm.data_ptr()), N,
                                None)

    try:
        assert lib.lf_set_device_wait_limit(0) == 0
        assert call() == 5  # LF_ETIMEOUT
    finally:
        assert lib.lf_set_device_wait_limit(-1) == 0
    assert call() == 0
    ref = Am.float() @ Bm.float()
    assert float((Cm - ref).abs().max() / ref.abs().max()) < 2e-5
