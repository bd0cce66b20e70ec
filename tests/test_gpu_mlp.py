"""Warm-start MLP kernels (BF16 tensor-core GEMMs, FP32 accumulation): loss
and every parameter gradient against a CPU FP64 restatement of the same
network that rounds to bf16 at the same points (inputs, weights, hidden
activations, output gradient, back-propagated activation gradients); and
training on a learnable map.  Tolerance: norm-wise relative 2e-3 per
gradient block (the device accumulates in fp32)."""
import ctypes as C

import numpy as np
import pytest

from lithoinv3d_b200 import _native

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def bf16(a):
    """Round to bfloat16 (nearest even), returned as float64."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


class Net:
    def __init__(self, n_in, width, depth, n_out, batch, seed=1):
        self.lib = _native.load()
        self.h = C.c_void_p()
        st = self.lib.lf_mlp_create(0, n_in, width, depth, n_out, batch, seed, C.byref(self.h))
        assert st == 0, st
        self.dims = [n_in] + [width] * depth + [n_out]
        n = C.c_size_t()
        self.lib.lf_mlp_param_count(self.h, C.byref(n))
        self.np = n.value
        self.batch = batch

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.lf_mlp_destroy(self.h)

    def params(self):
        p = np.zeros(self.np, np.float32)
        assert self.lib.lf_mlp_get_params(self.h, p.ctypes.data) == 0
        return p

    def unpack(self, flat):
        out, k = [], 0
        for a, b in zip(self.dims[:-1], self.dims[1:]):
            W = flat[k:k + a * b].reshape(b, a)
            k += a * b
            out.append((W, flat[k:k + b]))
            k += b
        return out

    def gradients(self, x, y):
        dx, dy = torch.tensor(x, dtype=torch.float32, device="cuda"), torch.tensor(y, dtype=torch.float32, device="cuda")
        g = np.zeros(self.np, np.float32)
        loss = C.c_float()
        st = self.lib.lf_mlp_gradients(self.h, dx.data_ptr(), dy.data_ptr(), C.byref(loss), g.ctypes.data)
        assert st == 0, self.lib.lf_mlp_last_error(self.h)
        return loss.value, g


def reference(layers, x, y):
    """FP64 forward/backward with bf16 rounding at the device's points."""
    rows, n_out = y.shape
    h = bf16(x)
    acts = [h]
    for W, b in layers[:-1]:
        h = bf16(np.maximum(h @ bf16(W).T + b, 0.0))
        acts.append(h)
    W, b = layers[-1]
    pred = h @ bf16(W).T + b
    inv = 1.0 / (rows * n_out)
    loss = 0.5 * np.sum((pred - y) ** 2) * inv
    dz = bf16((pred - y) * inv)
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, b = layers[l]
        grads[l] = (dz.T @ acts[l], dz.sum(axis=0))
        if l > 0:
            dh = bf16(dz @ bf16(W))
            dz = np.where(acts[l] > 0, dh, 0.0)
    return loss, grads


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


# LF_GEMM_TCGEN05, LF_GEMM_MMA_SYNC, LF_GEMM_TCGEN05_TMA, LF_GEMM_AUTO (the 2048-input case puts the
# first layer's reduction on the TMA kernel under AUTO)
@pytest.mark.parametrize("engine", [0, 1, 2, 3])
@pytest.mark.parametrize("n_in,width,depth,n_out", [(256, 128, 2, 70), (384, 256, 3, 200), (2048, 128, 2, 70)])
def test_mlp_gradients_match_cpu(n_in, width, depth, n_out, engine):
    batch = 128
    net = Net(n_in, width, depth, n_out, batch, seed=3)
    assert net.lib.lf_mlp_set_engine(net.h, engine) == 0
    rng = np.random.default_rng(4)
    x = rng.normal(size=(batch, n_in)).astype(np.float32)
    y = rng.normal(size=(batch, n_out)).astype(np.float32)
    layers = net.unpack(net.params().astype(np.float64))
    loss, g = net.gradients(x, y)
    rloss, rgrads = reference(layers, x.astype(np.float64), y.astype(np.float64))
    assert abs(loss - rloss) <= 2e-3 * rloss
    for (gW, gb), (rW, rb) in zip(net.unpack(g.astype(np.float64)), rgrads):
        assert rel(gW, rW) < 2e-3
        assert rel(gb, rb) < 2e-3


def test_mlp_learns_a_linear_map():
    n_in, n_out, batch = 256, 64, 256
    net = Net(n_in, 256, 2, n_out, batch, seed=5)
    rng = np.random.default_rng(6)
    A = rng.normal(size=(n_out, n_in)) / np.sqrt(n_in)
    x = torch.tensor(rng.normal(size=(batch, n_in)), dtype=torch.float32, device="cuda")
    y = x @ torch.tensor(A.T, dtype=torch.float32, device="cuda")
    loss = C.c_float()
    losses = []
    for _ in range(300):
        assert net.lib.lf_mlp_train_step(net.h, x.data_ptr(), y.data_ptr(), 1e-3, C.byref(loss)) == 0
        losses.append(loss.value)
    assert losses[-1] < 0.05 * losses[0]
    # predict reproduces the trained forward
    out = torch.zeros_like(y)
    assert net.lib.lf_mlp_predict(net.h, x.data_ptr(), batch, out.data_ptr()) == 0
    err = float(((out - y) ** 2).mean()) * 0.5
    assert err < 0.1 * losses[0]
