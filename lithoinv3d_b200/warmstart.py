"""Learned warm start for the L-BFGS-B inversion (no reference counterpart:
the reference starts LBFGSBOptimizer::minimize from the model's current
parameters with a steepest-descent first step, lbfgsb_optimizer.cpp:35-38,
162).

A ReLU MLP (lf_mlp_*: hand-written BF16 tensor-core kernels, FP32
accumulate) maps the data residual of the starting model -- gz and TMI on
the station grid, each channel scaled by a fixed RMS -- to the DOF update
that explains it.  Training pairs come from the GPU forward itself: seeded
smooth perturbations of the starting model (sums of Gaussian bumps in z)
and the residuals they cause.  At inversion time the network proposes the
start x_s = x0 + update, refines it by applying itself to the residual at
x_s (a learned Gauss-Newton step, kept only if the misfit drops), and, from
the secant pair s = x_s - x0, y = g(x_s) - g(x0), sets the initial
inverse-Hessian scale gamma_0 = s.y / y.y.
The analytic objective stays the judge: when f(x_s) >= f(x0) the plain
start is used.

    python -m lithoinv3d_b200.warmstart [--pairs N] [--heldout M] ...

runs the whole experiment on the config-2 family and prints one JSON line.
Device buffers are torch tensors (plumbing only; every computation is the
library's)."""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time
from typing import Optional

import numpy as np

from . import _native
from .api import COLLAPSED_DROP, GATHER_CHAIN, PREC_MIXED


class Network:
    """The lf_mlp network (width and batch multiples of 128)."""

    def __init__(self, n_in: int, n_out: int, width: int = 512, depth: int = 4, batch: int = 256, seed: int = 0,
                 device: int = 0):
        self.lib = _native.load()
        self.h = C.c_void_p()
        st = self.lib.lf_mlp_create(device, n_in, width, depth, n_out, batch, seed, C.byref(self.h))
        if st != 0:
            raise RuntimeError(f"lf_mlp_create failed ({st})")
        self.n_in, self.n_out, self.batch = n_in, n_out, batch

    def close(self):
        if getattr(self, "h", None):
            self.lib.lf_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _err(self, st, what):
        if st != 0:
            raise RuntimeError(f"{what}: {self.lib.lf_mlp_last_error(self.h).decode()}")

    def train(self, X, Y, epochs: int, lr: float, rng: np.random.Generator, lr_decay: float = 0.97):
        """X [N][n_in], Y [N][n_out]: float32 CUDA tensors.  Returns the mean
        loss of every epoch."""
        import torch

        n = X.shape[0]
        nb = n // self.batch
        losses = []
        loss = C.c_float()
        for e in range(epochs):
            perm = torch.as_tensor(rng.permutation(n), device=X.device)
            tot = 0.0
            for b in range(nb):
                idx = perm[b * self.batch:(b + 1) * self.batch]
                xb, yb = X[idx].contiguous(), Y[idx].contiguous()
                self._err(self.lib.lf_mlp_train_step(self.h, xb.data_ptr(), yb.data_ptr(), float(lr), C.byref(loss)),
                          "train_step")
                tot += loss.value
            losses.append(tot / max(nb, 1))
            lr *= lr_decay
        return losses

    def predict(self, X):
        import torch

        out = torch.zeros((X.shape[0], self.n_out), dtype=torch.float32, device=X.device)
        self._err(self.lib.lf_mlp_predict(self.h, X.contiguous().data_ptr(), X.shape[0], out.data_ptr()), "predict")
        return out

    def predict_one(self, feat: np.ndarray) -> np.ndarray:
        """One input row (host) -> one output row (host), through reused
        pinned host and device buffers."""
        import torch

        if getattr(self, "_io", None) is None:
            self._io = (torch.zeros(self.n_in, dtype=torch.float32).pin_memory(),
                        torch.zeros(self.n_out, dtype=torch.float32).pin_memory(),
                        torch.zeros(self.n_in, dtype=torch.float32, device="cuda"),
                        torch.zeros(self.n_out, dtype=torch.float32, device="cuda"))
        hin, hout, din, dout = self._io
        hin.numpy()[:] = feat
        din.copy_(hin)
        torch.cuda.synchronize()
        self._err(self.lib.lf_mlp_predict(self.h, din.data_ptr(), 1, dout.data_ptr()), "predict")
        hout.copy_(dout)
        return hout.numpy().copy()

    def zero_response(self) -> np.ndarray:
        """Output at a zero input (cached; the refinement steps remove it)."""
        if getattr(self, "_zero", None) is None:
            self._zero = self.predict_one(np.zeros(self.n_in, np.float32))
        return self._zero


def dof_xy(model) -> np.ndarray:
    """(x, y) of each global DOF's first referenced vertex."""
    t = model.tables()
    pos = np.asarray(t["pos"]).reshape(-1, 3)
    return pos[np.asarray(t["ref_vertex"])[np.asarray(t["dof_off"])[:-1]], :2]


def dof_z_scale(model) -> np.ndarray:
    t = model.tables()
    return np.asarray(t["ref_scale"])[np.asarray(t["dof_off"])[:-1]]


def smooth_field(xy: np.ndarray, rng: np.random.Generator, amp: float, width=(150.0, 500.0), bumps=(3, 6)):
    """Sum of Gaussian bumps in z (metres) at the DOF positions."""
    lo, hi = xy.min(0), xy.max(0)
    out = np.zeros(len(xy))
    for _ in range(int(rng.integers(bumps[0], bumps[1] + 1))):
        c = rng.uniform(lo, hi)
        w = rng.uniform(*width)
        out += rng.normal(0.0, amp) * np.exp(-np.sum((xy - c) ** 2, axis=1) / (2 * w * w))
    return out


class Family:
    """A fixed starting model, its bounds and data scales; draws true models
    and noisy data."""

    def __init__(self, problem, amp: float = 40.0, noise: float = 0.01, device: int = 0):
        self.p = problem
        self.model = problem.build_model()
        self.x0 = self.model.assemble_parameters()
        self.lo, self.hi = self.model.bounds()
        self.xy = dof_xy(self.model)
        self.zs = dof_z_scale(self.model)
        self.amp, self.noise = amp, noise
        self.ctx = problem.make_context(self.model, device=device)
        self.ctx.set_precision(PREC_MIXED)
        self.ctx.set_scatter_stateless(True)  # data that depend on the true model alone
        self.ctx.set_collapsed_facets(COLLAPSED_DROP)  # the forward the inversions fit
        self.g0, self.m0 = self.ctx.forward(self.x0)
        self.sg = float(np.sqrt(np.mean(self.g0 ** 2)))
        self.sm = float(np.sqrt(np.mean(self.m0 ** 2)))
        self.n_in = 2 * len(self.g0)
        self.n_out = len(self.x0)

    def draw(self, rng: np.random.Generator, amp_scale: float = 1.0):
        """A true model and its noisy data (noise = `noise` x data RMS)."""
        x = np.clip(self.x0 + smooth_field(self.xy, rng, self.amp * amp_scale) / self.zs, self.lo, self.hi)
        g, m = self.ctx.forward(x)
        gstd = self.noise * np.sqrt(np.mean(g ** 2))
        mstd = self.noise * np.sqrt(np.mean(m ** 2))
        return x, g + gstd * rng.normal(size=len(g)), m + mstd * rng.normal(size=len(m)), gstd, mstd

    def features(self, gobs, mobs) -> np.ndarray:
        return np.concatenate([(gobs - self.g0) / self.sg, (mobs - self.m0) / self.sm]).astype(np.float32)

    def target(self, x) -> np.ndarray:
        return ((x - self.x0) * self.zs / self.amp).astype(np.float32)

    def update(self, y) -> np.ndarray:
        return np.asarray(y, np.float64) * self.amp / self.zs

    def pairs(self, n: int, rng: np.random.Generator):
        """Training pairs; a third of them at reduced amplitude (0.05-0.5 of
        the family's), so that the network also sees the small residuals the
        refinement steps feed it."""
        X = np.zeros((n, self.n_in), np.float32)
        Y = np.zeros((n, self.n_out), np.float32)
        for i in range(n):
            scale = 1.0 if i % 3 else float(np.exp(rng.uniform(np.log(0.05), np.log(0.5))))
            x, g, m, _, _ = self.draw(rng, scale)
            X[i], Y[i] = self.features(g, m), self.target(x)
        return X, Y


def _misfit(fam: Family, g, m, gobs, mobs, gstd, mstd) -> float:
    return 0.5 * float(np.sum(((gobs - g) / gstd) ** 2) + np.sum(((mobs - m) / mstd) ** 2))


def invert(fam: Family, gobs, mobs, gstd, mstd, net: Optional[Network] = None, max_iter: int = 200,
           refine: int = 6, secant_gamma: bool = False, chain: bool = True):
    """L-BFGS-B from x0 (plain) or from the network's proposal, until the
    data misfit reaches chi^2 = N.

    With a network: x_1 = x0 + net(residual at x0); then, up to `refine`
    times, x_{k+1} = x_k + net(residual at x_k) - net(0) -- the network as an
    approximate inverse of the linearised forward (its output at zero
    residual removed), one forward per step -- keeping a step only when the
    misfit drops.  With secant_gamma the start's gamma_0 comes from the
    secant pair (x_k - x0, g(x_k) - g(x0)) at the cost of two gradient
    evaluations; on the c5 family that cost more than it saved (mean wall
    time 1.51x vs 1.62x over plain), so it is off by default.  With `chain`
    (default) both runs use the chain gather, the stateless scatter and drop
    collapsed facets: on control-point models the reference's DOF-vertex
    gather is not the objective's gradient and L-BFGS-B stalls before
    chi^2 = N.  Returns wall seconds
    (proposals included), objective(+gradient) and forward evaluations, final
    objective, whether the target was reached and whether a proposal was
    taken."""
    import torch

    ctx = fam.p.make_context(fam.model, grav_obs=gobs, grav_std=np.full(len(gobs), gstd), mag_obs=mobs,
                             mag_std=np.full(len(mobs), mstd))
    ctx.set_precision(PREC_MIXED)
    if chain:  # the objective's own gradient through the control-point interpolation (lf_set_gradient_gather)
        ctx.set_scatter_stateless(True)
        ctx.set_gradient_gather(GATHER_CHAIN)
        ctx.set_collapsed_facets(COLLAPSED_DROP)  # the objective then has no rounding-noise jumps
    ctx.set_graph_mode(True)
    target = 0.5 * (len(gobs) + len(mobs))  # chi^2 = N  <=>  0.5 sum (r / sigma)^2 = N / 2
    ctx.objective_and_gradient(fam.x0)  # capture the graphs and size the buffers outside the timed region
    ctx.forward(fam.x0)
    t0 = time.perf_counter()
    x_start, gamma, used, forwards, extra = fam.x0, 0.0, False, 0, 0
    if net is not None:
        g_cur, m_cur = fam.g0, fam.m0  # predictions of the starting model (fixed per family)
        f_cur = _misfit(fam, g_cur, m_cur, gobs, mobs, gstd, mstd)
        x_cur = fam.x0
        zero = net.zero_response()
        for k in range(1 + refine):
            feat = np.concatenate([(gobs - g_cur) / fam.sg, (mobs - m_cur) / fam.sm]).astype(np.float32)
            out = net.predict_one(feat)
            upd = fam.update(out if k == 0 else out - zero)
            x_new = np.clip(x_cur + upd, fam.lo, fam.hi)
            g_new, m_new = ctx.forward(x_new)
            forwards += 1
            f_new = _misfit(fam, g_new, m_new, gobs, mobs, gstd, mstd)
            if not f_new < f_cur:
                break
            x_cur, g_cur, m_cur, f_cur = x_new, g_new, m_new, f_new
            if f_cur <= target:
                break
        if x_cur is not fam.x0:
            x_start, used = x_cur, True
            if f_cur > target and secant_gamma:
                _, g0 = ctx.objective_and_gradient(fam.x0)
                _, gs = ctx.objective_and_gradient(x_cur)
                extra = 2
                s, y = x_cur - fam.x0, gs - g0
                sy, yy = float(s @ y), float(y @ y)
                gamma = sy / yy if yy > 0 and sy > 0 else 0.0
    start_ratio = (f_cur if used else None)
    if used and f_cur <= target:  # the proposal already fits the data to chi^2 = N
        wall = time.perf_counter() - t0
        ctx.close()
        return dict(wall_s=wall, evaluations=extra, forwards=forwards, final=f_cur, reached=True, proposal_used=True,
                    iterations=0, start_misfit_over_target=f_cur / target)
    x, res = ctx.lbfgsb(x_start, fam.lo, fam.hi, max_iterations=max_iter, initial_gamma=gamma, target_value=target)
    wall = time.perf_counter() - t0
    ctx.close()
    return dict(wall_s=wall, evaluations=res.evaluations + res.gradients + extra, forwards=forwards,
                final=res.final_value, reached=res.final_value <= target, proposal_used=used,
                iterations=res.iterations, start_misfit_over_target=(start_ratio / target) if used else None)


def experiment(problem, n_pairs: int, n_heldout: int, epochs: int, seed: int = 0, width: int = 512, depth: int = 4,
               lr: float = 1e-3, batch: int = 256):
    import torch

    rng = np.random.default_rng(seed)
    fam = Family(problem)
    t0 = time.perf_counter()
    X, Y = fam.pairs(n_pairs, rng)
    t_gen = time.perf_counter() - t0
    net = Network(fam.n_in, fam.n_out, width=width, depth=depth, batch=batch, seed=seed)
    Xd, Yd = torch.as_tensor(X, device="cuda"), torch.as_tensor(Y, device="cuda")
    t0 = time.perf_counter()
    losses = net.train(Xd, Yd, epochs, lr, rng)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    hrng = np.random.default_rng(seed + 1000)
    plain, learned = [], []
    for _ in range(n_heldout):
        x, g, m, gs, ms = fam.draw(hrng)
        plain.append(invert(fam, g, m, gs, ms, None))
        learned.append(invert(fam, g, m, gs, ms, net))
    net.close()
    fam.ctx.close()

    def agg(runs):
        return dict(mean_wall_s=float(np.mean([r["wall_s"] for r in runs])),
                    mean_evaluations=float(np.mean([r["evaluations"] for r in runs])),
                    mean_forwards=float(np.mean([r["forwards"] for r in runs])),
                    reached=int(sum(r["reached"] for r in runs)))

    return dict(pairs=n_pairs, heldout=n_heldout, epochs=epochs, gen_s=t_gen, train_s=t_train,
                loss_first=losses[0], loss_last=losses[-1], plain=agg(plain), learned=agg(learned),
                proposals_used=int(sum(r["proposal_used"] for r in learned)),
                median_start_misfit_over_target=float(np.median([r["start_misfit_over_target"] for r in learned
                                                                 if r["start_misfit_over_target"] is not None]
                                                                or [np.nan])),
                speedup_wall=float(np.mean([r["wall_s"] for r in plain]) / np.mean([r["wall_s"] for r in learned])),
                speedup_per_model_median=float(np.median([p["wall_s"] / l["wall_s"] for p, l in zip(plain, learned)])),
                speedup_per_model_geomean=float(np.exp(np.mean([np.log(p["wall_s"] / l["wall_s"])
                                                                for p, l in zip(plain, learned)]))),
                learned_without_lbfgs=int(sum(r["iterations"] == 0 for r in learned)),
                runs=[dict(plain=p, learned=l) for p, l in zip(plain, learned)])


def main():
    from . import synth

    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=100_000)
    ap.add_argument("--heldout", type=int, default=64)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None, help="also write the summary and the per-model runs to this JSON file")
    a = ap.parse_args()
    # the config-2 family: 4 groups on 24 x 24 x 12 voxels of 100 m, control-point
    # stride 4, 64 x 64 stations (2 x 64 x 64 residual inputs)
    p = synth.voxel_contact_model()
    out = experiment(p, a.pairs, a.heldout, a.epochs, a.seed)
    out["model"] = dict(triangles=p.n_triangles(), stations=len(p.grav_xyz), width=512, depth=4)
    runs = out.pop("runs")
    out["per_model_wall_ratio"] = [r["plain"]["wall_s"] / r["learned"]["wall_s"] for r in runs]
    out["fallbacks"] = int(sum(not r["learned"]["proposal_used"] for r in runs))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(dict(summary=out, runs=runs), fh, indent=1)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
