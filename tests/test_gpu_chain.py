"""Chain gather on the GPU (lf_set_gradient_gather(LF_GATHER_CHAIN)): the
objective gradient through the control-point interpolation and the
shared-vertex averaging, against the oracle's adjoint of the scatter
(lo_chain_gather) applied to its true vertex derivatives; and the projected
L-BFGS on an x/y/z-free control-point model, where the reference's
DOF-vertex gather (gravity_forward.cpp:270-289) is not the objective's
derivative and the line search stalls.

Tolerances (norm-wise relative, as the parity tests): FP64 1e-6, mixed 1e-5.
The station grids (16 x 16 over 800 m) share no coordinate with the 100 m
voxel lattice: a station exactly on an edge's line, where the reference's
lineIntegralTerm branch makes its forward discontinuous, would leave the
derivative undefined.
"""
import numpy as np
import pytest

from lithoinv3d_b200 import GATHER_CHAIN, GATHER_REFERENCE, PREC_FP64, PREC_MIXED, synth
from lithoinv3d_b200.api import COLLAPSED_DROP
from oracle_bindings import OracleModel, misfit, misfit_gradient

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def _data(p, model, seed=0, noise=0.01, perturb=5.0):
    t = model.tables()
    x0 = model.assemble_parameters()
    rng = np.random.default_rng(seed)
    om = OracleModel(t, p.densities, p.susceptibilities, p.inducing)
    om.scatter(x0 + rng.normal(0.0, perturb, len(x0)))
    out = []
    for pred in (om.forward_gz(p.grav_xyz), om.forward_tmi(p.mag_xyz)):
        s = max(noise * np.std(pred), 1e-6)
        out += [pred + s * rng.normal(size=len(pred)), np.full(len(pred), s)]
    return x0, out


def _oracle(p, t, x, gobs, gstd, mobs, mstd, chain):
    om = OracleModel(t, p.densities, p.susceptibilities, p.inducing)  # stateless: fresh positions
    om.scatter(x)
    pg, pm = om.forward_gz(p.grav_xyz), om.forward_tmi(p.mag_xyz)
    if chain:
        Jg, Jm = om.chain_jacobian(p.grav_xyz, 2), om.chain_jacobian(p.mag_xyz, 3)
    else:
        Jg, Jm = om.jacobian(p.grav_xyz, 2, true_h=-3e-3), om.jacobian(p.mag_xyz, 3, true_h=-3e-3)
    f = misfit(pg, gobs, gstd) + misfit(pm, mobs, mstd)
    return f, misfit_gradient(Jg, pg, gobs, gstd) + misfit_gradient(Jm, pm, mobs, mstd)


@pytest.mark.parametrize("freedom", [synth.XYZ_FREE, synth.Z_ONLY])
@pytest.mark.parametrize("prec,tol", [(PREC_FP64, 1e-6), (PREC_MIXED, 1e-5)])
def test_chain_gradient_vs_oracle(freedom, prec, tol):
    p = synth.voxel_contact_model(shape=(8, 8, 6), n_side=16, cp_stride=2, freedom_interior=freedom)
    model = p.build_model()
    t = model.tables()
    x0, (gobs, gstd, mobs, mstd) = _data(p, model)
    ctx = p.make_context(model, grav_obs=gobs, grav_std=gstd, mag_obs=mobs, mag_std=mstd)
    try:
        ctx.set_scatter_stateless(True)
        ctx.set_precision(prec)
        x = x0 + np.random.default_rng(3).normal(0.0, 4.0, len(x0))
        ctx.set_gradient_gather(GATHER_CHAIN)
        f, g = ctx.objective_and_gradient(x)
        f_o, g_o = _oracle(p, t, x, gobs, gstd, mobs, mstd, chain=True)
        # the misfit magnifies the mixed forward's ~1e-7 error by data / residual
        assert abs(f - f_o) <= (1e-10 if prec == PREC_FP64 else 1e-5) * f_o
        assert rel(g, g_o) < tol
        # switching back restores the reference's gather
        ctx.set_gradient_gather(GATHER_REFERENCE)
        _, g_ref = ctx.objective_and_gradient(x)
        _, g_ref_o = _oracle(p, t, x, gobs, gstd, mobs, mstd, chain=False)
        assert rel(g_ref, g_ref_o) < tol
        assert rel(g_ref, g_o) > 0.1  # the two gathers differ on this model
    finally:
        ctx.close()


def test_chain_gradient_with_smoothness_matches_directional_difference():
    """Smoothness enters the chain before the adjoint: the gradient's
    projection on a direction matches a central difference of the GPU's own
    FP64 objective (stateless scatter, so the objective is a function of p;
    collapsed facets dropped, so it is differentiable)."""
    p = synth.voxel_contact_model(shape=(8, 8, 6), n_side=16, cp_stride=2, freedom_interior=synth.XYZ_FREE)
    model = p.build_model()
    x0, (gobs, gstd, mobs, mstd) = _data(p, model)
    ctx = p.make_context(model, grav_obs=gobs, grav_std=gstd, mag_obs=mobs, mag_std=mstd)
    try:
        ctx.set_scatter_stateless(True)
        ctx.set_precision(PREC_FP64)
        ctx.set_collapsed_facets(COLLAPSED_DROP)
        ctx.set_gradient_gather(GATHER_CHAIN)
        ctx.set_objective(1.0, 1e-3, x0)
        ctx.set_smoothness(0.1)
        rng = np.random.default_rng(11)
        x = x0 + rng.normal(0.0, 4.0, len(x0))
        _, g = ctx.objective_and_gradient(x)
        d = rng.normal(0.0, 1.0, len(x0))
        h = 1e-3
        fd = (ctx.objective(x + h * d) - ctx.objective(x - h * d)) / (2 * h)
        assert abs(fd - g @ d) <= 1e-6 * np.linalg.norm(g) * np.linalg.norm(d), (fd, g @ d)
    finally:
        ctx.close()


def test_lbfgsb_with_chain_gather_does_not_stall():
    """x/y/z-free control-point model (the large-inversion construction at a
    smaller size): with the chain gather every line search succeeds, so the
    run ends on its iteration cap or its tolerance, never on the stall rule
    (collapsed facets dropped: their reference TMI term is discontinuous)."""
    p = synth.voxel_contact_model(shape=(16, 16, 8), n_side=24, cp_stride=4, freedom_interior=synth.XYZ_FREE)
    model = p.build_model()
    x0, (gobs, gstd, mobs, mstd) = _data(p, model, perturb=10.0)
    lo, hi = model.bounds()
    lo, hi = np.maximum(lo, x0 - 50.0), np.minimum(hi, x0 + 50.0)
    ctx = p.make_context(model, grav_obs=gobs, grav_std=gstd, mag_obs=mobs, mag_std=mstd)
    try:
        ctx.set_scatter_stateless(True)
        ctx.set_objective(1.0, 1e-3, x0)
        ctx.set_gradient_gather(GATHER_CHAIN)
        ctx.set_collapsed_facets(COLLAPSED_DROP)
        f0 = ctx.objective(np.clip(x0, lo, hi))
        x, res = ctx.lbfgsb(x0, lo, hi, max_iterations=60)
        msg = res.message.decode()
        assert msg in ("Maximum iterations reached", "Converged: projected gradient below tolerance"), msg
        assert res.final_value < 0.5 * f0
    finally:
        ctx.close()


@pytest.mark.parametrize("prec,tol", [(PREC_FP64, 1e-10), (PREC_MIXED, 1e-6)])
def test_dropped_collapsed_facets_forward_vs_oracle(prec, tol):
    """LF_COLLAPSED_DROP: the forward equals the reference's over the facets
    that are not collapsed onto a line (twice-area >= 1e-10 x longest edge^2)."""
    p = synth.voxel_contact_model(shape=(8, 8, 6), n_side=16, cp_stride=2, freedom_interior=synth.Z_ONLY)
    model = p.build_model()
    t = model.tables()
    x = model.assemble_parameters() + np.random.default_rng(3).normal(0.0, 4.0, model.n_dofs)
    om = OracleModel(t, p.densities, p.susceptibilities, p.inducing)
    om.scatter(x)
    P, T = om.pos.reshape(-1, 3), t["tri"].reshape(-1, 3)
    a, b, c = P[T[:, 0]], P[T[:, 1]], P[T[:, 2]]
    area2 = np.linalg.norm(np.cross(b - a, c - a), axis=1)
    longest = np.max([np.sum((b - a) ** 2, 1), np.sum((c - b) ** 2, 1), np.sum((a - c) ** 2, 1)], axis=0)
    keep = ~(area2 < 1e-10 * longest)
    assert (~keep).sum() > 0, "the model must have collapsed facets"
    grp = np.repeat(np.arange(len(p.densities)), np.diff(t["grp_tri_off"]))
    tk = dict(t)
    tk["tri"] = np.ascontiguousarray(T[keep].ravel(), dtype=np.int32)
    tk["grp_tri_off"] = np.searchsorted(grp[keep], np.arange(len(p.densities) + 1)).astype(np.int32)
    ok = OracleModel(tk, p.densities, p.susceptibilities, p.inducing)
    ok.pos[:] = om.pos
    want_g, want_m = ok.forward_gz(p.grav_xyz), ok.forward_tmi(p.mag_xyz)
    ctx = p.make_context(model)
    try:
        ctx.set_scatter_stateless(True)
        ctx.set_precision(prec)
        ctx.set_collapsed_facets(COLLAPSED_DROP)
        gz, tmi = ctx.forward(x)
    finally:
        ctx.close()
    assert rel(gz, want_g) < tol and rel(tmi, want_m) < tol
