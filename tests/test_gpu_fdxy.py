"""Finite-difference-XY gradient mode (lf_set_xy_derivative) against the
oracle: x and y vertex derivatives by per-facet forward differences of the
reference's facet formula with step h (faceNagyWithGradient
gravity_forward.cpp:48-85 differences every axis with h = 1e-4), z the true
derivative (oracle kinds 4 / 5), gathered at the DOF vertices as the
reference does.

Tolerances (norm-wise relative): FP64 1e-6, mixed 1e-5 (z comes from the
mixed analytic kernels; x and y are FP64 in both modes).
"""
import numpy as np
import pytest

from lithoinv3d_b200 import (GATHER_CHAIN, LithoError, PREC_FP64, PREC_MIXED, XY_ANALYTIC, XY_FORWARD_DIFFERENCE,
                             synth)
from oracle_bindings import OracleModel, misfit_gradient

pytestmark = pytest.mark.gpu

H = 0.5


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def problem():
    p = synth.voxel_contact_model(shape=(8, 8, 6), n_side=16, cp_stride=2, freedom_interior=synth.XYZ_FREE)
    model = p.build_model()
    t = model.tables()
    x0 = model.assemble_parameters()
    rng = np.random.default_rng(5)
    om = OracleModel(t, p.densities, p.susceptibilities, p.inducing)
    om.scatter(x0 + rng.normal(0.0, 5.0, len(x0)))
    data = []
    for pred in (om.forward_gz(p.grav_xyz), om.forward_tmi(p.mag_xyz)):
        s = max(0.01 * np.std(pred), 1e-6)
        data += [pred + s * rng.normal(size=len(pred)), np.full(len(pred), s)]
    return p, model, t, x0, data


def _oracle_gradient(p, t, x, data, kinds, h, chain=False):
    gobs, gstd, mobs, mstd = data
    om = OracleModel(t, p.densities, p.susceptibilities, p.inducing)
    om.scatter(x)
    pg, pm = om.forward_gz(p.grav_xyz), om.forward_tmi(p.mag_xyz)
    if chain:
        Jg = np.stack([om.chain_gather(r) for r in om.vertex_jacobian(p.grav_xyz, kinds[0], h)])
        Jm = np.stack([om.chain_gather(r) for r in om.vertex_jacobian(p.mag_xyz, kinds[1], h)])
    else:
        Jg, Jm = om.jacobian(p.grav_xyz, kinds[0], true_h=h), om.jacobian(p.mag_xyz, kinds[1], true_h=h)
    return misfit_gradient(Jg, pg, gobs, gstd) + misfit_gradient(Jm, pm, mobs, mstd)


@pytest.mark.parametrize("prec,tol", [(PREC_FP64, 1e-6), (PREC_MIXED, 1e-5)])
def test_fdxy_gradient_vs_oracle(problem, prec, tol):
    p, model, t, x0, data = problem
    gobs, gstd, mobs, mstd = data
    ctx = p.make_context(model, grav_obs=gobs, grav_std=gstd, mag_obs=mobs, mag_std=mstd)
    try:
        ctx.set_scatter_stateless(True)
        ctx.set_precision(prec)
        x = x0 + np.random.default_rng(8).normal(0.0, 4.0, len(x0))
        ctx.set_xy_derivative(XY_FORWARD_DIFFERENCE, H)
        _, g_fd = ctx.objective_and_gradient(x)
        want = _oracle_gradient(p, t, x, data, (4, 5), H)
        assert rel(g_fd, want) < tol
        # the step matters: at 0.5 m the forward difference is visibly not the derivative
        ctx.set_xy_derivative(XY_ANALYTIC, 0.0)
        _, g_an = ctx.objective_and_gradient(x)
        assert rel(g_an, _oracle_gradient(p, t, x, data, (2, 3), -3e-3)) < tol
        assert rel(g_fd, g_an) > 1e-5
        # with the chain gather as well
        ctx.set_xy_derivative(XY_FORWARD_DIFFERENCE, H)
        ctx.set_gradient_gather(GATHER_CHAIN)
        _, g_fc = ctx.objective_and_gradient(x)
        assert rel(g_fc, _oracle_gradient(p, t, x, data, (4, 5), H, chain=True)) < tol
    finally:
        ctx.close()


def test_fdxy_rejects_bad_step(problem):
    p, model, t, x0, data = problem
    ctx = p.make_context(model)
    try:
        for bad in (0.0, -1.0, float("nan"), float("inf")):
            with pytest.raises(LithoError):
                ctx.set_xy_derivative(XY_FORWARD_DIFFERENCE, bad)
        with pytest.raises(LithoError):
            ctx.set_xy_derivative(7, 0.5)
    finally:
        ctx.close()
