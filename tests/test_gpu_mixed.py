"""GPU parity of the mixed-precision path (FP32 far field, FP64 near field)
against the oracle.  Tolerances (norm-wise relative, max|x-x_ref|/max|x_ref|):
forward gz and TMI 1e-6; with every facet forced to FP64 (tau <= 0) 1e-10."""
import numpy as np
import pytest

from oracle_bindings import OracleModel
from lithoinv3d_b200 import PREC_MIXED, synth

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-6


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(b)))


def _case(problem, perturb=3.0, seed=0, sub=None):
    model = problem.build_model()
    om = OracleModel(model.tables(), problem.densities, problem.susceptibilities, problem.inducing)
    x = model.assemble_parameters() + np.random.default_rng(seed).normal(0, perturb, model.n_dofs)
    ctx = problem.make_context(model)
    ctx.set_precision(PREC_MIXED)
    om.scatter(x)
    idx = np.arange(len(problem.grav_xyz)) if sub is None else sub
    return ctx, om, x, idx


def test_mixed_forward_icosphere():
    p = synth.icosphere_model()
    ctx, om, x, idx = _case(p)
    gz, tmi = ctx.forward(x)
    assert rel(gz, om.forward_gz(p.grav_xyz)) < MIXED_TOL
    assert rel(tmi, om.forward_tmi(p.mag_xyz)) < MIXED_TOL
    assert ctx.near_pairs() < 0.5 * len(p.grav_xyz) * p.n_triangles()  # the FP32 far field carries the bulk


def test_mixed_forward_voxel_full_size():
    """The benchmark model (4 groups, 19k triangles, 4096 stations 1 m above
    the top) -- compared on 96 stations spread over the grid."""
    p = synth.voxel_contact_model()
    sub = np.linspace(0, len(p.grav_xyz) - 1, 96).astype(int)
    ctx, om, x, idx = _case(p, sub=sub)
    gz, tmi = ctx.forward(x)
    # collapsed facets: the reference's TMI there is rounding noise of the
    # normal; the FP32 far field reproduces it only to FP32 -- compare the
    # magnetics with those facets' share included (they are part of both sides)
    assert rel(gz[sub], om.forward_gz(p.grav_xyz[sub])) < MIXED_TOL
    assert rel(tmi[sub], om.forward_tmi(p.mag_xyz[sub])) < MIXED_TOL


@pytest.mark.parametrize("tau", [2.0, 2.5, 4.0])
def test_mixed_forward_far_ratios(tau):
    """Far-field ratios other than the default 3: below 3 the far pairs keep
    the range-tested series and the mid field (analytic gz) moves to within
    one or two facet sizes, where atanh(e)/e - 1 takes its half-argument
    steps (e > 0.2); above 3 the far pairs take the shortened series."""
    p = synth.voxel_contact_model(shape=(16, 16, 8), n_side=24, cp_stride=4, freedom_interior=synth.XYZ_FREE)
    ctx, om, x, idx = _case(p)
    ctx.set_far_field_ratio(tau)
    gz, tmi = ctx.forward(x)
    assert rel(gz, om.forward_gz(p.grav_xyz)) < MIXED_TOL
    assert rel(tmi, om.forward_tmi(p.mag_xyz)) < MIXED_TOL
    assert ctx.near_pairs() < 0.5 * len(p.grav_xyz) * p.n_triangles()


def test_mixed_all_near_is_fp64():
    p = synth.voxel_contact_model(shape=(10, 10, 6), n_side=12, cp_stride=2)
    ctx, om, x, idx = _case(p)
    ctx.set_far_field_ratio(0.0)
    gz, tmi = ctx.forward(x)
    assert rel(gz, om.forward_gz(p.grav_xyz)) < 1e-10
    assert rel(tmi, om.forward_tmi(p.mag_xyz)) < 1e-10


def test_mixed_objective_gradient_consistency():
    """Objective + gradient in mixed mode agree with FP64 mode to the mixed
    tolerances (objective 1e-6 relative, gradient 1e-5)."""
    p = synth.voxel_contact_model(shape=(10, 10, 6), n_side=12, cp_stride=2)
    model = p.build_model()
    om = OracleModel(model.tables(), p.densities, p.susceptibilities, p.inducing)
    x0 = model.assemble_parameters()
    xt = x0 + np.random.default_rng(1).normal(0, 4, len(x0))
    om.scatter(xt)
    gobs, mobs = om.forward_gz(p.grav_xyz), om.forward_tmi(p.mag_xyz)
    c64 = p.make_context(model, grav_obs=gobs, mag_obs=mobs)
    c32 = p.make_context(model, grav_obs=gobs, mag_obs=mobs)
    c32.set_precision(PREC_MIXED)
    f64, g64 = c64.objective_and_gradient(x0)
    f32, g32 = c32.objective_and_gradient(x0)
    # the objective moves by sum_i r_i * d(pred_i): bound it with the forward tolerance
    gz64, tm64 = c64.forward(x0)
    bound = MIXED_TOL * (np.sum(np.abs(gobs - gz64)) * np.max(np.abs(gz64)) +
                         np.sum(np.abs(mobs - tm64)) * np.max(np.abs(tm64)))
    assert abs(f32 - f64) < bound
    assert rel(g32, g64) < 1e-5


def test_mixed_gradient_full_size():
    """Mixed objective gradient on the benchmark model (4096 stations, 19k
    facets) against the FP64 path (itself held to the central-difference truth
    by test_gpu_parity.py): 1e-5 norm-wise relative.  Both contexts see the
    same call history: the shared-vertex averaging of the reference is
    stateful, so a context that evaluated another model first sits at a
    slightly different geometry."""
    p = synth.voxel_contact_model()
    model = p.build_model()
    gen = p.make_context(model)
    x0 = model.assemble_parameters()
    xt = x0 + np.random.default_rng(3).normal(0, 5, len(x0))
    gobs, mobs = gen.forward(xt)
    gen.close()
    gstd = np.full(len(gobs), 0.01 * np.std(gobs))
    mstd = np.full(len(mobs), 0.01 * np.std(mobs))
    ctx64 = p.make_context(model, grav_obs=gobs, grav_std=gstd, mag_obs=mobs, mag_std=mstd)
    ctx32 = p.make_context(model, grav_obs=gobs, grav_std=gstd, mag_obs=mobs, mag_std=mstd)
    ctx32.set_precision(PREC_MIXED)
    f64, g64 = ctx64.objective_and_gradient(x0)
    f32, g32 = ctx32.objective_and_gradient(x0)
    assert rel(g32, g64) < 1e-5
    assert abs(f32 - f64) / f64 < 1e-5


@pytest.mark.parametrize("shape,stride,side", [((9, 8, 5), 3, 8), ((16, 16, 8), 2, 32)])
def test_mixed_gradient_xyz_free(shape, stride, side):
    """x/y/z-free vertices: the mixed objective gradient against the FP64 path
    with zero observations, so that the residual is the prediction itself and
    the comparison measures the gradient kernels (1e-5) rather than the
    forward's 1e-7 error magnified by a small residual."""
    from lithoinv3d_b200 import XYZ_FREE
    p = synth.voxel_contact_model(shape=shape, n_side=side, cp_stride=stride, seed=7, freedom_interior=XYZ_FREE)
    model = p.build_model()
    x = model.assemble_parameters() + np.random.default_rng(5).normal(0, 3, model.n_dofs)
    zeros = np.zeros(len(p.grav_xyz))
    c64 = p.make_context(model, grav_obs=zeros, mag_obs=zeros)
    c32 = p.make_context(model, grav_obs=zeros, mag_obs=zeros)
    c32.set_precision(PREC_MIXED)
    f64, g64 = c64.objective_and_gradient(x)
    f32, g32 = c32.objective_and_gradient(x)
    assert rel(g32, g64) < 1e-5
    assert abs(f32 - f64) / f64 < 2e-6
