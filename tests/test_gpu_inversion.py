"""The single-body inversion on the device: 30 projected L-BFGS-B
iterations (LBFGSBOptimizer, lbfgsb_optimizer.cpp:162-263, restated in
csrc/lbfgsb.cpp) recovering vertex z of a perturbed icosphere (642 vertices,
1280 triangles, radius 200 m at 500 m depth) from joint gz + TMI data of a
seeded true perturbation with 1% Gaussian noise, z bounded to +-100 m.

The full-size run uses 40 x 40 stations at 50 m.  The reference's own
optimizer on its own (finite-difference) gradient is run beside ours on a
16 x 16 subsample of the same footprint, where it finishes in seconds on
one core (about 30 s); both must end at the same misfit within 2% (the reference's
gradient differs from the analytic one by ~1e-5 relative, so the two
trajectories are close but not identical)."""
import numpy as np
import pytest

from oracle_bindings import OracleModel, RefModel, ref_available
from lithoinv3d_b200 import PREC_MIXED, synth

pytestmark = pytest.mark.gpu

AXIS_SCALE = 10.0   # params in units of 10 m
BOUND = 10.0        # +-100 m


def c1_problem(n_side=40, spacing=50.0):
    return synth.icosphere_model(subdiv=3, n_side=n_side, spacing=spacing, axis_scale=AXIS_SCALE)


def c1_data(p, model, seed=11):
    """True model: x0 + N(0, 20 m) in z; data + 1% of RMS Gaussian noise."""
    rng = np.random.default_rng(seed)
    x0 = model.assemble_parameters()
    x_true = x0 + np.clip(rng.normal(0.0, 2.0, len(x0)), -BOUND, BOUND)
    om = OracleModel(model.tables(), p.densities, p.susceptibilities, p.inducing)
    om.scatter(x_true)
    g, t = om.forward_gz(p.grav_xyz), om.forward_tmi(p.mag_xyz)
    sg, st = 0.01 * np.sqrt(np.mean(g ** 2)), 0.01 * np.sqrt(np.mean(t ** 2))
    gobs = g + sg * rng.normal(size=len(g))
    tobs = t + st * rng.normal(size=len(t))
    return x0, x_true, gobs, np.full(len(g), sg), tobs, np.full(len(t), st)


@pytest.mark.parametrize("mixed", [False, True])
def test_c1_inversion_30_iterations(mixed):
    p = c1_problem()
    model = p.build_model()
    x0, x_true, gobs, gstd, tobs, tstd = c1_data(p, model)
    ctx = p.make_context(model, grav_obs=gobs, grav_std=gstd, mag_obs=tobs, mag_std=tstd)
    if mixed:
        ctx.set_precision(PREC_MIXED)
    f0 = ctx.objective(x0)
    x, res = ctx.lbfgsb(x0, x0 - BOUND, x0 + BOUND, max_iterations=30)
    assert res.iterations == 30 or res.converged
    # 642 z values from 3200 data: the misfit falls towards the noise level
    # (chi^2 / 2 = number of data / 2), not to zero
    noise_floor = 0.5 * (len(gobs) + len(tobs))
    assert res.final_value < 0.5 * f0
    assert res.final_value > 0.5 * noise_floor
    assert np.all(x >= x0 - BOUND - 1e-12) and np.all(x <= x0 + BOUND + 1e-12)
    assert abs(ctx.objective(x) - res.final_value) <= 1e-9 * res.final_value


@pytest.mark.skipif(not ref_available(), reason="reference library not built")
def test_c1_inversion_matches_reference_optimizer():
    p = c1_problem(n_side=16, spacing=125.0)
    model = p.build_model()
    x0, x_true, gobs, gstd, tobs, tstd = c1_data(p, model)
    ctx = p.make_context(model, grav_obs=gobs, grav_std=gstd, mag_obs=tobs, mag_std=tstd)
    x, res = ctx.lbfgsb(x0, x0 - BOUND, x0 + BOUND, max_iterations=30)
    ref = RefModel(p, grav_obs=gobs, grav_std=gstd, mag_obs=tobs, mag_std=tstd)
    xr, fr, itr = ref.lbfgsb(x0, x0 - BOUND, x0 + BOUND, max_iter=30)
    f0 = ctx.objective(x0)
    assert res.final_value < 0.5 * f0 and fr < 0.5 * f0
    assert abs(res.final_value - fr) <= 0.02 * fr
