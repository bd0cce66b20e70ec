"""Property step of the alternating inversion (lf_property_inversion) against
the reference's runPropertyInversion parts A and B (runner.cpp:708-917),
restated in the test harness with the reference's own unit responses and
LBFGSBOptimizer.  The GPU unit responses agree with the reference's to
~1e-13, so the small optimisations end at the same properties to 1e-7
(relative to the largest parameter of each part)."""
import copy

import numpy as np
import pytest

from oracle_bindings import RefModel, ref_available
from lithoinv3d_b200 import synth

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]

OPT = dict(density_range=(-1.0, 1.0), susceptibility_range=(0.0, 0.2), remanence_range=(0.0, 5.0),
           remanence_component_range=(-5.0, 5.0), damping=0.01, max_iterations=60, tolerance=1e-8)


def close(a, b, tol):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b))) <= tol * max(float(np.max(np.abs(b))), 1e-30)


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_property_inversion_matches_reference(mode):
    p = synth.voxel_contact_model(shape=(10, 10, 5), n_side=12, cp_stride=2, seed=9)
    m = p.build_model()
    rng = np.random.default_rng(mode)
    x = m.assemble_parameters() + rng.normal(0, 5.0, m.n_dofs)
    # observations of the same geometry with shifted properties, 1 % noise
    pt = copy.copy(p)
    pt.densities = [d + rng.uniform(-0.1, 0.1) for d in p.densities]
    pt.susceptibilities = [c * rng.uniform(0.5, 1.5) for c in p.susceptibilities]
    truth = pt.make_context(pt.build_model())
    gz, tmi = truth.forward(x)
    gstd, mstd = np.full(len(gz), 0.01 * np.std(gz)), np.full(len(tmi), 0.01 * np.std(tmi))
    gobs, mobs = gz + gstd * rng.normal(size=len(gz)), tmi + mstd * rng.normal(size=len(tmi))

    ctx = p.make_context(m, grav_obs=gobs, grav_std=gstd, mag_obs=mobs, mag_std=mstd)
    ctx.set_field(*p.inducing, remanence_mode=mode)
    ppg = {0: 1, 1: 2, 2: 4}[mode]
    dens, mag = ctx.property_inversion(x, magnetic_per_group=ppg, **OPT)

    ref = RefModel(p, gobs, gstd, mobs, mstd, remanence_mode=mode)
    opt = [*OPT["density_range"], *OPT["susceptibility_range"], *OPT["remanence_range"],
           *OPT["remanence_component_range"], OPT["damping"], OPT["tolerance"]]
    rdens, rmag = ref.property_inversion(x, opt, OPT["max_iterations"], len(p.meshes), ppg)
    assert close(dens, rdens, 1e-7)
    assert close(mag, rmag, 1e-7)
    # the densities moved towards the truth and the context now uses them
    assert np.max(np.abs(dens - pt.densities)) < np.max(np.abs(np.asarray(p.densities) - pt.densities))
    g_after, _ = ctx.forward(x)
    assert close(g_after, ref.forward_gz(x), 1e-7)  # the two density sets agree to 1e-7
