"""Matrix-free data-weight calibration (lf_calibrate_data_weights) against
the compiled reference's JointObjective::calibrateDataWeights, which forms
both dense Jacobians.  Both run a power iteration from different random
starts (the reference uses Eigen's Random), and the reference's Jacobian is
its per-facet forward difference (~1e-5 relative from the analytic one), so
the calibrated alpha_mag is compared to 1e-3 relative."""
import numpy as np
import pytest

from oracle_bindings import OracleModel, RefModel, ref_available
from lithoinv3d_b200 import PREC_MIXED, synth

pytestmark = pytest.mark.gpu


def case():
    p = synth.icosphere_model(subdiv=2, n_side=12, spacing=80.0)
    m = p.build_model()
    x0 = m.assemble_parameters()
    om = OracleModel(m.tables(), p.densities, p.susceptibilities, p.inducing)
    om.scatter(x0 + np.random.default_rng(1).normal(0, 2, len(x0)))
    g, t = om.forward_gz(p.grav_xyz), om.forward_tmi(p.mag_xyz)
    gstd = np.full(len(g), 0.01 * np.std(g))
    tstd = np.full(len(t), 0.01 * np.std(t))
    return p, m, x0, g, gstd, t, tstd


def test_power_iteration_eigenvalues_consistent():
    p, m, x0, g, gstd, t, tstd = case()
    ctx = p.make_context(m, grav_obs=g, grav_std=gstd, mag_obs=t, mag_std=tstd)
    a1, eg1, em1 = ctx.calibrate_data_weights(x0, seed=1)
    assert eg1 > 0 and em1 > 0
    assert abs(a1 - eg1 / em1) <= 1e-12 * a1
    # a second calibration from another start finds the same eigenvalues and
    # multiplies alpha again (the reference mutates alpha the same way)
    a2, eg2, em2 = ctx.calibrate_data_weights(x0, seed=7)
    assert abs(eg2 - eg1) <= 1e-6 * eg1 and abs(em2 - em1) <= 1e-6 * em1
    assert abs(a2 - a1 * eg2 / em2) <= 1e-9 * a2
    # mixed precision contexts calibrate in FP64 as well
    cm = p.make_context(m, grav_obs=g, grav_std=gstd, mag_obs=t, mag_std=tstd)
    cm.set_precision(PREC_MIXED)
    am, egm, emm = cm.calibrate_data_weights(x0, seed=1)
    assert abs(am - a1) <= 1e-9 * a1


@pytest.mark.skipif(not ref_available(), reason="reference library not built")
def test_calibration_matches_reference():
    p, m, x0, g, gstd, t, tstd = case()
    ctx = p.make_context(m, grav_obs=g, grav_std=gstd, mag_obs=t, mag_std=tstd)
    a, eg, em = ctx.calibrate_data_weights(x0, seed=3)
    ref = RefModel(p, grav_obs=g, grav_std=gstd, mag_obs=t, mag_std=tstd)
    a_ref = ref.calibrate(x0)
    assert abs(a - a_ref) <= 1e-3 * a_ref
