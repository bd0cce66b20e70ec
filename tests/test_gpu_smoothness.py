"""SurfaceSmoothness regularisation on the device (lf_set_smoothness) against
the compiled reference's JointObjective with SurfaceSmoothness registered
(where it is built) and against the oracle's restatement.  Tolerances
(relative): smoothness value and gradient 1e-12 (exact arithmetic, only the
summation order of the penalty differs); whole objective / gradient as the
FP64 parity tests, 1e-10 / 1e-6."""
import numpy as np
import pytest

from oracle_bindings import OracleModel, RefModel, ref_available
from lithoinv3d_b200 import PREC_MIXED, LithoError, Model, XYZ_FREE, synth

pytestmark = pytest.mark.gpu

W = 0.35


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def freedoms(p):
    return np.concatenate([np.broadcast_to(np.asarray(f, np.uint8), (len(V),)) for V, F, f in p.meshes])


@pytest.fixture(scope="module", params=["voxel_z_cp2", "voxel_xyz_cp3", "icosphere_xyz"])
def case(request):
    if request.param == "voxel_z_cp2":
        p = synth.voxel_contact_model(shape=(10, 10, 6), n_side=12, cp_stride=2)
    elif request.param == "voxel_xyz_cp3":
        p = synth.voxel_contact_model(shape=(9, 8, 5), n_side=8, cp_stride=3, seed=7, freedom_interior=XYZ_FREE)
    else:
        p = synth.icosphere_model(subdiv=2, n_side=10, freedom=XYZ_FREE, axis_scale=10.0)
    m = p.build_model()
    x0 = m.assemble_parameters()
    x = x0 + np.random.default_rng(5).normal(0, 3, len(x0))
    om = OracleModel(m.tables(), p.densities, p.susceptibilities, p.inducing)
    om.scatter(x0 + np.random.default_rng(6).normal(0, 4, len(x0)))
    gobs, mobs = om.forward_gz(p.grav_xyz), om.forward_tmi(p.mag_xyz)
    return p, m, x, gobs, mobs


def test_smoothness_term_matches_oracle(case):
    p, m, x, gobs, mobs = case
    c0 = p.make_context(m, grav_obs=gobs, mag_obs=mobs)
    c1 = p.make_context(m, grav_obs=gobs, mag_obs=mobs)
    c1.set_smoothness(W)
    comp0, comp1 = c0.objective_components(x), c1.objective_components(x)
    f0, g0 = c0.objective_and_gradient(x)
    f1, g1 = c1.objective_and_gradient(x)
    om = OracleModel(m.tables(), p.densities, p.susceptibilities, p.inducing)
    om.scatter(x)
    v_o, g_o = om.smoothness(freedoms(p), W)
    assert v_o > 0
    assert abs((comp1[2] - comp0[2]) - v_o) <= 1e-12 * v_o
    assert abs((f1 - f0) - v_o) <= 1e-12 * max(abs(f1), v_o)
    assert rel(g1 - g0, g_o) < 1e-9
    # turning it off restores the plain objective
    c1.set_smoothness(0.0)
    assert abs(c1.objective(x) - f0) <= 1e-12 * abs(f0)


def test_smoothness_explicit_freedoms_and_mixed(case):
    p, m, x, gobs, mobs = case
    ca = p.make_context(m, grav_obs=gobs, mag_obs=mobs)
    ca.set_smoothness(W)
    cb = p.make_context(m, grav_obs=gobs, mag_obs=mobs)
    cb.set_smoothness(W, freedoms(p))
    fa, ga = ca.objective_and_gradient(x)
    fb, gb = cb.objective_and_gradient(x)
    assert fa == fb and np.array_equal(ga, gb)
    # mixed precision: the smoothness term is the same FP64 computation
    cm = p.make_context(m, grav_obs=gobs, mag_obs=mobs)
    cm.set_precision(PREC_MIXED)
    f_plain, g_plain = cm.objective_and_gradient(x)
    cm.set_smoothness(W)
    fm, gm = cm.objective_and_gradient(x)
    f0, g0 = p.make_context(m, grav_obs=gobs, mag_obs=mobs).objective_and_gradient(x)
    assert rel(gm - g_plain, ga - g0) < 1e-9


@pytest.mark.skipif(not ref_available(), reason="reference library not built")
def test_joint_objective_with_smoothness_matches_reference(case):
    p, m, x, gobs, mobs = case
    ctx = p.make_context(m, grav_obs=gobs, mag_obs=mobs)
    ctx.set_smoothness(W)
    ref = RefModel(p, grav_obs=gobs, mag_obs=mobs, smooth_weight=W)
    comp = ctx.objective_components(x)
    rcomp = ref.objective(x)
    assert abs(comp[2] - rcomp[2]) <= 1e-12 * abs(rcomp[2])
    assert abs(comp[4] - rcomp[4]) <= 1e-10 * abs(rcomp[4])


def test_smoothness_rejects_along_vector_and_bad_weight():
    p = synth.icosphere_model(subdiv=1, n_side=4)
    V, F, fr = p.meshes[0]
    m = Model()
    m.add_group(0, 0.3, 0.02)
    m.set_group_mesh(0, V, F, fr)
    ctx = p.make_context(m)
    with pytest.raises(LithoError):
        ctx.set_smoothness(-1.0)
    bad = np.full(len(V), 4, np.uint8)  # ALONG_VECTOR
    with pytest.raises(LithoError):
        ctx.set_smoothness(1.0, bad)
    ctx.set_smoothness(1.0)
