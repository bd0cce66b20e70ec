"""GPU parity: the CUDA path through the C ABI against the oracle (the C
restatement of the reference, pinned to the reference itself by
test_oracle_pin.py and the golden fixtures).

Tolerances (norm-wise relative, max|x - x_ref| / max|x_ref|):
  FP64 path: forward 1e-10, scatter exact, objective 1e-10,
  analytic Jacobian / gradient vs the O(h^4) central-difference truth 1e-6.
"""
import numpy as np
import pytest

from oracle_bindings import OracleModel, misfit
from lithoinv3d_b200 import GRAVITY, MAGNETIC, LithoError, synth

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-10
GRAD_TOL = 1e-6


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def setup(problem, seed=0, noise=0.01, perturb=5.0):
    model = problem.build_model()
    t = model.tables()
    om = OracleModel(t, problem.densities, problem.susceptibilities, problem.inducing)
    x0 = model.assemble_parameters()
    rng = np.random.default_rng(seed)
    x_true = x0 + rng.normal(0.0, perturb, len(x0))
    om.scatter(x_true)
    g_true = om.forward_gz(problem.grav_xyz)
    gobs = g_true + noise * np.std(g_true) * rng.normal(size=len(g_true))
    gstd = np.full(len(gobs), max(noise * np.std(g_true), 1e-6))
    mobs = mstd = None
    if problem.mag_xyz is not None:
        m_true = om.forward_tmi(problem.mag_xyz)
        mobs = m_true + noise * np.std(m_true) * rng.normal(size=len(m_true))
        mstd = np.full(len(mobs), max(noise * np.std(m_true), 1e-6))
    ctx = problem.make_context(model, grav_obs=gobs, grav_std=gstd, mag_obs=mobs, mag_std=mstd)
    # fresh oracle state at the model's start positions
    om2 = OracleModel(t, problem.densities, problem.susceptibilities, problem.inducing)
    return dict(model=model, ctx=ctx, om=om2, x0=x0, gobs=gobs, gstd=gstd, mobs=mobs, mstd=mstd, t=t)


@pytest.fixture(scope="module")
def ico():
    return setup(synth.icosphere_model())


@pytest.fixture(scope="module")
def vox():
    return setup(synth.voxel_contact_model(shape=(10, 10, 6), n_side=12, cp_stride=2))


def test_forward_icosphere_fp64(ico):
    ctx, om, x0 = ico["ctx"], ico["om"], ico["x0"]
    rng = np.random.default_rng(7)
    x = x0 + rng.normal(0, 3, len(x0))
    gz, tmi = ctx.forward(x)
    om.scatter(x)
    p = synth.icosphere_model()
    assert rel(gz, om.forward_gz(p.grav_xyz)) < FWD_TOL
    assert rel(tmi, om.forward_tmi(p.mag_xyz)) < FWD_TOL


def test_scatter_positions_exact(vox):
    ctx, om, x0, model = vox["ctx"], vox["om"], vox["x0"], vox["model"]
    rng = np.random.default_rng(3)
    for _ in range(3):  # the shared-vertex averaging is stateful: check a sequence
        x = x0 + rng.normal(0, 4, len(x0))
        ctx.forward(x)
        om.scatter(x)
        pos = ctx.positions(model.info().n_vertices)
        np.testing.assert_array_equal(pos, om.pos)


def test_forward_voxel_fp64(vox):
    ctx, om, x0 = vox["ctx"], vox["om"], vox["x0"]
    p = synth.voxel_contact_model(shape=(10, 10, 6), n_side=12, cp_stride=2)
    x = x0 + np.random.default_rng(11).normal(0, 4, len(x0))
    gz, tmi = ctx.forward(x)
    om.scatter(x)
    assert rel(gz, om.forward_gz(p.grav_xyz)) < FWD_TOL
    assert rel(tmi, om.forward_tmi(p.mag_xyz)) < FWD_TOL


@pytest.mark.parametrize("which", [GRAVITY, MAGNETIC])
def test_jacobian_vs_true_derivative(vox, which):
    ctx, om, x0 = vox["ctx"], vox["om"], vox["x0"]
    p = synth.voxel_contact_model(shape=(10, 10, 6), n_side=12, cp_stride=2)
    x = x0 + np.random.default_rng(5).normal(0, 4, len(x0))
    J = ctx.jacobian(x, which)
    om.scatter(x)
    sta = p.grav_xyz if which == GRAVITY else p.mag_xyz
    Jt = om.jacobian(sta, 2 + which)
    assert rel(J, Jt) < GRAD_TOL
    # the reference's own forward-difference Jacobian is ~1e-5 from the truth
    Jfd = om.jacobian(sta, which)
    assert rel(Jfd, Jt) < 1e-3


def test_jacobian_icosphere(ico):
    ctx, om, x0 = ico["ctx"], ico["om"], ico["x0"]
    p = synth.icosphere_model()
    sub = slice(0, 1600, 37)
    J = ctx.jacobian(x0, GRAVITY)[sub]
    om.scatter(x0)
    Jt = om.jacobian(p.grav_xyz[sub], 2)
    assert rel(J, Jt) < GRAD_TOL


def _oracle_objective_gradient(S, problem, x, alpha=1.0):
    om = S["om"]
    om.scatter(x)
    gz = om.forward_gz(problem.grav_xyz)
    f = misfit(gz, S["gobs"], S["gstd"])
    w = 1.0 / S["gstd"]
    Jg = om.jacobian(problem.grav_xyz, 2)
    grad = -Jg.T @ (w * w * (S["gobs"] - gz))
    fm = 0.0
    if problem.mag_xyz is not None:
        tm = om.forward_tmi(problem.mag_xyz)
        fm = misfit(tm, S["mobs"], S["mstd"])
        wm = 1.0 / S["mstd"]
        Jm = om.jacobian(problem.mag_xyz, 3)
        grad += -alpha * Jm.T @ (wm * wm * (S["mobs"] - tm))
    return f, fm, grad


def test_objective_and_gradient_voxel(vox):
    p = synth.voxel_contact_model(shape=(10, 10, 6), n_side=12, cp_stride=2)
    x = vox["x0"] + np.random.default_rng(9).normal(0, 4, len(vox["x0"]))
    comps = vox["ctx"].objective_components(x)
    f, g = vox["ctx"].objective_and_gradient(x)
    fo, fmo, go = _oracle_objective_gradient(vox, p, x)
    assert abs(comps[0] - fo) / fo < FWD_TOL
    assert abs(comps[1] - fmo) / fmo < FWD_TOL
    assert abs(f - (fo + fmo)) / (fo + fmo) < FWD_TOL
    assert rel(g, go) < GRAD_TOL


def test_objective_and_gradient_icosphere(ico):
    p = synth.icosphere_model()
    x = ico["x0"] + np.random.default_rng(2).normal(0, 2, len(ico["x0"]))
    f, g = ico["ctx"].objective_and_gradient(x)
    fo, fmo, go = _oracle_objective_gradient(ico, p, x)
    assert abs(f - (fo + fmo)) / (fo + fmo) < FWD_TOL
    assert rel(g, go) < GRAD_TOL


def test_reference_model_regularisation(vox):
    ctx, x0 = vox["ctx"], vox["x0"]
    x = x0 + np.random.default_rng(4).normal(0, 4, len(x0))
    f0, g0 = ctx.objective_and_gradient(x)
    lam = 0.37
    ctx.set_objective(1.0, lam, x0)
    try:
        f1, g1 = ctx.objective_and_gradient(x)
        comps = ctx.objective_components(x)
    finally:
        ctx.set_objective(1.0, 0.0, None)
    np.testing.assert_allclose(f1 - f0, 0.5 * lam * np.sum((x - x0) ** 2), rtol=1e-10)
    np.testing.assert_allclose(comps[2], 0.5 * lam * np.sum((x - x0) ** 2), rtol=1e-10)
    np.testing.assert_allclose(g1 - g0, lam * (x - x0), rtol=1e-9, atol=1e-12)


def test_alpha_zero_skips_magnetics(vox):
    ctx, x0 = vox["ctx"], vox["x0"]
    ctx.set_objective(0.0)
    try:
        comps = ctx.objective_components(x0)
        f, g = ctx.objective_and_gradient(x0)
    finally:
        ctx.set_objective(1.0)
    assert comps[1] == 0.0  # joint_objective.cpp:123 skips the magnetic term
    assert abs(f - comps[0]) <= 1e-12 * abs(f)


def test_lbfgsb_reduces_misfit(vox):
    ctx, model = vox["ctx"], vox["model"]
    x0 = vox["x0"]
    lo, hi = model.bounds()
    f0 = ctx.objective(x0)
    x, res = ctx.lbfgsb(x0, lo, hi, max_iterations=10)
    assert res.iterations >= 1
    assert res.final_value < 0.5 * f0
    assert np.all(x >= lo) and np.all(x <= hi)


def test_edge_cases_station_on_geometry():
    """Stations on a vertex, on an edge line and in a facet plane: the branch
    semantics of lineIntegralTerm / solidAngle are reproduced (zero terms)."""
    V = np.array([[0, 0, -10], [10, 0, -10], [0, 10, -10], [0, 0, -20.0]])
    F = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]], np.int32)
    from lithoinv3d_b200 import Z_ONLY
    sta = np.array([[0, 0, -10], [5, 0, -10], [20, 0, -10], [2, 2, -10], [3, 3, 5], [1e3, -2e3, 50.0]])
    p = synth.Problem("tet", [0.5], [0.03], [(V, F, Z_ONLY)], sta, sta)
    if synth.signed_volume(V, F) < 0:
        p.meshes[0] = (V, F[:, [0, 2, 1]].copy(), Z_ONLY)
    S = setup(p, noise=0.0, perturb=0.0)
    gz, tmi = S["ctx"].forward(S["x0"])
    S["om"].scatter(S["x0"])
    np.testing.assert_allclose(gz, S["om"].forward_gz(sta), rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(tmi, S["om"].forward_tmi(sta), rtol=1e-10, atol=1e-11)


def test_ragged_sizes_single_station():
    p = synth.icosphere_model(subdiv=1, n_side=1)
    S = setup(p, noise=0.0, perturb=1.0)
    gz, tmi = S["ctx"].forward(S["x0"])
    S["om"].scatter(S["x0"])
    assert rel(gz, S["om"].forward_gz(p.grav_xyz)) < FWD_TOL
    assert rel(tmi, S["om"].forward_tmi(p.mag_xyz)) < FWD_TOL


def test_gravity_only_and_separate_station_sets():
    p = synth.icosphere_model(subdiv=2, n_side=7, joint=False)
    S = setup(p, noise=0.0, perturb=1.0)
    gz, tmi = S["ctx"].forward(S["x0"])
    assert tmi.size == 0
    mag = synth.station_grid(5, 80.0, 3.0, center=(30.0, -20.0))
    S["ctx"].set_magnetic_data(mag)
    gz2, tmi2 = S["ctx"].forward(S["x0"])
    S["om"].scatter(S["x0"])
    assert rel(gz2, S["om"].forward_gz(p.grav_xyz)) < FWD_TOL
    assert rel(tmi2, S["om"].forward_tmi(mag)) < FWD_TOL


def test_invalid_inputs_rejected(vox):
    ctx, x0 = vox["ctx"], vox["x0"]
    bad = x0.copy()
    bad[0] = np.nan
    with pytest.raises(LithoError) as e:
        ctx.forward(bad)
    assert e.value.status == 1
    with pytest.raises(LithoError):
        ctx.set_gravity_data(np.array([[0.0, np.inf, 1.0]]))
    # the context stays usable
    gz, _ = ctx.forward(x0)
    assert np.all(np.isfinite(gz))
