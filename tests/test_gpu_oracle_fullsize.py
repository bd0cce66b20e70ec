"""The mixed-precision path at the benchmarked sizes, held to the oracle (the
C restatement of the reference, itself pinned to the compiled reference) --
not to this library's own FP64 kernels.

* Contact model (4 groups, 19,076 facets, the bench's model): forward gz /
  TMI on a 128-station subset spread over the 64 x 64 grid, and the joint
  objective gradient over that subset with noisy observations of a seeded
  true model, against -J^T W^2 r from the oracle's true derivative
  (objective.cpp:42-55, joint_objective.cpp:46-58).
* 256-body batch (2.5 M facets): the whole batch's forward in one launch,
  compared body by body with the oracle on 8 bodies across the batch
  (including the largest), and the gradient of 2 bodies in a context of all
  256 bodies with 24 stations each.
* Large model (194k facets, x/y/z-free): the gradient over a 64-station
  subset against the oracle's true derivative (56,898 DOFs): at the default
  far-field ratio contracted with the GPU's own residual (the residual is
  0.5 % of the data, which magnifies the forward's 6e-8 error ~190 times),
  and at tau = 6 against the truth itself.

Tolerances (norm-wise relative, max|x - x_ref| / max|x_ref|): gz and TMI
1e-6, gradient 1e-5.  The objective is bounded by the forward tolerance
times the residual mass (it is a sum of squared residuals)."""
import numpy as np
import pytest

from oracle_bindings import OracleModel, jacobian_parallel
from lithoinv3d_b200 import PREC_MIXED, synth
from lithoinv3d_b200.synth import Problem

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-6
GRAD_TOL = 1e-5


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def oracle_gradient(Jg, Jm, pred_g, pred_m, obs_g, obs_m, std_g, std_m, alpha_mag=1.0):
    """-Jg^T Wg^2 (obs - pred) - alpha Jm^T Wm^2 (obs - pred), W = 1/sigma."""
    wg, wm = 1.0 / std_g, 1.0 / std_m
    return -Jg.T @ (wg * wg * (obs_g - pred_g)) - alpha_mag * Jm.T @ (wm * wm * (obs_m - pred_m))


def noisy_data(om_true, sta, rng):
    gz, tmi = om_true.forward_gz(sta), om_true.forward_tmi(sta)
    std_g = np.full(len(gz), 0.01 * np.std(gz))
    std_m = np.full(len(tmi), 0.01 * np.std(tmi))
    return gz + std_g * rng.normal(size=len(gz)), tmi + std_m * rng.normal(size=len(tmi)), std_g, std_m


def test_contact_model_mixed_forward_and_gradient_vs_oracle():
    full = synth.voxel_contact_model()
    sub = np.linspace(0, len(full.grav_xyz) - 1, 128).astype(int)
    p = Problem(full.name, full.densities, full.susceptibilities, full.meshes, full.grav_xyz[sub],
                full.mag_xyz[sub], inducing=full.inducing, cp_stride=full.cp_stride)
    model = p.build_model()
    tables = model.tables()
    x0 = model.assemble_parameters()
    rng = np.random.default_rng(1234)
    x_true = x0 + rng.normal(0.0, 5.0, len(x0))
    om_true = OracleModel(tables, p.densities, p.susceptibilities, p.inducing)
    om_true.scatter(x_true)
    obs_g, obs_m, std_g, std_m = noisy_data(om_true, p.grav_xyz, rng)

    om = OracleModel(tables, p.densities, p.susceptibilities, p.inducing)
    om.scatter(x0)
    pred_g, pred_m = om.forward_gz(p.grav_xyz), om.forward_tmi(p.mag_xyz)
    Jg = jacobian_parallel(tables, p.densities, p.susceptibilities, p.inducing, x0, p.grav_xyz, 2)
    Jm = jacobian_parallel(tables, p.densities, p.susceptibilities, p.inducing, x0, p.mag_xyz, 3)
    g_ref = oracle_gradient(Jg, Jm, pred_g, pred_m, obs_g, obs_m, std_g, std_m)
    f_ref = 0.5 * np.sum(((obs_g - pred_g) / std_g) ** 2) + 0.5 * np.sum(((obs_m - pred_m) / std_m) ** 2)

    fwd = p.make_context(model)
    fwd.set_precision(PREC_MIXED)
    gz, tmi = fwd.forward(x0)
    fwd.close()
    assert rel(gz, pred_g) < FWD_TOL
    assert rel(tmi, pred_m) < FWD_TOL

    ctx = p.make_context(model, grav_obs=obs_g, grav_std=std_g, mag_obs=obs_m, mag_std=std_m)
    ctx.set_precision(PREC_MIXED)
    f, g = ctx.objective_and_gradient(x0)
    ctx.close()
    bound = FWD_TOL * (np.sum(np.abs(obs_g - pred_g) / std_g ** 2) * np.max(np.abs(pred_g)) +
                       np.sum(np.abs(obs_m - pred_m) / std_m ** 2) * np.max(np.abs(pred_m)))
    assert abs(f - f_ref) < bound, (f, f_ref, bound)
    assert rel(g, g_ref) < GRAD_TOL, rel(g, g_ref)


@pytest.fixture(scope="module")
def batch256():
    p = synth.batch_bodies_model(n_bodies=256)
    off = np.concatenate([[0], np.cumsum(p.station_groups)])
    return p, off


def _body(p, off, b, sta_idx=None):
    V, F, fr = p.meshes[b]
    st = p.grav_xyz[off[b]:off[b + 1]]
    if sta_idx is not None:
        st = st[sta_idx]
    q = Problem("body", [p.densities[b]], [p.susceptibilities[b]], [(V, F, fr)], st, st, inducing=p.inducing)
    return q


def _sampled_bodies(p):
    counts = np.array([len(F) for _, F, _ in p.meshes])
    order = np.argsort(counts)
    pick = {int(order[-1])}  # the largest body
    for q in np.linspace(0, len(order) - 2, 7):
        pick.add(int(order[int(round(q))]))
    return sorted(pick), counts


def test_batch256_mixed_forward_vs_oracle(batch256):
    p, off = batch256
    model = p.build_model()
    ctx = p.make_context(model)
    ctx.set_precision(PREC_MIXED)
    x = model.assemble_parameters() + np.random.default_rng(1).normal(0, 2, model.n_dofs)
    gz, tmi = ctx.forward(x)
    ctx.close()
    dof_off = np.concatenate([[0], np.cumsum([len(V) for V, _, _ in p.meshes])])  # z-only: one DOF per vertex
    assert dof_off[-1] == model.n_dofs
    picks, counts = _sampled_bodies(p)
    assert len(picks) >= 8 and counts[picks].max() == counts.max() and counts.max() > 40000
    for b in picks:
        ns = off[b + 1] - off[b]
        sidx = np.linspace(0, ns - 1, min(ns, 64)).astype(int)
        q = _body(p, off, b, sidx)
        mb = q.build_model()
        om = OracleModel(mb.tables(), q.densities, q.susceptibilities, q.inducing)
        om.scatter(x[dof_off[b]:dof_off[b + 1]])
        s = off[b] + sidx
        assert rel(gz[s], om.forward_gz(q.grav_xyz)) < FWD_TOL, b
        assert rel(tmi[s], om.forward_tmi(q.mag_xyz)) < FWD_TOL, b


def test_batch256_mixed_gradient_vs_oracle(batch256):
    """All 256 bodies (every facet) with 24 stations per body; the gradients
    of the largest body and of a mid-sized one against the oracle."""
    p, off = batch256
    per = 24
    sel = [off[b] + np.linspace(0, off[b + 1] - off[b] - 1, per).astype(int) for b in range(len(p.meshes))]
    st = p.grav_xyz[np.concatenate(sel)]
    q_all = Problem("batch", p.densities, p.susceptibilities, p.meshes, st, st, inducing=p.inducing,
                    station_groups=[per] * len(p.meshes))
    model = q_all.build_model()
    x0 = model.assemble_parameters()
    dof_off = np.concatenate([[0], np.cumsum([len(V) for V, _, _ in p.meshes])])
    counts = np.array([len(F) for _, F, _ in p.meshes])
    order = np.argsort(counts)
    check = [int(order[-1]), int(order[len(order) // 2])]
    rng = np.random.default_rng(7)
    obs_g, obs_m = np.zeros(len(st)), np.zeros(len(st))
    std_g, std_m = np.ones(len(st)), np.ones(len(st))
    refs = {}
    for b in check:
        q = _body(p, off, b, np.linspace(0, off[b + 1] - off[b] - 1, per).astype(int))
        mb = q.build_model()
        tb = mb.tables()
        xb = x0[dof_off[b]:dof_off[b + 1]]
        om_t = OracleModel(tb, q.densities, q.susceptibilities, q.inducing)
        om_t.scatter(xb + rng.normal(0, 3.0, len(xb)))
        og, omg, sg, sm = noisy_data(om_t, q.grav_xyz, rng)
        s = slice(b * per, (b + 1) * per)
        obs_g[s], obs_m[s], std_g[s], std_m[s] = og, omg, sg, sm
        om = OracleModel(tb, q.densities, q.susceptibilities, q.inducing)
        om.scatter(xb)
        pg, pm = om.forward_gz(q.grav_xyz), om.forward_tmi(q.mag_xyz)
        Jg = jacobian_parallel(tb, q.densities, q.susceptibilities, q.inducing, xb, q.grav_xyz, 2)
        Jm = jacobian_parallel(tb, q.densities, q.susceptibilities, q.inducing, xb, q.mag_xyz, 3)
        refs[b] = oracle_gradient(Jg, Jm, pg, pm, og, omg, sg, sm)
    ctx = q_all.make_context(model, grav_obs=obs_g, grav_std=std_g, mag_obs=obs_m, mag_std=std_m)
    ctx.set_precision(PREC_MIXED)
    _, g = ctx.objective_and_gradient(x0)
    ctx.close()
    for b in check:
        assert rel(g[dof_off[b]:dof_off[b + 1]], refs[b]) < GRAD_TOL, b


def test_large_model_mixed_gradient_vs_oracle():
    full = synth.large_model()
    sub = np.linspace(0, len(full.grav_xyz) - 1, 64).astype(int)
    p = Problem(full.name, full.densities, full.susceptibilities, full.meshes, full.grav_xyz[sub],
                full.mag_xyz[sub], inducing=full.inducing, cp_stride=full.cp_stride)
    model = p.build_model()
    tables = model.tables()
    x0 = model.assemble_parameters()
    rng = np.random.default_rng(99)
    x_true = x0 + rng.normal(0.0, 2.0, len(x0))
    om_true = OracleModel(tables, p.densities, p.susceptibilities, p.inducing)
    om_true.scatter(x_true)
    obs_g, obs_m, std_g, std_m = noisy_data(om_true, p.grav_xyz, rng)
    om = OracleModel(tables, p.densities, p.susceptibilities, p.inducing)
    om.scatter(x0)
    pred_g, pred_m = om.forward_gz(p.grav_xyz), om.forward_tmi(p.mag_xyz)
    Jg = jacobian_parallel(tables, p.densities, p.susceptibilities, p.inducing, x0, p.grav_xyz, 2)
    Jm = jacobian_parallel(tables, p.densities, p.susceptibilities, p.inducing, x0, p.mag_xyz, 3)
    g_ref = oracle_gradient(Jg, Jm, pred_g, pred_m, obs_g, obs_m, std_g, std_m)
    # At the default far-field ratio (tau = 3) the forward is within 6e-8
    # of the oracle, but the residual is only 0.5 % of the data here, so that
    # error reaches the gradient magnified ~190 times (1.4e-5 measured).  The
    # gradient kernels themselves are held to the truth at the GPU's own
    # residual; the whole chain is held to it at tau = 6 (more pairs in FP64).
    for tau, own in ((3.0, True), (6.0, False)):
        ctx = p.make_context(model, grav_obs=obs_g, grav_std=std_g, mag_obs=obs_m, mag_std=std_m)
        ctx.set_scatter_stateless(True)  # forward and gradient at the same positions
        ctx.set_precision(PREC_MIXED)
        ctx.set_far_field_ratio(tau)
        gz, tmi = ctx.forward(x0)
        _, g = ctx.objective_and_gradient(x0)
        ctx.close()
        assert rel(gz, pred_g) < FWD_TOL and rel(tmi, pred_m) < FWD_TOL
        want = oracle_gradient(Jg, Jm, gz, tmi, obs_g, obs_m, std_g, std_m) if own else g_ref
        assert rel(g, want) < GRAD_TOL, (tau, rel(g, want), rel(g, g_ref))
