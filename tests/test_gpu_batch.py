"""Batched bodies (lf_set_station_groups): many independent closed bodies in
one model, each with its own station grid, evaluated by one persistent
forward launch and one gradient launch.  Checked body by body against the
oracle (forward: FP64 1e-10, mixed 1e-6 norm-wise relative) and against
separate single-body contexts (objective and gradient 1e-10 in FP64)."""
import numpy as np
import pytest

from oracle_bindings import OracleModel
from lithoinv3d_b200 import PREC_MIXED, synth
from lithoinv3d_b200.synth import Problem

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def batch():
    p = synth.batch_bodies_model(n_bodies=12, t_range=(500, 3000), side_range=(8, 24))
    m = p.build_model()
    x0 = m.assemble_parameters()
    off = np.concatenate([[0], np.cumsum(p.station_groups)])
    bodies = []
    dof = 0
    for b, (V, F, fr) in enumerate(p.meshes):
        st = p.grav_xyz[off[b]:off[b + 1]]
        q = Problem("body", [p.densities[b]], [p.susceptibilities[b]], [(V, F, fr)], st, st)
        mb = q.build_model()
        nb = mb.n_dofs
        bodies.append((q, mb, slice(dof, dof + nb), slice(off[b], off[b + 1])))
        dof += nb
    assert dof == m.n_dofs
    return p, m, x0, bodies


@pytest.mark.parametrize("mixed", [False, True])
def test_batched_forward_matches_oracle(batch, mixed):
    p, m, x0, bodies = batch
    ctx = p.make_context(m)
    if mixed:
        ctx.set_precision(PREC_MIXED)
    x = x0 + np.random.default_rng(1).normal(0, 3, len(x0))
    gz, tmi = ctx.forward(x)
    tol = 1e-6 if mixed else 1e-10
    for q, mb, ds, ss in bodies:
        om = OracleModel(mb.tables(), q.densities, q.susceptibilities, q.inducing)
        om.scatter(x[ds])
        assert rel(gz[ss], om.forward_gz(q.grav_xyz)) < tol
        assert rel(tmi[ss], om.forward_tmi(q.mag_xyz)) < tol


def test_batched_objective_gradient_match_single_bodies(batch):
    p, m, x0, bodies = batch
    rng = np.random.default_rng(2)
    xt = x0 + rng.normal(0, 4, len(x0))
    gen = p.make_context(m)
    gobs, mobs = gen.forward(xt)
    gen.close()
    ctx = p.make_context(m, grav_obs=gobs, mag_obs=mobs)
    f, g = ctx.objective_and_gradient(x0)
    fg = ctx.group_objectives(len(bodies))
    ftot = 0.0
    for b, (q, mb, ds, ss) in enumerate(bodies):
        cb = q.make_context(mb, grav_obs=gobs[ss], mag_obs=mobs[ss])
        fb, gb = cb.objective_and_gradient(x0[ds])
        assert abs(fg[b] - fb) <= 1e-10 * abs(fb)
        assert rel(g[ds], gb) < 1e-10
        ftot += fb
    assert abs(f - ftot) <= 1e-10 * abs(ftot)


def test_batched_mixed_gradient_and_graph(batch):
    p, m, x0, bodies = batch
    x = x0 + np.random.default_rng(3).normal(0, 3, len(x0))
    zeros = np.zeros(len(p.grav_xyz))
    c64 = p.make_context(m, grav_obs=zeros, mag_obs=zeros)
    c32 = p.make_context(m, grav_obs=zeros, mag_obs=zeros)
    c32.set_precision(PREC_MIXED)
    f64, g64 = c64.objective_and_gradient(x)
    f32, g32 = c32.objective_and_gradient(x)
    assert rel(g32, g64) < 1e-5 and abs(f32 - f64) < 2e-6 * f64
    c32.set_graph_mode(True)
    for _ in range(3):
        fr, gr = c32.objective_and_gradient(x)
        assert fr == f32 and np.array_equal(gr, g32)
