"""The oracle's adjoint of the parameter scatter (lo_chain_gather) against
central differences of the oracle's own scatter + forward, on contact models
with control-point interpolation and shared-vertex averaging.

The reference's Jacobian gathers vertex derivatives at the DOF vertices only
(gravity_forward.cpp:270-289): with control-point interpolation that is not
the derivative of the forward with respect to the parameters, which the
second test records.  CPU only."""
import numpy as np
import pytest

from lithoinv3d_b200 import synth
from oracle_bindings import OracleModel

pytestmark = pytest.mark.filterwarnings("ignore")


def _problem(freedom):
    p = synth.voxel_contact_model(shape=(8, 8, 6), n_side=8, cp_stride=2, freedom_interior=freedom)
    model = p.build_model()
    return p, model, model.tables()


def _positions(p, tables, x):
    om = OracleModel(tables, p.densities, p.susceptibilities, p.inducing)
    om.scatter(x)
    return om.pos.reshape(-1, 3).copy()


def _smooth_dofs(p, tables, x):
    """DOFs that move no vertex of a collapsed facet (twice-area below 1e-10 x
    the longest edge squared).  The control-point interpolation collapses a
    few facets; the reference's TMI facet term does not vanish with the area
    (magnetic_forward.cpp:312-347), so the forward is not differentiable
    where such a facet opens up."""
    P, T = _positions(p, tables, x), tables["tri"].reshape(-1, 3)
    a, b, c = P[T[:, 0]], P[T[:, 1]], P[T[:, 2]]
    area2 = np.linalg.norm(np.cross(b - a, c - a), axis=1)
    longest = np.max([np.sum((b - a) ** 2, 1), np.sum((c - b) ** 2, 1), np.sum((a - c) ** 2, 1)], axis=0)
    bad_v = np.zeros(len(P), bool)
    bad_v[T[area2 < 1e-10 * longest].ravel()] = True
    ok = []
    for j in range(len(x)):
        e = np.zeros(len(x))
        e[j] = 1.0
        moved = np.any(_positions(p, tables, x + e) != P, axis=1)
        if not np.any(moved & bad_v):
            ok.append(j)
    return np.array(ok)


def _weighted_gz(p, tables, x, w):
    om = OracleModel(tables, p.densities, p.susceptibilities, p.inducing)
    om.scatter(x)
    return float(w @ om.forward_gz(p.grav_xyz)), float(w @ om.forward_tmi(p.mag_xyz))


@pytest.mark.parametrize("freedom", [synth.XYZ_FREE, synth.Z_ONLY])
def test_chain_gather_is_the_derivative_of_the_scattered_forward(freedom):
    p, model, t = _problem(freedom)
    assert len(t["interp_off"]) > 1 and np.diff(t["interp_off"]).max() > 0, "model must interpolate"
    assert np.diff(t["sync_off"]).max() >= 2, "model must average shared vertices"
    x0 = model.assemble_parameters()
    rng = np.random.default_rng(7)
    x = x0 + rng.normal(0.0, 5.0, len(x0))
    w = rng.normal(0.0, 1.0, len(p.grav_xyz))
    om = OracleModel(t, p.densities, p.susceptibilities, p.inducing)
    om.scatter(x)
    gg = om.chain_gather(om.vertex_jacobian(p.grav_xyz, 2).T @ w)
    gm = om.chain_gather(om.vertex_jacobian(p.mag_xyz, 3).T @ w)
    # DOF vertices lie >= 100 m below the stations: h = 1e-2 m has O(h^2 / d^2)
    # truncation below 1e-8 and rounding near 1e-12
    h = 1e-2
    ok = _smooth_dofs(p, t, x)
    assert len(ok) > len(x0) // 2
    for j in rng.choice(ok, 12, replace=False):
        e = np.zeros(len(x0))
        e[j] = h
        fp, fm = _weighted_gz(p, t, x + e, w), _weighted_gz(p, t, x - e, w)
        fd_g, fd_m = (fp[0] - fm[0]) / (2 * h), (fp[1] - fm[1]) / (2 * h)
        assert abs(gg[j] - fd_g) <= 1e-6 * np.abs(gg).max(), (j, gg[j], fd_g)
        assert abs(gm[j] - fd_m) <= 1e-6 * np.abs(gm).max(), (j, gm[j], fd_m)


def test_reference_gather_is_not_the_derivative_with_interpolation():
    p, model, t = _problem(synth.Z_ONLY)
    x0 = model.assemble_parameters()
    rng = np.random.default_rng(7)
    x = x0 + rng.normal(0.0, 5.0, len(x0))
    w = rng.normal(0.0, 1.0, len(p.grav_xyz))
    om = OracleModel(t, p.densities, p.susceptibilities, p.inducing)
    om.scatter(x)
    g_ref = om.jacobian(p.grav_xyz, 2, true_h=-3e-3).T @ w
    g_chain = om.chain_gather(om.vertex_jacobian(p.grav_xyz, 2).T @ w)
    assert np.abs(g_ref - g_chain).max() > 0.1 * np.abs(g_chain).max()


def test_fdxy_kinds_are_forward_differences_of_the_forward():
    """Oracle kinds 4 / 5 (finite-difference-XY mode): the x / y columns of
    the vertex Jacobian are forward differences of the whole forward with
    one vertex moved (the per-facet differences sum to it), the z columns are
    the true derivative (kinds 2 / 3)."""
    p, model, t = _problem(synth.XYZ_FREE)
    x = model.assemble_parameters() + np.random.default_rng(3).normal(0.0, 5.0, model.n_dofs)
    om = OracleModel(t, p.densities, p.susceptibilities, p.inducing)
    om.scatter(x)
    P, T = om.pos.reshape(-1, 3), t["tri"].reshape(-1, 3)
    a, b, c = P[T[:, 0]], P[T[:, 1]], P[T[:, 2]]
    area2 = np.linalg.norm(np.cross(b - a, c - a), axis=1)
    longest = np.max([np.sum((b - a) ** 2, 1), np.sum((c - b) ** 2, 1), np.sum((a - c) ** 2, 1)], axis=0)
    bad = np.zeros(len(P), bool)
    bad[T[area2 < 1e-10 * longest].ravel()] = True
    h = 0.5
    sta = p.grav_xyz[::4]
    for kind, fwd in ((4, "forward_gz"), (5, "forward_tmi")):
        Jfd = om.vertex_jacobian(sta, kind, h)
        Jt = om.vertex_jacobian(sta, kind - 2, -3e-3)
        np.testing.assert_allclose(Jfd[:, 2::3], Jt[:, 2::3], rtol=0, atol=1e-12 * np.abs(Jt).max())
        base = getattr(om, fwd)(sta)
        rng = np.random.default_rng(kind)
        moved = [v for v in rng.permutation(len(P)) if not bad[v] and np.abs(Jt[:, 3 * v:3 * v + 3]).max() > 0]
        for v in moved[:6]:
            for ax in (0, 1):
                o2 = OracleModel(t, p.densities, p.susceptibilities, p.inducing)
                o2.pos[:] = om.pos
                o2.pos.reshape(-1, 3)[v, ax] += h
                fd = (getattr(o2, fwd)(sta) - base) / h
                np.testing.assert_allclose(Jfd[:, 3 * v + ax], fd, rtol=0, atol=1e-9 * np.abs(Jt).max())
