"""Pins the oracle (C restatement, oracle/litho_oracle.c) and the product's
host model builder to the reference's own sources compiled here
(oracle/_ref).  Everything is compared bit-for-bit: the restatement keeps
the reference's operation order.  Skipped where the reference tree was not
available to build oracle/_ref."""
import numpy as np
import pytest

import oracle_bindings as ob
from lithoinv3d_b200 import FIXED, XYZ_FREE, Z_ONLY, synth

pytestmark = pytest.mark.skipif(not ob.ref_available(), reason="oracle/_ref not built (no reference tree)")


def _problems():
    yield "icosphere", synth.icosphere_model(subdiv=2, n_side=8, spacing=100.0)
    yield "icosphere_xyz_scaled", synth.icosphere_model(subdiv=1, n_side=5, spacing=120.0, freedom=XYZ_FREE,
                                                         axis_scale=10.0)
    yield "voxel_cp2", synth.voxel_contact_model(shape=(10, 10, 6), n_side=8, cp_stride=2)
    yield "voxel_nocp", synth.voxel_contact_model(shape=(6, 6, 4), n_side=6, cp_stride=0, seed=5)
    yield "voxel_cp3_xyz", synth.voxel_contact_model(shape=(9, 8, 5), n_side=6, cp_stride=3, seed=7,
                                                     freedom_interior=XYZ_FREE)


@pytest.fixture(scope="module", params=list(_problems()), ids=lambda p: p[0])
def case(request):
    name, p = request.param
    model = p.build_model()
    rm = ob.RefModel(p)
    om = ob.OracleModel(model.tables(), p.densities, p.susceptibilities, p.inducing)
    return p, model, rm, om


def test_dof_tables_match_reference(case):
    p, model, rm, om = case
    t = model.tables()
    off, rv, ra, rs = rm.dof_tables()
    assert rm.np == model.n_dofs
    np.testing.assert_array_equal(off, t["dof_off"])
    np.testing.assert_array_equal(rv, t["ref_vertex"])
    np.testing.assert_array_equal(ra, t["ref_axis"])
    np.testing.assert_array_equal(rs, t["ref_scale"])
    np.testing.assert_array_equal(rm.is_control_point() == 0, np.diff(t["interp_off"]) > 0)


def test_assemble_and_bounds_match_reference(case):
    p, model, rm, om = case
    np.testing.assert_array_equal(rm.assemble(), model.assemble_parameters())
    lo, hi = rm.bounds()
    l2, h2 = model.bounds()
    np.testing.assert_array_equal(lo, l2)
    np.testing.assert_array_equal(hi, h2)


def test_scatter_sequence_matches_reference(case):
    p, model, rm, om = case
    x0 = rm.assemble()
    rng = np.random.default_rng(1)
    for _ in range(3):
        x = x0 + rng.normal(0, 3, len(x0))
        rm.apply(x)
        om.scatter(x)
        model.apply_parameters(x)
        np.testing.assert_array_equal(om.pos, rm.positions())
        np.testing.assert_array_equal(model.positions(), rm.positions())


def test_forward_matches_reference(case):
    p, model, rm, om = case
    x = rm.assemble() + np.random.default_rng(2).normal(0, 3, rm.np)
    om.scatter(x)
    np.testing.assert_array_equal(om.forward_gz(p.grav_xyz), rm.forward_gz(x))
    np.testing.assert_array_equal(om.forward_tmi(p.mag_xyz), rm.forward_tmi(x))


def test_unit_responses_match_reference(case):
    """GravityForward / MagneticForward::computeGroupUnitResponse* against the
    oracle with a unit property on one group."""
    p, model, rm, om = case
    x = rm.assemble() + np.random.default_rng(6).normal(0, 3, rm.np)
    om.scatter(x)
    d = np.array([0.3, -0.5, 0.8])
    for g in range(len(p.densities)):
        np.testing.assert_array_equal(om.forward_unit(p.grav_xyz, 0, g), rm.unit_response(x, 0, g))
        np.testing.assert_array_equal(om.forward_unit(p.mag_xyz, 1, g), rm.unit_response(x, 1, g))
        np.testing.assert_array_equal(om.forward_unit(p.mag_xyz, 2, g, d), rm.unit_response(x, 2, g, d))


def test_smoothness_matches_reference(case):
    """SurfaceSmoothness::evaluate / gradient against the C restatement:
    value and DOF gradient bit for bit."""
    p, model, rm, om = case
    rs = ob.RefModel(p, smooth_weight=0.7)
    x = rs.assemble() + np.random.default_rng(8).normal(0, 3, rs.np)
    om.scatter(x)
    fr = np.concatenate([np.broadcast_to(np.asarray(f, np.uint8), (len(V),)) for V, F, f in p.meshes])
    v_o, g_o = om.smoothness(fr, 0.7)
    v_r, g_r = rs.smoothness(x)
    assert v_o == v_r
    np.testing.assert_array_equal(g_o, g_r)


def test_fd_jacobian_matches_reference(case):
    p, model, rm, om = case
    if p.n_triangles() > 2000:
        pytest.skip("large")
    x = rm.assemble() + np.random.default_rng(3).normal(0, 3, rm.np)
    om.scatter(x)
    np.testing.assert_array_equal(om.jacobian(p.grav_xyz, 0), rm.jacobian_gz(x))
    np.testing.assert_array_equal(om.jacobian(p.mag_xyz, 1), rm.jacobian_tmi(x))


def test_group_magnetization_matches_reference(case):
    p, model, rm, om = case
    for g in range(len(p.densities)):
        amp, d = rm.group_magnetization(g)
        assert amp == om.amp[g]
        np.testing.assert_array_equal(d, om.mdir[g])


def test_objective_and_gradient_semantics(case):
    """JointObjective::evaluateComponents / gradient == misfits and
    -J^T W^2 r of the restatement (FD Jacobian, reference semantics)."""
    p, model, rm0, om = case
    if p.n_triangles() > 2000:
        pytest.skip("large")
    rng = np.random.default_rng(4)
    S = len(p.grav_xyz)
    gobs, gstd = rng.normal(0, 1, S), np.abs(rng.normal(1, 0.1, S))
    mobs, mstd = rng.normal(0, 50, S), np.zeros(S)  # std 0 -> weight 1
    rm = ob.RefModel(p, gobs, gstd, mobs, mstd, alpha_mag=0.7)
    x = rm.assemble() + rng.normal(0, 2, rm.np)
    comps = rm.objective(x)
    grad = rm.gradient(x)
    om.scatter(x)
    gz, tm = om.forward_gz(p.grav_xyz), om.forward_tmi(p.mag_xyz)
    fg = ob.misfit(gz, gobs, gstd)
    fm = ob.misfit(tm, mobs, mstd)
    np.testing.assert_allclose(comps[0], fg, rtol=1e-13)
    np.testing.assert_allclose(comps[1], fm, rtol=1e-13)
    np.testing.assert_allclose(comps[4], fg + 0.7 * fm, rtol=1e-13)
    g2 = ob.misfit_gradient(om.jacobian(p.grav_xyz, 0), gz, gobs, gstd) + \
        ob.misfit_gradient(om.jacobian(p.mag_xyz, 1), tm, mobs, mstd, 0.7)
    np.testing.assert_allclose(grad, g2, rtol=1e-9, atol=1e-12 * np.max(np.abs(g2)))


def test_reference_fd_jacobian_error_vs_truth():
    """The reference's per-facet forward differences (h = 1e-4 m) are
    ~1e-5 relative from the true derivative; the oracle's Richardson central
    differences are the truth the analytic device gradient is held to."""
    p = synth.icosphere_model(subdiv=2, n_side=6, spacing=120.0)
    model = p.build_model()
    om = ob.OracleModel(model.tables(), p.densities, p.susceptibilities, p.inducing)
    x = model.assemble_parameters()
    om.scatter(x)
    Jfd = om.jacobian(p.grav_xyz, 0)
    Jt = om.jacobian(p.grav_xyz, 2, 1e-2)
    Jt2 = om.jacobian(p.grav_xyz, 2, 5e-3)
    scale = np.max(np.abs(Jt))
    assert np.max(np.abs(Jt - Jt2)) / scale < 1e-6     # the truth is converged (FP64 roundoff ~1e-7)
    err = np.max(np.abs(Jfd - Jt)) / scale
    assert 1e-7 < err < 1e-4
