"""Per-group unit responses (lf_unit_response) against the oracle with a
unit property on one group, and against the compiled reference's
GravityForward / MagneticForward::computeGroupUnitResponse* where it is
built.  Tolerances (norm-wise relative): FP64 path 1e-10, mixed path 1e-6."""
import numpy as np
import pytest

from oracle_bindings import OracleModel, RefModel, ref_available
from lithoinv3d_b200 import PREC_MIXED, LithoError, Model, synth
from lithoinv3d_b200.api import UNIT_DIRECTION, UNIT_GRAVITY, UNIT_INDUCED, UNIT_REMANENCE

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-10
MIXED_TOL = 1e-6
DIR = np.array([0.3, -0.5, 0.8])


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def vox():
    p = synth.voxel_contact_model(shape=(10, 10, 6), n_side=12, cp_stride=2)
    m = p.build_model()
    x = m.assemble_parameters() + np.random.default_rng(4).normal(0, 3, m.n_dofs)
    om = OracleModel(m.tables(), p.densities, p.susceptibilities, p.inducing)
    om.scatter(x)
    return p, m, x, om


@pytest.mark.parametrize("mixed", [False, True])
def test_unit_responses_every_group(vox, mixed):
    p, m, x, om = vox
    ctx = p.make_context(m)
    if mixed:
        ctx.set_precision(PREC_MIXED)
    tol = MIXED_TOL if mixed else FWD_TOL
    for g in range(len(p.densities)):
        assert rel(ctx.unit_response(x, UNIT_GRAVITY, g), om.forward_unit(p.grav_xyz, UNIT_GRAVITY, g)) < tol
        assert rel(ctx.unit_response(x, UNIT_INDUCED, g), om.forward_unit(p.mag_xyz, UNIT_INDUCED, g)) < tol
        assert rel(ctx.unit_response(x, UNIT_DIRECTION, g, DIR),
                   om.forward_unit(p.mag_xyz, UNIT_DIRECTION, g, DIR)) < tol
    # the full forward is unchanged afterwards (group table restored)
    gz, tmi = ctx.forward(x)
    assert rel(gz, om.forward_gz(p.grav_xyz)) < tol
    assert rel(tmi, om.forward_tmi(p.mag_xyz)) < tol
    # unit responses weighted by the group densities sum to the forward
    gsum = sum(p.densities[g] * ctx.unit_response(x, UNIT_GRAVITY, g) for g in range(len(p.densities)))
    assert rel(gsum, gz) < 10 * tol


def test_unit_remanence_direction():
    p = synth.icosphere_model(subdiv=2, n_side=10)
    V, F, fr = p.meshes[0]
    m = Model()
    m.add_group(0, 0.3, 0.02, rem_magnitude=0.0, rem_inclination=35.0, rem_declination=-20.0)
    m.set_group_mesh(0, V, F, fr)
    ctx = p.make_context(m)
    x = m.assemble_parameters()
    I, D = np.radians(35.0), np.radians(-20.0)
    R = np.array([np.cos(I) * np.cos(D), np.cos(I) * np.sin(D), -np.sin(I)])
    om = OracleModel(m.tables(), p.densities, p.susceptibilities, p.inducing)
    om.scatter(x)
    got = ctx.unit_response(x, UNIT_REMANENCE, 0)
    assert rel(got, om.forward_unit(p.mag_xyz, UNIT_REMANENCE, 0, R)) < FWD_TOL


def test_unit_response_rejects_bad_arguments(vox):
    p, m, x, om = vox
    ctx = p.make_context(m)
    with pytest.raises(LithoError):
        ctx.unit_response(x, UNIT_GRAVITY, len(p.densities))
    with pytest.raises(LithoError):
        ctx.unit_response(x, 7, 0)
    with pytest.raises(LithoError):
        ctx.unit_response(x, UNIT_DIRECTION, 0, None)


@pytest.mark.skipif(not ref_available(), reason="reference library not built")
def test_unit_responses_match_reference(vox):
    p, m, x, om = vox
    ref = RefModel(p)
    ctx = p.make_context(m)
    for g in range(len(p.densities)):
        assert rel(ctx.unit_response(x, UNIT_GRAVITY, g), ref.unit_response(x, UNIT_GRAVITY, g)) < FWD_TOL
        assert rel(ctx.unit_response(x, UNIT_INDUCED, g), ref.unit_response(x, UNIT_INDUCED, g)) < FWD_TOL
        assert rel(ctx.unit_response(x, UNIT_DIRECTION, g, DIR),
                   ref.unit_response(x, UNIT_DIRECTION, g, DIR)) < FWD_TOL
