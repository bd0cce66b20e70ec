"""The runner's gradient smoothing (lf_smooth_gradient) against
InversionRunner::smoothGradient restated on the compiled reference's model
(runner.cpp:643-706).  Sums and blends are rounded in the reference's order,
so the comparison is exact."""
import numpy as np
import pytest

from oracle_bindings import RefModel, ref_available
from lithoinv3d_b200 import XYZ_FREE, synth

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]


@pytest.fixture(scope="module", params=["voxel_z_cp2", "voxel_xyz_cp3", "icosphere_xyz", "voxel_z_all"])
def case(request):
    if request.param == "voxel_z_cp2":
        p = synth.voxel_contact_model(shape=(10, 10, 6), n_side=8, cp_stride=2)
    elif request.param == "voxel_xyz_cp3":
        p = synth.voxel_contact_model(shape=(9, 8, 5), n_side=8, cp_stride=3, seed=7, freedom_interior=XYZ_FREE)
    elif request.param == "voxel_z_all":
        p = synth.voxel_contact_model(shape=(8, 8, 4), n_side=8, cp_stride=0, seed=2)
    else:
        p = synth.icosphere_model(subdiv=2, n_side=8, freedom=XYZ_FREE, axis_scale=10.0)
    # control points at a stride > 1 are rarely mesh neighbours of each other,
    # so there the blend may leave every entry as it was
    return p, p.build_model(), request.param in ("icosphere_xyz", "voxel_z_all")


@pytest.mark.parametrize("weight", [0.3, 1.0, 0.0])
def test_smooth_gradient_matches_reference(case, weight):
    p, m, adjacent = case
    g = np.random.default_rng(11).normal(0, 1.0, m.n_dofs)
    ref = RefModel(p)
    want = ref.smooth_gradient(g, weight)
    ctx = p.make_context(m)
    got = ctx.smooth_gradient(g, weight)
    assert np.array_equal(got, want)
    if weight == 0:
        assert np.array_equal(got, g)
    elif adjacent:
        assert not np.array_equal(got, g)  # the blend changed something
