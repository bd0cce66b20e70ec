"""The oracle (C restatement) and the host model builder against the golden
fixtures in tests/golden/ -- outputs of the reference's own code compiled
here (tests/golden/make_golden.py).  Runs without the reference tree."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle_bindings as ob
from lithoinv3d_b200 import synth

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
_dp = C.POINTER(C.c_double)


def p(a):
    return np.ascontiguousarray(a, np.float64).ctypes.data_as(_dp)


def test_primitives_bit_exact():
    g = np.load(os.path.join(GOLD, "primitives.npz"))
    o = ob.oracle()
    for i in range(len(g["obs"])):
        a, b, c = g["tri"][i]
        o_ = g["obs"][i]
        assert o.lo_solid_angle(p(a), p(b), p(c), p(o_)) == g["solid_angle"][i]
        assert o.lo_line_integral_term(p(a), p(b), p(o_)) == g["line_integral"][i]
        assert o.lo_face_nagy(p(o_), p(a), p(b), p(c)) == g["gravity_facet"][i]
        assert o.lo_magnetic_facet(p(o_), p(a), p(b), p(c), p(g["mdir"]), p(g["fdir"])) == g["magnetic_facet"][i]
    # the degenerate branches are present in the fixture
    assert g["solid_angle"][0] == 0.0 and g["gravity_facet"][5] == 0.0


CASES = {
    "icosphere_s1": lambda: synth.icosphere_model(subdiv=1, n_side=6, spacing=90.0),
    "voxel_8x8x4_cp2": lambda: synth.voxel_contact_model(shape=(8, 8, 4), n_side=6, cp_stride=2, seed=4),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_model_case(name):
    g = np.load(os.path.join(GOLD, name + ".npz"))
    prob = CASES[name]()
    model = prob.build_model()
    t = model.tables()
    for k in ("dof_off", "ref_vertex", "ref_axis", "ref_scale"):
        np.testing.assert_array_equal(t[k], g[k])
    np.testing.assert_array_equal(model.assemble_parameters(), g["x0"])
    lo, hi = model.bounds()
    np.testing.assert_array_equal(lo, g["lower"])
    np.testing.assert_array_equal(hi, g["upper"])
    om = ob.OracleModel(t, prob.densities, prob.susceptibilities, prob.inducing)
    x = g["x"]
    om.scatter(x)
    np.testing.assert_array_equal(om.pos, g["pos"])
    gz = om.forward_gz(prob.grav_xyz)
    tm = om.forward_tmi(prob.mag_xyz)
    np.testing.assert_array_equal(gz, g["gz"])
    np.testing.assert_array_equal(tm, g["tmi"])
    np.testing.assert_array_equal(om.jacobian(prob.grav_xyz, 0), g["J_gz"])
    np.testing.assert_array_equal(om.jacobian(prob.mag_xyz, 1), g["J_tmi"])
    a = float(g["alpha_mag"])
    fg = ob.misfit(gz, g["gobs"], g["gstd"])
    fm = ob.misfit(tm, g["mobs"], g["mstd"])
    np.testing.assert_allclose(g["objective"][[0, 1, 4]], [fg, fm, fg + a * fm], rtol=1e-13)
    grad = ob.misfit_gradient(g["J_gz"], gz, g["gobs"], g["gstd"]) + \
        ob.misfit_gradient(g["J_tmi"], tm, g["mobs"], g["mstd"], a)
    np.testing.assert_allclose(grad, g["gradient"], rtol=1e-9, atol=1e-12 * np.abs(grad).max())
