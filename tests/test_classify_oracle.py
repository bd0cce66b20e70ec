"""The reference harness's point classification and constraint penalty
(oracle/_ref: LithologyModel::classifyPoint, ConstraintHandler) pinned to
geometric truth on CPU before the GPU tests use it as the checker: points
well inside a perturbed icosphere classify as its group, points well outside
as -1, points below the bottom depth as -1, and the penalty counts the
squared thickness of every violated interval."""
import numpy as np
import pytest

from oracle_bindings import RefModel, ref_available
from lithoinv3d_b200 import synth

pytestmark = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")


def sphere_points(rng, center, r_lo, r_hi, n):
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.asarray(center) + d * rng.uniform(r_lo, r_hi, (n, 1))


def test_icosphere_inside_outside():
    p = synth.icosphere_model(subdiv=2, n_side=4)  # radius 200 m at 500 m depth, vertices perturbed by 20 m
    ref = RefModel(p)
    rng = np.random.default_rng(0)
    inside = sphere_points(rng, (0.0, 0.0, -500.0), 0.0, 120.0, 300)
    outside = sphere_points(rng, (0.0, 0.0, -500.0), 300.0, 900.0, 300)
    assert np.all(ref.classify(inside) == 0)
    assert np.all(ref.classify(outside) == -1)
    ref.set_bottom_depth(-450.0)
    assert np.all(ref.classify(inside[inside[:, 2] < -450.0]) == -1)


def test_penalty_counts_violated_thickness():
    p = synth.icosphere_model(subdiv=2, n_side=4)
    ref = RefModel(p)
    x0 = ref.assemble()
    # interval 1 inside the body labelled 0 (satisfied); interval 2 inside
    # labelled -2 (violated, 30 m thick); interval 3 outside labelled 0
    # (violated, 10 m thick): penalty = w (30^2 + 10^2)
    xy = np.array([[0.0, 0.0], [10.0, -5.0], [900.0, 900.0]])
    z_top = np.array([480.0, 485.0, 100.0])
    z_bottom = np.array([520.0, 515.0, 110.0])
    group = np.array([0, -2, 0], np.int32)
    ref.set_constraints(xy, z_top, z_bottom, group, weight=2.0)
    assert ref.constraint_value(x0) == 2.0 * (30.0 ** 2 + 10.0 ** 2)
