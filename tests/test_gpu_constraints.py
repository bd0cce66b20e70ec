"""Point classification and the borehole-constraint penalty on the device
(lf_classify_points, lf_constraint_penalty, lf_constraint_gradient) against
the compiled reference's LithologyModel::classifyPoint and
ConstraintHandler.  Classification is integer work and the penalty a sum of
squared interval thicknesses, so every comparison is exact."""
import numpy as np
import pytest

from oracle_bindings import RefModel, ref_available
from lithoinv3d_b200 import LithoError, synth

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]


def label_grid(p, cell=100.0):
    """The voxel labels as the reference's label grid: [iz][iy][ix], iz
    counted upward from the base, origin at the base corner."""
    lab = p.extra["labels"]
    nx, ny, nz = lab.shape
    grid = np.ascontiguousarray(lab.transpose(2, 1, 0)[::-1], np.int32)
    return grid, (-nx * cell / 2.0, -ny * cell / 2.0, -nz * cell), (cell, cell, cell)


def sample_points(p, m, x, rng, n_random=1500):
    """Random points in and around the model, plus points on the perturbed
    vertices and face centres (rays that graze edges and faces)."""
    lo = np.array([-700.0, -700.0, -700.0])
    hi = np.array([700.0, 700.0, 50.0])
    pts = [rng.uniform(lo, hi, (n_random, 3))]
    ref = RefModel(p)
    ref.apply(x)
    pos = ref.positions()
    pts.append(pos[rng.choice(len(pos), 200, replace=False)])
    tri = m.tables()["tri"]
    cen = pos[tri].mean(1)
    pts.append(cen[rng.choice(len(cen), 200, replace=False)])
    return np.concatenate(pts), ref


@pytest.fixture(scope="module")
def contact():
    p = synth.voxel_contact_model(shape=(12, 12, 6), n_side=8, cp_stride=2, seed=4)
    m = p.build_model()
    x0 = m.assemble_parameters()
    x = x0 + np.random.default_rng(2).normal(0, 20.0, len(x0))
    return p, m, x


def test_classify_ray_cast_matches_reference(contact):
    p, m, x = contact
    pts, ref = sample_points(p, m, x, np.random.default_rng(0))
    want = ref.classify(pts)
    ctx = p.make_context(m)
    got = ctx.classify_points(pts, params=x)
    assert np.array_equal(got, want)
    assert len(np.unique(want)) >= 3  # several groups and the outside are exercised
    # the same positions are kept for a call without parameters
    assert np.array_equal(ctx.classify_points(pts[:100]), want[:100])


def test_classify_label_grid_and_bottom_depth(contact):
    p, m, x = contact
    grid, origin, spacing = label_grid(p)
    grid = grid.copy()
    grid[:, ::3, ::2] = -1  # unlabelled voxels fall back to the ray cast
    pts, ref = sample_points(p, m, x, np.random.default_rng(1))
    ref.set_label_grid(grid, origin, spacing)
    ref.set_bottom_depth(-450.0)
    want = ref.classify(pts)
    ctx = p.make_context(m)
    ctx.set_label_grid(grid, origin, spacing)
    ctx.set_bottom_depth(-450.0)
    got = ctx.classify_points(pts, params=x)
    assert np.array_equal(got, want)
    assert np.all(got[pts[:, 2] < -450.0] == -1)
    ctx.set_label_grid(None, origin, spacing)  # removing the grid: ray casting only
    ref2 = RefModel(p)
    ref2.apply(x)
    ref2.set_bottom_depth(-450.0)
    assert np.array_equal(ctx.classify_points(pts), ref2.classify(pts))


def constraint_set(p, m, x, rng):
    """Intervals whose midpoints sit 0.3 m above or below control-point
    vertices (so that a 1 m step of a DOF flips their class) plus random
    intervals; groups drawn from the classes at x and from random ids."""
    ref = RefModel(p)
    ref.apply(x)
    pos = ref.positions()
    t = m.tables()
    cp_vertices = np.unique(t["ref_vertex"][t["ref_axis"] == 2])
    pick = pos[rng.choice(cp_vertices, 24, replace=False)]
    mid = pick + np.where(rng.random(len(pick)) < 0.5, 0.3, -0.3)[:, None] * np.array([0.0, 0.0, 1.0])
    rnd = rng.uniform([-550.0, -550.0, -550.0], [550.0, 550.0, -20.0], (16, 3))
    mid = np.concatenate([mid, rnd])
    half = rng.uniform(0.5, 40.0, len(mid))
    z_top, z_bottom = -mid[:, 2] - half, -mid[:, 2] + half
    cls = ref.classify(mid)
    group = np.where(rng.random(len(mid)) < 0.6, cls, rng.integers(-1, len(p.meshes), len(mid))).astype(np.int32)
    return mid[:, :2].copy(), z_top, z_bottom, group


def test_constraint_penalty_and_gradient_match_reference(contact):
    p, m, x = contact
    xy, zt, zb, group = constraint_set(p, m, x, np.random.default_rng(3))
    ref = RefModel(p)
    ref.set_constraints(xy, zt, zb, group, weight=7.5)
    ctx = p.make_context(m)
    ctx.set_constraints(xy, zt, zb, group, weight=7.5)
    assert ctx.constraint_penalty(x) == ref.constraint_value(x)
    g_ref = ref.constraint_gradient(x)
    g = ctx.constraint_gradient(x)
    assert np.count_nonzero(g_ref) > 0
    assert np.array_equal(g, g_ref)
    # the reference leaves its model at the last perturbed parameters; so does the context
    probe = np.random.default_rng(4).uniform([-600, -600, -600], [600, 600, 0], (400, 3))
    assert np.array_equal(ctx.classify_points(probe), ref.classify(probe))
    # a second round from that state stays in step
    x2 = x + np.random.default_rng(5).normal(0, 2.0, len(x))
    assert ctx.constraint_penalty(x2) == ref.constraint_value(x2)


def test_constraints_with_label_grid_and_defaults(contact):
    p, m, x = contact
    grid, origin, spacing = label_grid(p)
    xy, zt, zb, group = constraint_set(p, m, x, np.random.default_rng(6))
    ref = RefModel(p)
    ref.set_label_grid(grid, origin, spacing)
    ref.set_constraints(xy, zt, zb, group)  # default weight 1e6
    ctx = p.make_context(m)
    ctx.set_label_grid(grid, origin, spacing)
    ctx.set_constraints(xy, zt, zb, group)
    assert ctx.constraint_penalty(x) == ref.constraint_value(x)
    assert np.array_equal(ctx.constraint_gradient(x), ref.constraint_gradient(x))
    # later sweeps replay a captured CUDA graph; they must stay in step too
    for k in range(2):
        xk = x + np.random.default_rng(10 + k).normal(0, 3.0, len(x))
        assert np.array_equal(ctx.constraint_gradient(xk), ref.constraint_gradient(xk))


def test_constraint_input_errors(contact):
    p, m, x = contact
    ctx = p.make_context(m)
    with pytest.raises(LithoError):
        ctx.set_constraints([[0.0, 0.0]], [np.nan], [1.0], [0])
    with pytest.raises(LithoError):
        ctx.classify_points([[0.0, 0.0, np.inf]])
    with pytest.raises(LithoError):
        ctx.set_label_grid(np.zeros((2, 2, 2), np.int32), (0, 0, 0), (1.0, 0.0, 1.0))
    ctx.set_constraints(np.zeros((0, 2)), [], [], [])  # no intervals: zero penalty and gradient
    assert ctx.constraint_penalty(x) == 0.0
    assert not np.any(ctx.constraint_gradient(x))
