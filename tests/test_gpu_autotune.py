"""Autotuner (lf_autotune): the chosen launch shapes come from the candidate
sets, and the objective and gradient under any shape agree with the default
shapes up to the summation order of partial sums: 1e-12 relative in FP64;
1e-6 in mixed precision, where chunk boundaries regroup the FP32 far-field
partial sums (the mixed gradient's own tolerance is 1e-5).  In mixed
precision the tuner also picks the forward engine (per-facet records or
facet patches), the station-block size of the patch forward (128 or 256)
and the far-field ratio tau from {2, 2.5, 3, 4}, the latter only within its
accuracy gate against the FP64 path, which the test re-checks."""
import numpy as np
import pytest

from lithoinv3d_b200 import PREC_MIXED, LithoError, synth
from lithoinv3d_b200.api import FWD_FACET, FWD_PATCH

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("mixed", [False, True])
def test_autotune_keeps_results(mixed):
    p = synth.voxel_contact_model(shape=(12, 12, 6), n_side=24, cp_stride=2)
    m = p.build_model()
    x0 = m.assemble_parameters()
    gen = p.make_context(m)
    gobs, mobs = gen.forward(x0 + np.random.default_rng(3).normal(0, 4, len(x0)))
    gen.close()
    ctx = p.make_context(m, grav_obs=gobs, mag_obs=mobs)
    if mixed:
        ctx.set_precision(PREC_MIXED)
    tol = 1e-6 if mixed else 1e-12
    f0, g0 = ctx.objective_and_gradient(x0)
    t, ms = ctx.autotune(x0, repeats=2)
    assert ms > 0
    assert t.fwd_target_blocks in ((0,) if mixed else ()) + (148 * 4, 148 * 8, 148 * 16, 148 * 32, 148 * 64, 148 * 128)
    assert t.grad_target_warps in (148 * 16, 148 * 32, 148 * 64, 148 * 128, 148 * 256)
    assert t.near_tiles_per_chunk in (0, 1, 2, 4, 8)
    assert t.patch_threads in (128, 256)
    assert t.far_ratio in (2.0, 2.5, 3.0, 4.0)
    assert t.fwd_engine in (FWD_FACET, FWD_PATCH)
    if t.fwd_target_blocks == 0:
        assert t.fwd_engine == FWD_PATCH
    got = ctx.tuning()
    assert (got.fwd_target_blocks, got.grad_target_warps, got.near_tiles_per_chunk, got.patch_threads,
            got.far_ratio, got.fwd_engine) == (t.fwd_target_blocks, t.grad_target_warps, t.near_tiles_per_chunk,
                                               t.patch_threads, t.far_ratio, t.fwd_engine)
    f1, g1 = ctx.objective_and_gradient(x0)
    if mixed:  # tau may have moved: hold the tuned result to the FP64 path
        ref = p.make_context(m, grav_obs=gobs, mag_obs=mobs)
        fr, gr = ref.objective_and_gradient(x0)
        ref.close()
        assert rel(g1, gr) < 1e-5 and abs(f1 - fr) <= 1e-5 * abs(fr)
        ctx.set_tuning(t.fwd_target_blocks, t.grad_target_warps, t.near_tiles_per_chunk, far_ratio=3.0)
        f0, g0 = ctx.objective_and_gradient(x0)
    else:
        assert abs(f1 - f0) <= tol * abs(f0) and rel(g1, g0) < tol
    # extreme shapes give the same numbers too
    for shape in ((148, 148, 1, 128), (148 * 32, 148 * 256, 3, 256)) + (((0, 148 * 32, 0, 128), (0, 148 * 32, 0, 256))
                                                                        if mixed else ()):
        ctx.set_tuning(*shape)
        f2, g2 = ctx.objective_and_gradient(x0)
        assert abs(f2 - f0) <= tol * abs(f0) and rel(g2, g0) < tol
    if mixed:  # the two forward engines agree within the mixed path's tolerances
        for engine in (FWD_FACET, FWD_PATCH):
            ctx.set_tuning(148 * 8, 148 * 64, 0, 128, 3.0, engine)
            fe, ge = ctx.objective_and_gradient(x0)
            assert abs(fe - f0) <= 1e-6 * abs(f0) and rel(ge, g0) < 1e-5
    with pytest.raises(LithoError):
        ctx.set_tuning(-1, 1, 0)
    with pytest.raises(LithoError):
        ctx.set_tuning(148 * 8, 148 * 64, 0, 128, 3.0, 7)
