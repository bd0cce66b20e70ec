"""Learned warm start (lithoinv3d_b200.warmstart): trained on pairs that the
GPU forward generates, the network's proposal must reach the chi^2 = N
misfit in fewer objective evaluations, on average over held-out models,
than plain L-BFGS-B from the starting model -- and never end worse, since
the plain start is kept whenever the proposal does not lower the
objective."""
import numpy as np
import pytest

from lithoinv3d_b200 import synth
from lithoinv3d_b200.warmstart import experiment

pytestmark = pytest.mark.gpu


def test_warm_start_gains_over_plain():
    p = synth.voxel_contact_model(shape=(10, 10, 6), n_side=16, cp_stride=0)
    out = experiment(p, n_pairs=3072, n_heldout=8, epochs=40, seed=0, width=256, depth=3, batch=256)
    assert out["loss_last"] < 0.5 * out["loss_first"]
    assert out["learned"]["reached"] >= out["plain"]["reached"]
    learned_cost = out["learned"]["mean_evaluations"] + out["learned"]["mean_forwards"]
    assert learned_cost < out["plain"]["mean_evaluations"]
    for r in out["runs"]:
        if r["plain"]["reached"]:
            assert r["learned"]["reached"]


def test_warm_start_on_config2_family_beats_plain_wall_time():
    """The config-2 family itself (4 groups on 24 x 24 x 12 voxels of 100 m,
    control-point stride 4, 64 x 64 stations, network 4 x 512) at reduced
    training size: the learned start must reach chi^2 = N in less mean wall
    time than plain L-BFGS-B over the held-out models."""
    p = synth.voxel_contact_model()
    out = experiment(p, n_pairs=6144, n_heldout=16, epochs=30, seed=0, width=512, depth=4, batch=256)
    assert out["loss_last"] < 0.5 * out["loss_first"]
    # chi^2 = N lies inside the noise of a few held-out models (both starts end
    # within a few per cent of it): one such model may fall either way
    assert out["learned"]["reached"] >= out["plain"]["reached"] - 1
    assert out["speedup_per_model_geomean"] > 1.5, out["speedup_per_model_geomean"]
    assert out["learned"]["mean_wall_s"] < out["plain"]["mean_wall_s"], (out["learned"], out["plain"])
