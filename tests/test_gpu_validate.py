"""Model validation (lf_validate_model) against the compiled reference's
LithologyModel::validate: pass / fail, the failure text (overlap counts,
spike magnitudes) and the worst violation must be identical -- the overlap
counts come from the GPU ray-cast classification of every vertex, so this
also checks that classification against the reference on vertices that lie
exactly on shared contact surfaces."""
import numpy as np
import pytest

from oracle_bindings import RefModel, ref_available
from lithoinv3d_b200 import synth

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]

BIG = 10 ** 6


@pytest.fixture(scope="module")
def contact():
    p = synth.voxel_contact_model(shape=(12, 12, 6), n_side=8, cp_stride=2, seed=4)
    m = p.build_model()
    return p, m, m.assemble_parameters()


def cases(x0):
    rng = np.random.default_rng(1)
    spike = x0.copy()
    spike[10] += 2000.0
    return [(x0, 0, 0), (x0, BIG, BIG), (x0 + rng.normal(0, 20.0, len(x0)), 0, BIG),
            (x0 + rng.normal(0, 60.0, len(x0)), BIG, BIG), (spike, BIG, BIG)]


def test_validate_matches_reference(contact):
    p, m, x0 = contact
    ctx = p.make_context(m)
    ref = RefModel(p)
    outcomes = set()
    for x, overlap_base, adj_base in cases(x0):
        ref.apply(x)
        want = ref.validate(overlap_base, adj_base)
        got = ctx.validate_model(x, overlap_base, adj_base)
        assert got == want
        outcomes.add(want[1].split(":")[0])
    # passes, adjacent and non-adjacent overlap failures and a spike are all exercised
    assert {"", "Adjacent overlap", "Spike detected"} <= outcomes
