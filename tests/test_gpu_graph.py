"""Graph mode (lf_set_graph_mode): evaluations replayed from a captured CUDA
graph give the same bits as direct launches, through parameter changes,
setters that invalidate the graph, a unit-response call that re-plans the
forward chunks, and a whole L-BFGS-B run."""
import numpy as np
import pytest

from lithoinv3d_b200 import PREC_MIXED, synth
from lithoinv3d_b200.api import UNIT_GRAVITY

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["fp64", "mixed"])
def pair(request):
    p = synth.voxel_contact_model(shape=(10, 10, 6), n_side=12, cp_stride=2)
    m = p.build_model()
    x0 = m.assemble_parameters()
    gen = p.make_context(m)
    gobs, mobs = gen.forward(x0 + np.random.default_rng(2).normal(0, 4, len(x0)))
    gen.close()
    ctxs = []
    for graph in (False, True):
        c = p.make_context(m, grav_obs=gobs, mag_obs=mobs)
        if request.param == "mixed":
            c.set_precision(PREC_MIXED)
        c.set_smoothness(0.1)
        if graph:
            c.set_graph_mode(True)
        ctxs.append(c)
    return p, m, x0, ctxs[0], ctxs[1]


def test_replay_matches_direct_launches(pair):
    p, m, x0, eager, graph = pair
    rng = np.random.default_rng(9)
    xs = [x0 + rng.normal(0, 2, len(x0)) for _ in range(4)]
    for x in xs + xs:  # second round replays captured graphs
        fe, ge = eager.objective_and_gradient(x)
        fg, gg = graph.objective_and_gradient(x)
        assert fe == fg and np.array_equal(ge, gg)
        np.testing.assert_array_equal(eager.objective_components(x), graph.objective_components(x))


def test_setters_and_replans_invalidate(pair):
    p, m, x0, eager, graph = pair
    x = x0 + 0.5
    graph.objective_and_gradient(x)
    for c in (eager, graph):
        c.set_objective(alpha_mag=0.3)
    fe, ge = eager.objective_and_gradient(x)
    fg, gg = graph.objective_and_gradient(x)
    assert fe == fg and np.array_equal(ge, gg)
    for c in (eager, graph):  # re-plans the forward chunks for one group
        c.unit_response(x, UNIT_GRAVITY, 1)
    fe, ge = eager.objective_and_gradient(x)
    fg, gg = graph.objective_and_gradient(x)
    assert fe == fg and np.array_equal(ge, gg)
    for c in (eager, graph):
        c.set_objective(alpha_mag=1.0)


def test_counters_advance_on_replay(pair):
    p, m, x0, eager, graph = pair
    graph.objective_and_gradient(x0)
    graph.objective_and_gradient(x0)  # now replayed
    graph.reset_counters()
    graph.objective_and_gradient(x0)
    graph.objective_and_gradient(x0)
    c = graph.counters()
    assert c.launches > 0 and c.forward_pairs == 2 * len(p.grav_xyz) * p.n_triangles()


def test_lbfgsb_same_path(pair):
    p, m, x0, eager, graph = pair
    lo, hi = m.bounds()
    xe, re = eager.lbfgsb(x0, lo, hi, max_iterations=8)
    xg, rg = graph.lbfgsb(x0, lo, hi, max_iterations=8)
    assert re.iterations == rg.iterations and re.final_value == rg.final_value
    assert np.array_equal(xe, xg)
