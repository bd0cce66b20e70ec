"""The large single inversion (194k facets, 40,000 stations on topography,
x/y/z-free vertices, joint data, reference-model regularisation): mixed
forward against the oracle at 40 stations (1e-6), mixed gradient against
the FP64 path at zero observations (1e-5), and a few L-BFGS-B iterations
that lower the objective."""
import numpy as np
import pytest

from oracle_bindings import OracleModel
from lithoinv3d_b200 import PREC_MIXED, synth

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.fixture(scope="module")
def large():
    p = synth.large_model()
    m = p.build_model()
    x0 = m.assemble_parameters()
    return p, m, x0


def test_large_forward_matches_oracle(large):
    p, m, x0 = large
    x = x0 + np.random.default_rng(1).normal(0, 2, len(x0))
    ctx = p.make_context(m)
    ctx.set_precision(PREC_MIXED)
    gz, tmi = ctx.forward(x)
    sub = np.linspace(0, len(p.grav_xyz) - 1, 40).astype(int)
    om = OracleModel(m.tables(), p.densities, p.susceptibilities, p.inducing)
    om.scatter(x)
    assert rel(gz[sub], om.forward_gz(p.grav_xyz[sub])) < 1e-6
    assert rel(tmi[sub], om.forward_tmi(p.mag_xyz[sub])) < 1e-6


def test_large_gradient_and_inversion(large):
    p, m, x0 = large
    x = x0 + np.random.default_rng(2).normal(0, 2, len(x0))
    zeros = np.zeros(len(p.grav_xyz))
    c64 = p.make_context(m, grav_obs=zeros, mag_obs=zeros)
    c32 = p.make_context(m, grav_obs=zeros, mag_obs=zeros)
    c32.set_precision(PREC_MIXED)
    _, g64 = c64.objective_and_gradient(x)
    _, g32 = c32.objective_and_gradient(x)
    assert rel(g32, g64) < 1e-5
    c64.close()
    gobs, mobs = c32.forward(x)
    # data errors of 1% of the data RMS and +-50 m bounds around the start, as
    # an inversion of this model would set them (with unit weights and
    # unbounded x/y the first steepest-descent trial step is kilometres long)
    gstd = np.full(len(gobs), 0.01 * np.sqrt(np.mean(gobs ** 2)))
    mstd = np.full(len(mobs), 0.01 * np.sqrt(np.mean(mobs ** 2)))
    ctx = p.make_context(m, grav_obs=gobs, grav_std=gstd, mag_obs=mobs, mag_std=mstd)
    ctx.set_precision(PREC_MIXED)
    ctx.set_scatter_stateless(True)  # line-search trials must not leave displaced vertices behind
    ctx.set_objective(alpha_mag=1.0, ref_weight=1e-3, ref_params=x0)
    f0 = ctx.objective(x0)
    _, res = ctx.lbfgsb(x0, x0 - 50.0, x0 + 50.0, max_iterations=5)
    assert res.final_value < f0


def test_stateless_scatter_is_path_independent(large):
    """Default: the reference's path-dependent averaging (the model after p2
    depends on having evaluated p1 first); stateless: it does not."""
    p, m, x0 = large
    rng = np.random.default_rng(3)
    x1, x2 = x0 + rng.normal(0, 30, len(x0)), x0 + rng.normal(0, 2, len(x0))
    for stateless in (False, True):
        a, b = p.make_context(m), p.make_context(m)
        for c in (a, b):
            c.set_scatter_stateless(stateless)
        a.forward(x1)
        ga, _ = a.forward(x2)
        gb, _ = b.forward(x2)
        if stateless:
            assert np.array_equal(ga, gb)
        else:
            assert not np.array_equal(ga, gb)
