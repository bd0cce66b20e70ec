"""Generates tests/golden/*.npz from the reference's own code compiled here
(oracle/_ref/libref_litho.so, built by oracle/Makefile from the reference
sources).  Run from the repository root:  python tests/golden/make_golden.py

The reference ships no golden vectors for this path, so these fixtures are
its outputs on small seeded inputs: geometry primitives (including the
degenerate branches), and the forward, forward-difference Jacobian,
objective and gradient of two small models.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle_bindings as ob  # noqa: E402
from lithoinv3d_b200 import synth  # noqa: E402

_dp = C.POINTER(C.c_double)


def primitives(lib):
    rng = np.random.default_rng(20261203)
    n = 200
    tri = rng.normal(0, 100, (n, 3, 3))
    obs = rng.normal(0, 150, (n, 3))
    # degenerate and near-degenerate cases
    tri[0] = [[0, 0, 0], [10, 0, 0], [0, 10, 0]]; obs[0] = [0, 0, 0]          # station on a vertex
    tri[1] = [[0, 0, 0], [10, 0, 0], [0, 10, 0]]; obs[1] = [5, 0, 0]          # on an edge
    tri[2] = [[0, 0, 0], [10, 0, 0], [0, 10, 0]]; obs[2] = [20, 0, 0]         # on an edge line, outside
    tri[3] = [[0, 0, 0], [10, 0, 0], [0, 10, 0]]; obs[3] = [2, 2, 0]          # in the facet plane, inside
    tri[4] = [[0, 0, 0], [10, 0, 0], [0, 10, 0]]; obs[4] = [2, 2, 1e-9]       # just above
    tri[5] = [[0, 0, 0], [10, 0, 0], [20, 0, 0]]; obs[5] = [3, 4, 5]          # zero-area facet
    tri[6] = [[0, 0, 0], [0, 0, 0], [0, 10, 0]]; obs[6] = [3, 4, 5]           # degenerate edge
    tri[7] = [[0, 0, 0], [10, 0, 0], [0, 10, 0]]; obs[7] = [-5, 0, 0]         # edge line, behind p1
    for f in ("ref_solid_angle", "ref_line_integral_term", "ref_gravity_facet", "ref_magnetic_facet"):
        getattr(lib, f).restype = C.c_double
    m = np.array([0.3, -0.2, -0.93]); m /= np.linalg.norm(m)
    fd = np.array([0.5, 0.0, -0.866]); fd /= np.linalg.norm(fd)
    sa, lit, gf, mf = (np.zeros(n) for _ in range(4))
    p = lambda a: np.ascontiguousarray(a, np.float64).ctypes.data_as(_dp)  # noqa: E731
    for i in range(n):
        a, b, c = tri[i]
        sa[i] = lib.ref_solid_angle(p(a), p(b), p(c), p(obs[i]))
        lit[i] = lib.ref_line_integral_term(p(a), p(b), p(obs[i]))
        gf[i] = lib.ref_gravity_facet(p(obs[i]), p(a), p(b), p(c))
        mf[i] = lib.ref_magnetic_facet(p(obs[i]), p(a), p(b), p(c), p(m), p(fd))
    np.savez_compressed(os.path.join(HERE, "primitives.npz"), tri=tri, obs=obs, mdir=m, fdir=fd,
                        solid_angle=sa, line_integral=lit, gravity_facet=gf, magnetic_facet=mf)


def model_case(name, problem, seed):
    rng = np.random.default_rng(seed)
    S = len(problem.grav_xyz)
    gobs, gstd = rng.normal(0, 1, S), np.abs(rng.normal(0.5, 0.05, S))
    mobs, mstd = rng.normal(0, 20, S), np.abs(rng.normal(2.0, 0.1, S))
    rm = ob.RefModel(problem, gobs, gstd, mobs, mstd, alpha_mag=0.5)
    x0 = rm.assemble()
    x = x0 + rng.normal(0, 3, len(x0))
    off, rv, ra, rs = rm.dof_tables()
    out = dict(x0=x0, x=x, gobs=gobs, gstd=gstd, mobs=mobs, mstd=mstd, alpha_mag=0.5,
               dof_off=off, ref_vertex=rv, ref_axis=ra, ref_scale=rs)
    lo, hi = rm.bounds()
    out.update(lower=lo, upper=hi)
    out["gz"] = rm.forward_gz(x)
    out["tmi"] = rm.forward_tmi(x)
    out["pos"] = rm.positions()
    out["J_gz"] = rm.jacobian_gz(x)
    out["J_tmi"] = rm.jacobian_tmi(x)
    out["objective"] = rm.objective(x)
    out["gradient"] = rm.gradient(x)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


def main():
    if not ob.ref_available():
        raise SystemExit("build oracle/_ref first: make -C oracle")
    lib = ob.ref()
    primitives(lib)
    model_case("icosphere_s1", synth.icosphere_model(subdiv=1, n_side=6, spacing=90.0), 11)
    model_case("voxel_8x8x4_cp2", synth.voxel_contact_model(shape=(8, 8, 4), n_side=6, cp_stride=2, seed=4), 12)


if __name__ == "__main__":
    main()
