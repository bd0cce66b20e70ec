"""The drop-in inside the reference: GpuGravityForward / GpuMagneticForward
(oracle/gpu_dropin.hpp, compiled against the reference's own headers) behind
its ForwardModel interface, driven by the reference's unmodified
ObjectiveFunction, JointObjective and LBFGSBOptimizer (objective.cpp,
joint_objective.cpp, lbfgsb_optimizer.cpp in oracle/_ref).

* compute: the GPU operators against GravityForward::compute /
  MagneticForward::compute on the same model and parameters, 1e-10 relative
  (FP64 path);
* computeJacobian: the analytic GPU Jacobian against the true derivative
  (oracle, Richardson central differences), 1e-6; the reference's own
  per-facet forward-difference Jacobian (h = 1e-4 m) is within 1e-3 of both
  (its rounding error, amplified by the small step, is ~1e-4 here);
* the single-body inversion (icosphere, 16 x 16 stations, 30 L-BFGS-B
  iterations, z bounded to +-100 m): the reference optimizer on the GPU
  operators ends within 2% of the misfit it reaches on its own operators."""
import numpy as np
import pytest

from oracle_bindings import TRUE_H, OracleModel, RefModel, ref_available
from lithoinv3d_b200 import library_path
from test_gpu_inversion import BOUND, c1_data, c1_problem

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="reference library not built")]


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_reference_objective_and_optimizer_on_gpu_operators():
    p = c1_problem(n_side=16, spacing=125.0)
    model = p.build_model()
    x0, x_true, gobs, gstd, tobs, tstd = c1_data(p, model)
    cpu = RefModel(p, grav_obs=gobs, grav_std=gstd, mag_obs=tobs, mag_std=tstd)
    gpu = RefModel(p, grav_obs=gobs, grav_std=gstd, mag_obs=tobs, mag_std=tstd)
    gpu.use_gpu(library_path())
    x = x0 + np.random.default_rng(4).normal(0.0, 1.0, len(x0))
    for params in (x0, x):
        assert rel(gpu.forward_gz(params), cpu.forward_gz(params)) < 1e-10
        assert rel(gpu.forward_tmi(params), cpu.forward_tmi(params)) < 1e-10
    truth = OracleModel(model.tables(), p.densities, p.susceptibilities, p.inducing)
    truth.scatter(x)
    for kind, gpu_j, cpu_j in ((2, gpu.jacobian_gz(x), cpu.jacobian_gz(x)), (3, gpu.jacobian_tmi(x),
                                                                              cpu.jacobian_tmi(x))):
        true_j = truth.jacobian(p.grav_xyz, kind, true_h=TRUE_H)
        assert rel(gpu_j, true_j) < 1e-6
        assert rel(cpu_j, true_j) < 1e-3 and rel(gpu_j, cpu_j) < 1e-3
    o_cpu, o_gpu = cpu.objective(x), gpu.objective(x)
    assert abs(o_gpu[4] - o_cpu[4]) <= 1e-9 * o_cpu[4]
    fresh_cpu = RefModel(p, grav_obs=gobs, grav_std=gstd, mag_obs=tobs, mag_std=tstd)
    fresh_gpu = RefModel(p, grav_obs=gobs, grav_std=gstd, mag_obs=tobs, mag_std=tstd)
    fresh_gpu.use_gpu(library_path())
    _, f_cpu, it_cpu = fresh_cpu.lbfgsb(x0, x0 - BOUND, x0 + BOUND, max_iter=30)
    _, f_gpu, it_gpu = fresh_gpu.lbfgsb(x0, x0 - BOUND, x0 + BOUND, max_iter=30)
    f0 = cpu.objective(x0)[4]
    assert f_gpu < 0.5 * f0 and f_cpu < 0.5 * f0
    assert abs(f_gpu - f_cpu) <= 0.02 * f_cpu, (f_gpu, f_cpu, it_gpu, it_cpu)
