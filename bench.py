#!/usr/bin/env python
"""Benchmark: joint gravity + TMI forward + objective-gradient evaluations per
second on the multi-unit contact model (4 lithology groups on a 24x24x12 grid
of 100 m voxels, ~19k triangles, 64x64 stations 1 m above the flat top,
control-point stride 4, z-free vertices).

One step = one evaluation at one parameter vector: parameter scatter
(control-point interpolation + shared-vertex averaging), gz and TMI at every
station over every facet, joint misfit, and the misfit gradient with respect
to every DOF (analytic vertex derivatives contracted with the weighted
residuals; the Jacobian is never formed).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision mixed|fp64]

Precision: `mixed` (default) evaluates far and mid-field station-facet
pairs in FP32 and near ones in FP64 (gz/TMI within 1e-6, gradient within
1e-5 of the FP64 path); `fp64` evaluates every pair in FP64.

Prints one JSON line on rank 0.  `value` is whole-job evaluations/s with the
parameter vector resident in HBM; `e2e` is the same through the C ABI with
host buffers (H2D of the parameters and D2H of objective + gradient inside
the timed region).  Multi-GPU runs are independent replicas (weak scaling):
the path needs no exchange on one model.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+grad evals/s (joint gz+TMI forward and objective gradient)"
WORKLOAD = "multi-unit contact model: 4 groups, 24x24x12 voxels of 100 m, 64x64 stations at 1 m, CP stride 4"
WORKLOAD_LARGE = ("large single inversion: 6 units on a 60x60x30 grid of 100 m voxels (~194k triangles), "
                  "x/y/z-free vertices, 200x200 stations on a seeded 8-sinusoid topography, joint gz+TMI with "
                  "reference-model regularisation")
WORKLOAD_BATCH = ("batched bodies: 256 closed bodies (perturbed lat-long spheres and star-shaped prisms), "
                  "triangles log-uniform in [500, 50000], per-body square station grids of side U[16, 128] "
                  "at U[25, 100] m, one persistent forward launch")
WORKLOAD_CONSTRAINTS = ("borehole-constraint gradient on the multi-unit contact model: 64 intervals (32 within "
                        "0.3 m of control-point vertices, 32 random), 1,313 DOFs, central differences with a 1 m "
                        "step (2 x np scatter + ray-cast classification passes per gradient)")
L2_FLUSH_BYTES = 256 << 20

# Algorithmic work per station-facet pair (frozen; never tuned).  Forward: one
# gz + TMI pair sharing the solid angle and the edge line integrals, with the
# per-facet constants hoisted (unit normal, edge directions and lengths, the
# in-plane edge normals, the magnetic direction products):
#   r_a, r_b, r_c = v - o                        9 flops
#   |r_a|, |r_b|, |r_c|                          15 flops + 3 sqrt
#   triple product r_a . (r_b x r_c)             14
#   solid-angle denominator 23, atan2, factor 2  24 + 1 atan2
#   height h = n . r_a                           5
#   per edge (x 3): s1, s2 = r . e (10), numerator and denominator (2),
#     their ratio (1 div + 1), log, d_perp (5), gz/TMI accumulation (4)
#                                                66 + 3 div + 3 log
#   final gz / TMI combine                       5
#   total 138 flops (add/sub/mul 1, FMA 2) + 3 sqrt + 3 div + 3 log + 1 atan2.
# Gradient pair (both data types, analytic derivatives of the three vertices
# contracted with the residual adjoints): 331 flops; its special-function ops
# are the forward's 10 plus the three vertex-distance reciprocals, 13.
FLOPS_FWD_PAIR = 138
FLOPS_GRAD_PAIR = 331
SFU_FWD_PAIR = 10   # 3 sqrt + 3 div + 3 log + 1 atan2, one special-function op each
SFU_GRAD_PAIR = 13
# DRAM bytes (read + write) of one mixed-precision forward launch on this
# workload, per engine, from ncu captures (dram__bytes_read.sum +
# dram__bytes_write.sum): the facet records (224 bytes each, ~4.3 MB) or the
# patch blobs (~5 MB) and the stations come from DRAM once and from L2 for
# every further station block; the partial sums stay in L2.
FORWARD_DRAM_BYTES_PER_LAUNCH = {"k_forward_mixed": 7.412e6, "k_forward_patch": 9.605e6}
# Nominal B200 CUDA-core rates at the 1.965 GHz boost clock (no measured
# figure for these pipes exists in MEASURED_PEAKS.json): FP32 148 SMs x 128
# lanes x 2 flop; special-function unit 148 x 16 ops; FP64 148 x 64 x 2 flop.
CLOCK_HZ = 1.965e9
FP32_PEAK_FLOPS = 148 * 128 * 2 * CLOCK_HZ
SFU_PEAK_OPS = 148 * 16 * CLOCK_HZ
FP64_PEAK_FLOPS = 148 * 64 * 2 * CLOCK_HZ


def pair_roofline(flops: int, sfu: int, precision: str) -> float:
    """Roofline of one station-facet pair in pairs/s: the FP32 pipe or the
    special-function unit, whichever binds (FP64 pipe in FP64 mode)."""
    if precision == "fp64":
        return FP64_PEAK_FLOPS / flops
    return min(FP32_PEAK_FLOPS / flops, SFU_PEAK_OPS / sfu)


def max_over_ranks(values, dist=None, device="cpu"):
    """Element-wise maximum over ranks: every replica times its own steps and
    the job takes as long as its slowest rank."""
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def job_rate(world: int, steps: int, slowest_ms: float) -> float:
    """Whole-job evaluations/s: every rank evaluated `steps` times."""
    return world * steps / (slowest_ms / 1e3)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps; default 1000 on the contact model (about a second of device time, so "
                         "that the clock sampler sees several samples), 20 large, 5 batch, 50 otherwise")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-stations", type=int, default=256)
    ap.add_argument("--bodies", type=int, default=256,
                    help="number of bodies of the batch workload (256 is the configuration; fewer for profiling)")
    ap.add_argument("--workload", choices=["contact", "batch", "large", "constraints"], default="contact",
                    help="contact: the 4-group contact model (headline); batch: 256 batched bodies; "
                         "large: the 194k-facet single inversion")
    ap.add_argument("--lbfgs-iters", type=int, default=0,
                    help="after timing, run this many L-BFGS-B iterations and report their wall time")
    ap.add_argument("--gather", choices=["reference", "chain"], default="reference",
                    help="objective-gradient gather: the reference's DOF-vertex gather, or the exact derivative "
                         "through the control-point interpolation and shared-vertex averaging")
    ap.add_argument("--xy-derivative", choices=["analytic", "fd"], default="analytic",
                    help="x/y vertex derivatives of the gradient: closed form, or per-facet forward differences "
                         "with --xy-step (the large-inversion configuration's h = 0.5 m)")
    ap.add_argument("--xy-step", type=float, default=0.5)
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the context's default launch shapes (short profiling runs)")
    ap.add_argument("--drop-collapsed", action="store_true",
                    help="facets collapsed onto a line contribute nothing to the forward either (their reference "
                         "TMI term is rounding noise and discontinuous)")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 50 if args.impl == "reference" else {"contact": 1000, "large": 20, "batch": 5}.get(args.workload, 50)
    return args


def make_problem(workload: str = "contact", bodies: int = 256):
    from lithoinv3d_b200 import synth

    if workload == "batch":
        p = synth.batch_bodies_model(n_bodies=bodies)
    elif workload == "large":
        p = synth.large_model()
    else:
        p = synth.voxel_contact_model()
    model = p.build_model()
    return p, model


def synthetic_data(p, model):
    """Observations of a seeded true model (x0 + N(0, 5 m)) plus 1% noise,
    computed once by the GPU forward (setup only, untimed)."""
    import numpy as np

    x0 = model.assemble_parameters()
    rng = np.random.default_rng(1234)
    x_true = x0 + rng.normal(0.0, 5.0, len(x0))
    ctx = p.make_context(model)
    gz, tmi = ctx.forward(x_true)
    ctx.close()
    gstd = np.full(len(gz), 0.01 * np.std(gz))
    mstd = np.full(len(tmi), 0.01 * np.std(tmi))
    gobs = gz + gstd * rng.normal(size=len(gz))
    mobs = tmi + mstd * rng.normal(size=len(tmi))
    return x0, gobs, gstd, mobs, mstd


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.path = f"/tmp/litho_clocks_{os.getpid()}.csv"
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(p, x0, gobs, gstd, mobs, mstd, n_sta: int):
    """The reference's own CPU path (oracle/_ref, single-threaded as the
    reference is) timed on a bounded station sample of the same workload,
    scaled to whole-workload evaluations/s.  Falls back to the C restatement
    (kind "port") when the compiled reference is absent."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bindings as ob
    from lithoinv3d_b200 import synth

    S = len(p.grav_xyz)
    idx = np.linspace(0, S - 1, n_sta).astype(int)
    sub = synth.Problem(p.name, p.densities, p.susceptibilities, p.meshes, p.grav_xyz[idx], p.mag_xyz[idx],
                        inducing=p.inducing, axis_scale=p.axis_scale, cp_stride=p.cp_stride)
    if ob.ref_available():
        rm = ob.RefModel(sub, gobs[idx], gstd[idx], mobs[idx], mstd[idx])
        t0 = time.perf_counter()
        rm.objective(x0)
        rm.gradient(x0)
        dt = time.perf_counter() - t0
        kind = "reference"
    else:
        model = sub.build_model()
        om = ob.OracleModel(model.tables(), sub.densities, sub.susceptibilities, sub.inducing)
        t0 = time.perf_counter()
        om.scatter(x0)
        om.forward_gz(sub.grav_xyz)
        om.forward_tmi(sub.mag_xyz)
        om.jacobian(sub.grav_xyz, 0)
        om.forward_gz(sub.grav_xyz)
        om.jacobian(sub.mag_xyz, 1)
        om.forward_tmi(sub.mag_xyz)
        dt = time.perf_counter() - t0
        kind = "port"
    per_eval = dt * S / n_sta
    return {"value": 1.0 / per_eval, "unit": "evals/s", "cores": 1, "kind": kind,
            "sample": f"one objective+gradient evaluation on {n_sta} of {S} stations "
                      f"({dt:.1f} s), scaled by station count"}


REF_STATIONS_PER_CORE = 8


def _ref_process(conn, idx, seed):
    """One single-threaded reference process (the reference has no threading)
    over the station sample `idx` of the contact workload.  Set-up, untimed:
    the seeded geometry from numpy (synth.voxel_contact_model builds meshes
    only), the reference's LithologyModel / forwards / JointObjective
    (oracle/_ref), and observations of a seeded true model computed by the
    reference's own forward.  Each step message then times exactly one
    objective evaluation and one gradient (objective.cpp:83-105,
    joint_objective.cpp:42-173) and sends back that duration.  Nothing from
    the GPU library is loaded here."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bindings as ob
    from lithoinv3d_b200 import synth

    p = synth.voxel_contact_model()
    sub = synth.Problem(p.name, p.densities, p.susceptibilities, p.meshes, p.grav_xyz[idx], p.mag_xyz[idx],
                        inducing=p.inducing, axis_scale=p.axis_scale, cp_stride=p.cp_stride)
    truth = ob.RefModel(sub)
    x0 = truth.assemble()
    rng = np.random.default_rng(seed)
    x_true = x0 + rng.normal(0.0, 5.0, len(x0))
    gz, tmi = truth.forward_gz(x_true), truth.forward_tmi(x_true)
    del truth
    gstd = np.full(len(gz), 0.01 * max(float(np.sqrt(np.mean(gz ** 2))), 1e-30))
    mstd = np.full(len(tmi), 0.01 * max(float(np.sqrt(np.mean(tmi ** 2))), 1e-30))
    rm = ob.RefModel(sub, gz + gstd * rng.normal(size=len(gz)), gstd, tmi + mstd * rng.normal(size=len(tmi)), mstd)
    conn.send(("ready", len(p.grav_xyz), p.n_triangles(), int(len(x0))))
    while True:
        msg = conn.recv()
        if msg != "step":
            break
        t0 = time.perf_counter()
        rm.objective(x0)
        rm.gradient(x0)
        conn.send(time.perf_counter() - t0)
    conn.close()


def run_reference(args):
    """--impl reference: the reference's CPU implementation of the path (its
    own sources compiled into oracle/_ref; the C restatement is not used
    here) on every host core, one persistent single-threaded process per core
    over a station sample of the contact workload.  A step sends every
    process one objective + gradient evaluation of its stations; the step
    time is the slowest process's own timed region, so spawn, set-up and
    pickling stay outside.  Under torchrun only rank 0 runs."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp

    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bindings as ob
    from lithoinv3d_b200 import synth

    if not ob.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_litho.so (the reference's own "
                                                             "sources, built by oracle/Makefile) is not present"}))
        return
    try:
        ncore = len(os.sched_getaffinity(0))
    except AttributeError:
        ncore = os.cpu_count() or 1
    S = len(synth.voxel_contact_model(n_side=64).grav_xyz)
    n_sample = min(S, REF_STATIONS_PER_CORE * ncore)
    idx_all = np.linspace(0, S - 1, n_sample).astype(int)
    chunks = [idx_all[i::ncore] for i in range(ncore)]
    ctx = mp.get_context("spawn")
    procs, conns = [], []
    for i, c in enumerate(chunks):
        a, b = ctx.Pipe()
        pr = ctx.Process(target=_ref_process, args=(b, c, 1234 + i), daemon=True)
        pr.start()
        procs.append(pr)
        conns.append(a)
    info = [cn.recv() for cn in conns]
    _, S, T, np_ = info[0]
    times = []
    for step in range(args.warmup + args.steps):
        for cn in conns:
            cn.send("step")
        dt = max(cn.recv() for cn in conns)  # the slowest process ends the step
        if step >= args.warmup:
            times.append(dt)
    for cn in conns:
        cn.send("stop")
    for pr in procs:
        pr.join(timeout=30)
    t_step = sum(times) / len(times)
    value = (n_sample / S) / t_step  # whole-workload evaluations per second
    sample = (f"{n_sample} of {S} stations per step ({REF_STATIONS_PER_CORE} per process), one single-threaded "
              f"reference process per core ({ncore}); each step times one objective + gradient per process, "
              f"the slowest process's time; evals/s scaled by station count")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3,
            "ms_per_full_evaluation": t_step * 1e3 * S / n_sample,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded voxel model and observations)",
            "config": workload_config("contact", T, S, np_),
            "details": {"stations_per_step": int(n_sample), "processes": ncore},
            "cpu_baseline": {"value": value, "unit": "evals/s", "cores": ncore, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def workload_config(workload: str, triangles: int, stations: int, dofs: int, bodies: int = 256) -> dict:
    """The workload as both arms name it (identical dicts for the same
    workload); implementation details go elsewhere in the line."""
    name = {"batch": WORKLOAD_BATCH.replace("256", str(bodies)), "large": WORKLOAD_LARGE}.get(workload, WORKLOAD)
    return {"workload": name, "triangles": int(triangles), "stations": int(stations), "dofs": int(dofs),
            "l2": "GPU arm: L2 flushed between steps (256 MiB write); CPU arm: not applicable"}


def constraint_intervals(pos, cp_vertices, n_group, rng, n_near=32, n_random=32):
    """Borehole intervals for the constraint workload: midpoints 0.3 m above
    or below control-point vertices (a 1 m DOF step flips their class) and
    random midpoints inside the model; half-thickness U(0.5, 40) m."""
    import numpy as np

    pick = pos[rng.choice(cp_vertices, n_near, replace=False)]
    mid = pick + np.where(rng.random(n_near) < 0.5, 0.3, -0.3)[:, None] * np.array([0.0, 0.0, 1.0])
    mid = np.concatenate([mid, rng.uniform([-1150.0, -1150.0, -1150.0], [1150.0, 1150.0, -20.0], (n_random, 3))])
    half = rng.uniform(0.5, 40.0, len(mid))
    group = rng.integers(0, n_group, len(mid)).astype(np.int32)
    return mid[:, :2].copy(), -mid[:, 2] - half, -mid[:, 2] + half, group


def run_constraints(args):
    """--workload constraints: ConstraintHandler::gradient (lf_constraint_gradient)
    per second on one GPU; the CPU baseline is the compiled reference's
    ConstraintHandler::evaluate (one scatter + classification of every
    interval, the unit of the gradient's 2 np evaluations) on a sample."""
    import numpy as np
    import torch

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    p, model = make_problem("contact")
    t = model.tables()
    x0 = model.assemble_parameters()
    cp_vertices = np.unique(t["ref_vertex"][t["ref_axis"] == 2])
    xy, zt, zb, group = constraint_intervals(t["pos"], cp_vertices, len(p.meshes), np.random.default_rng(11))
    ctx = p.make_context(model, device=local)
    ctx.set_constraints(xy, zt, zb, group)
    for _ in range(args.warmup):
        g = ctx.constraint_gradient(x0)
    torch.cuda.synchronize()
    ctx.reset_counters()
    with ClockSampler(local) as clocks:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            g = ctx.constraint_gradient(x0)  # synchronous: H2D params, 2 np passes, D2H gradient
        dt = time.perf_counter() - t0
    launches = int(ctx.counters().launches)
    value = args.steps / dt
    np_ = model.n_dofs
    line = {"metric": "constraint-gradient evals/s (ConstraintHandler::gradient)", "value": value,
            "unit": "evals/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded voxel model and intervals)",
            "config": {"workload": WORKLOAD_CONSTRAINTS, "intervals": len(xy), "dofs": np_,
                       "triangles": int(len(t["tri"])), "nonzero_gradient_entries": int(np.count_nonzero(g))},
            "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 8 * np_,
                    "d2h_bytes_per_step": 8 * np_},
            "gpu_launches": launches, "launches_per_step": launches / args.steps,
            "clocks": clocks.summary()}
    if rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_bindings as ob

        if ob.ref_available():
            rm = ob.RefModel(p)
            rm.set_constraints(xy, zt, zb, group)
            n_eval = 20
            t0 = time.perf_counter()
            for j in range(n_eval):
                xp = x0.copy()
                xp[j] += 1.0
                rm.constraint_value(xp)
            per_eval = (time.perf_counter() - t0) / n_eval
            cpu = 1.0 / (2 * np_ * per_eval)
            line["cpu_baseline"] = {"value": cpu, "unit": "evals/s", "cores": 1, "kind": "reference",
                                    "sample": f"{n_eval} ConstraintHandler::evaluate calls ({per_eval * 1e3:.1f} ms "
                                              f"each), scaled to the gradient's 2 x {np_} evaluations"}
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "constraints":
        run_constraints(args)
        return
    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from lithoinv3d_b200 import PREC_FP64, PREC_MIXED

    p, model = make_problem(args.workload, args.bodies)
    x0, gobs, gstd, mobs, mstd = synthetic_data(p, model)
    ctx = p.make_context(model, device=local, grav_obs=gobs, grav_std=gstd, mag_obs=mobs, mag_std=mstd)
    ctx.set_precision(PREC_MIXED if args.precision == "mixed" else PREC_FP64)
    if args.workload == "large":  # reference-model regularisation around the start (reference_model.cpp:16-25)
        ctx.set_objective(alpha_mag=1.0, ref_weight=1e-3, ref_params=x0)
        ctx.set_scatter_stateless(True)
    if args.gather == "chain":
        from lithoinv3d_b200 import GATHER_CHAIN

        ctx.set_gradient_gather(GATHER_CHAIN)
    if args.drop_collapsed:
        from lithoinv3d_b200.api import COLLAPSED_DROP

        ctx.set_collapsed_facets(COLLAPSED_DROP)
    if args.xy_derivative == "fd":
        from lithoinv3d_b200 import XY_FORWARD_DIFFERENCE

        ctx.set_xy_derivative(XY_FORWARD_DIFFERENCE, args.xy_step)
    ctx.set_graph_mode(True)
    tuned = ctx.tuning() if args.no_autotune else ctx.autotune(x0, repeats=3)[0]
    np_ = model.n_dofs
    dev = torch.device("cuda", local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    xs = [torch.tensor(x0 + d, dtype=torch.float64, device=dev) for d in (0.0, 0.5)]
    d_f = torch.zeros(1, dtype=torch.float64, device=dev)
    d_g = torch.zeros(np_, dtype=torch.float64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()

    def step(i):
        ctx.objective_grad_device(xs[i % 2].data_ptr(), d_f.data_ptr(), d_g.data_ptr())

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()

    # ---- device-resident timing: per-step events on the library's stream;
    # each evaluation is a replayed CUDA graph (captured during warm-up) ----
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    ctx.reset_counters()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(i))  # evicts L2 between steps (outside the events)
                evs[i][0].record(stream)
            step(i)
            with torch.cuda.stream(stream):
                evs[i][1].record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = sum(step_ms)
    cnt = ctx.counters()
    near_pairs = ctx.near_pairs() if args.precision == "mixed" else 0
    # ---- per-kernel device times for the roofline: a separate pass with
    # events around every pair kernel (direct launches, not graph replay) ----
    ctx.set_profiling(True)
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(i))
        step(i)
    torch.cuda.synchronize()
    fwd_ms, fwd_n, grad_ms, grad_n = ctx.kernel_times()
    ctx.set_profiling(False)
    near_frac = near_pairs / max(cnt.forward_pairs, 1) if args.precision == "mixed" else 1.0
    launches = int(cnt.launches)
    pairs_fwd = int(cnt.forward_pairs)
    pairs_grad = int(cnt.gradient_pairs)

    # ---- end to end through the C ABI with pinned host buffers ----
    hx = torch.from_numpy(x0.copy()).pin_memory()
    hg = torch.zeros(np_, dtype=torch.float64).pin_memory()
    hx_np, hg_np = hx.numpy(), hg.numpy()
    import ctypes as C

    lib = ctx.lib
    fbuf = np.zeros(1)
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for i in range(2):
        lib.lf_objective_grad(ctx.h, hx_np.ctypes.data_as(C.POINTER(C.c_double)),
                              fbuf.ctypes.data_as(C.POINTER(C.c_double)), hg_np.ctypes.data_as(C.POINTER(C.c_double)))
    torch.cuda.synchronize()
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(i))
            e2e_ev[i][0].record(stream)
        st = lib.lf_objective_grad(ctx.h, hx_np.ctypes.data_as(C.POINTER(C.c_double)),
                                   fbuf.ctypes.data_as(C.POINTER(C.c_double)),
                                   hg_np.ctypes.data_as(C.POINTER(C.c_double)))
        assert st == 0, st
        with torch.cuda.stream(stream):
            e2e_ev[i][1].record(stream)
    torch.cuda.synchronize()
    e2e_ms = sum(a.elapsed_time(b) for a, b in e2e_ev)

    # max over ranks (replicas)
    total_ms, e2e_ms = max_over_ranks([total_ms, e2e_ms], dist, dev)
    ms_per_step = total_ms / args.steps
    value = job_rate(world, args.steps, total_ms)
    e2e_value = job_rate(world, args.steps, e2e_ms)

    # dominant kernel roofline: pairs/s against the pipe that binds the
    # algorithmic per-pair work (FP32 or special-function unit in mixed mode,
    # FP64 in FP64 mode), reported as flop-equivalents
    grad_per_launch_ms = grad_ms / max(grad_n, 1)
    fwd_per_launch_ms = fwd_ms / max(fwd_n, 1)
    pps_fwd = pairs_fwd / max(fwd_ms / 1e3, 1e-12)
    pps_grad = pairs_grad / max(grad_ms / 1e3, 1e-12)
    if grad_ms >= fwd_ms:
        kname = "k_gradient_warp_fp64 + k_gradient_warp_far32" if args.precision == "mixed" else "k_gradient_warp_fp64"
        kms, pps, flops, sfu = grad_per_launch_ms, pps_grad, FLOPS_GRAD_PAIR, SFU_GRAD_PAIR
    else:
        kname = (("k_forward_mixed" if tuned.fwd_engine == 0 else "k_forward_patch") if args.precision == "mixed"
                 else "k_forward_fp64")
        kms, pps, flops, sfu = fwd_per_launch_ms, pps_fwd, FLOPS_FWD_PAIR, SFU_FWD_PAIR
    peak_pps = pair_roofline(flops, sfu, args.precision)
    roofline = {"bound": "fp64" if args.precision == "fp64" else "fp32+sfu", "kernel": kname,
                "achieved": pps * flops / 1e12, "peak": peak_pps * flops / 1e12, "unit": "TFLOP/s",
                "frac": pps / peak_pps,
                "fp32_pipe_frac": (pps * flops / FP32_PEAK_FLOPS) if args.precision == "mixed" else None,
                "traffic": (FORWARD_DRAM_BYTES_PER_LAUNCH.get(kname) if args.workload == "contact" else None),
                "peak_source": ("nominal CUDA-core rates at 1.965 GHz (FP32 74.4 TFLOP/s, SFU 4.65 Tops/s, "
                                "FP64 37.2 TFLOP/s); MEASURED_PEAKS.json holds only HBM and bf16 GEMM figures"),
                "flops_per_pair": flops, "sfu_ops_per_pair": sfu, "kernel_ms_per_launch": kms,
                "pairs_per_s": {"forward": pps_fwd, "gradient": pps_grad}}

    line = {"metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic (seeded voxel model and observations)",
            "config": workload_config(args.workload, p.n_triangles(), len(p.grav_xyz), np_, args.bodies),
            "details": {"parallelism": f"replicas x{world}", "precision": args.precision,
                        "fp64_near_pair_fraction": round(near_frac, 4), "cuda_graph": True,
                        "gradient_gather": args.gather,
                        "collapsed_facets": "dropped" if args.drop_collapsed else "reference",
                        "xy_derivative": (f"forward difference, h = {args.xy_step} m" if args.xy_derivative == "fd"
                                          else "analytic"),
                        "tuning": {"fwd_target_blocks": tuned.fwd_target_blocks,
                                   "grad_target_warps": tuned.grad_target_warps,
                                   "near_tiles_per_chunk": tuned.near_tiles_per_chunk,
                                   "patch_threads": tuned.patch_threads, "far_ratio": tuned.far_ratio,
                                   "fwd_engine": "facet" if tuned.fwd_engine == 0 else "patch"}},
            "e2e": {"value": e2e_value, "unit": "evals/s", "h2d_bytes_per_step": 8 * np_,
                    "d2h_bytes_per_step": 8 * (np_ + 1)},
            "gpu_launches": launches, "roofline": roofline}
    clk = clocks.summary()
    line["clocks"] = clk
    if args.lbfgs_iters > 0:  # the inversion itself (untimed by the events above; host wall clock)
        lo, hi = model.bounds()
        if args.workload == "large":  # +-50 m around the start in every free axis
            lo, hi = np.maximum(lo, x0 - 50.0), np.minimum(hi, x0 + 50.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, res = ctx.lbfgsb(x0, lo, hi, max_iterations=args.lbfgs_iters)
        wall = time.perf_counter() - t0
        f0 = ctx.objective(x0)
        line["details"]["lbfgsb"] = {"iterations": res.iterations, "evaluations": res.evaluations,
                                    "gradients": res.gradients, "wall_s": wall, "objective_start": f0,
                                    "objective_final": res.final_value, "message": res.message.decode(),
                                    "gather": args.gather}
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload == "contact":
        try:
            line["cpu_baseline"] = cpu_baseline(p, x0, gobs, gstd, mobs, mstd, args.cpu_stations)
        except Exception as e:  # the baseline is reported, never the target
            line["cpu_baseline"] = {"value": None, "error": str(e)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
