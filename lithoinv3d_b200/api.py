"""Python host API over the C ABI (include/litho_gpu.h).

`Model` is the setup-time lithology model (groups, closed meshes, vertex
freedoms, global DOFs, control points); `Context` owns one CUDA device
context and evaluates the forward, objective, gradient, Jacobian and the
projected L-BFGS inversion on it.  Arrays are numpy float64 / int32 / uint8.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _native
from ._native import Counters, LbfgsbOptions, LbfgsbResult, ModelInfo, Tuning

# VertexFreedom numbering (surface_mesh.h:9-19)
FIXED, Z_ONLY, X_ONLY, Y_ONLY, ALONG_VECTOR, XY_FREE, XZ_FREE, YZ_FREE, XYZ_FREE = range(9)
GRAVITY, MAGNETIC = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
GATHER_REFERENCE, GATHER_CHAIN = 0, 1
XY_ANALYTIC, XY_FORWARD_DIFFERENCE = 0, 1
FWD_FACET, FWD_PATCH = 0, 1
COLLAPSED_KEEP, COLLAPSED_DROP = 0, 1
UNIT_GRAVITY, UNIT_INDUCED, UNIT_DIRECTION, UNIT_REMANENCE = range(4)


class LithoError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"{_native.STATUS.get(status, status)}: {msg}")


def _d(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _u8(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def read_surface(path: str):
    """lf_read_surface: (vertices [n, 3], triangles [m, 3] 0-based) of a .ts or .obj file."""
    lib = _native.load()
    nv, nt = C.c_int(0), C.c_int(0)
    b = str(path).encode()
    st = lib.lf_read_surface(b, C.byref(nv), C.byref(nt), None, None)
    if st != 0:
        raise LithoError(st, f"read_surface: {path}")
    xyz = np.zeros((nv.value, 3))
    tri = np.zeros((nt.value, 3), np.int32)
    st = lib.lf_read_surface(b, C.byref(nv), C.byref(nt), _d(xyz), _i(tri))
    if st != 0:
        raise LithoError(st, f"read_surface: {path}")
    return xyz, tri


def write_tsurf(path: str, name: str, xyz, tri):
    """lf_write_tsurf: a GOCAD TSurf of the given vertices and triangles."""
    lib = _native.load()
    x = f64(xyz).reshape(-1, 3)
    t = i32(tri).reshape(-1, 3)
    st = lib.lf_write_tsurf(str(path).encode(), name.encode(), len(x), _d(x), len(t), _i(t))
    if st != 0:
        raise LithoError(st, f"write_tsurf: {path}")


class Model:
    """Host lithology model (LithologyModel / SurfaceMesh setup semantics)."""

    def __init__(self):
        self.lib = _native.load()
        h = C.c_void_p()
        self._check(self.lib.lf_model_create(C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.lf_model_destroy(self.h)
            self.h = None

    @staticmethod
    def _check(st: int, what: str = ""):
        if st != 0:
            raise LithoError(st, what)

    def add_group(self, gid: int, density: float, susceptibility: float = 0.0, rem_magnitude: float = 0.0,
                  rem_inclination: float = 0.0, rem_declination: float = 0.0,
                  rem_vector: Optional[Sequence[float]] = None) -> int:
        out = C.c_int(-1)
        rv = f64(rem_vector) if rem_vector is not None else None
        self._check(self.lib.lf_model_add_group(self.h, gid, density, susceptibility, rem_magnitude,
                                                rem_inclination, rem_declination, _d(rv), C.byref(out)),
                    "add_group")
        return out.value

    def set_group_mesh(self, group: int, vertices, triangles, freedom) -> None:
        v = f64(vertices).reshape(-1, 3)
        t = i32(triangles).reshape(-1, 3)
        fr = np.ascontiguousarray(np.broadcast_to(np.asarray(freedom, dtype=np.uint8), (len(v),)))
        self._check(self.lib.lf_model_set_group_mesh(self.h, group, len(v), _d(v), _u8(fr), len(t), _i(t)),
                    "set_group_mesh")

    def set_axis_scale(self, axis: int, scale: float, group: int = -1) -> None:
        self._check(self.lib.lf_model_set_axis_scale(self.h, group, axis, scale), "set_axis_scale")

    def set_depth_bounds(self, min_z: float, max_z: float, group: int = -1) -> None:
        self._check(self.lib.lf_model_set_depth_bounds(self.h, group, min_z, max_z), "set_depth_bounds")

    def set_interior_grid(self, interior_dim: int, padding_rings: int, group: int = -1) -> None:
        self._check(self.lib.lf_model_set_interior_grid(self.h, group, interior_dim, padding_rings))

    def set_control_point_stride(self, stride: int) -> int:
        out = C.c_int(0)
        self._check(self.lib.lf_model_set_control_point_stride(self.h, stride, C.byref(out)))
        return out.value

    def set_mesh_control_point_stride(self, group: int, stride: int) -> int:
        out = C.c_int(0)
        self._check(self.lib.lf_model_set_mesh_control_point_stride(self.h, group, stride, C.byref(out)))
        return out.value

    def build_shared_vertex_sync(self) -> None:
        self._check(self.lib.lf_model_build_shared_vertex_sync(self.h))

    def apply_model_bounds(self, margin_multiplier: float = 1.0) -> None:
        self._check(self.lib.lf_model_apply_model_bounds(self.h, margin_multiplier))

    def info(self) -> ModelInfo:
        inf = ModelInfo()
        self._check(self.lib.lf_model_get_info(self.h, C.byref(inf)))
        return inf

    @property
    def n_dofs(self) -> int:
        return self.info().n_dofs

    def assemble_parameters(self) -> np.ndarray:
        p = np.zeros(self.n_dofs)
        self._check(self.lib.lf_model_assemble_parameters(self.h, _d(p)))
        return p

    def bounds(self):
        n = self.n_dofs
        lo, hi = np.zeros(n), np.zeros(n)
        self._check(self.lib.lf_model_get_bounds(self.h, _d(lo), _d(hi)))
        return lo, hi

    def apply_parameters(self, params) -> None:
        p = f64(params)
        self._check(self.lib.lf_model_apply_parameters(self.h, _d(p)))

    def positions(self) -> np.ndarray:
        out = np.zeros((self.info().n_vertices, 3))
        self._check(self.lib.lf_model_get_positions(self.h, _d(out)))
        return out

    def tables(self) -> dict:
        inf = self.info()
        t = dict(
            pos=np.zeros((inf.n_vertices, 3)), tri=np.zeros((inf.n_triangles, 3), np.int32),
            grp_tri_off=np.zeros(inf.n_groups + 1, np.int32), dof_off=np.zeros(inf.n_dofs + 1, np.int32),
            ref_vertex=np.zeros(inf.n_refs, np.int32), ref_axis=np.zeros(inf.n_refs, np.uint8),
            ref_scale=np.zeros(inf.n_refs), interp_off=np.zeros(inf.n_vertices + 1, np.int32),
            interp_src=np.zeros(inf.n_interp, np.int32), interp_w=np.zeros(inf.n_interp),
            sync_off=np.zeros(inf.n_sync + 1, np.int32), sync_vertex=np.zeros(inf.n_sync_entries, np.int32))
        self._check(self.lib.lf_model_export_tables(
            self.h, _d(t["pos"]), _i(t["tri"]), _i(t["grp_tri_off"]), _i(t["dof_off"]), _i(t["ref_vertex"]),
            _u8(t["ref_axis"]), _d(t["ref_scale"]), _i(t["interp_off"]), _i(t["interp_src"]), _d(t["interp_w"]),
            _i(t["sync_off"]), _i(t["sync_vertex"])))
        return t


class Context:
    """One device context: forward / objective / gradient / Jacobian / L-BFGS-B.

    Mirrors the reference's operator API: `forward_gravity` is
    GravityForward::compute, `forward_magnetic` MagneticForward::compute,
    `jacobian` computeJacobian, `objective_components` JointObjective::
    evaluateComponents and `objective_and_gradient` evaluate + gradient."""

    def __init__(self, device: int = 0):
        self.lib = _native.load()
        h = C.c_void_p()
        st = self.lib.lf_create(C.byref(h), device)
        if st != 0:
            raise LithoError(st, "lf_create (a CUDA device is required)")
        self.h = h
        self.n_dofs = 0
        self.n_groups = 0
        self.n_grav = 0
        self.n_mag = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.lf_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, st: int, what: str = ""):
        if st != 0:
            msg = self.lib.lf_last_error(self.h)
            raise LithoError(st, f"{what}: {msg.decode() if msg else ''}")

    @property
    def stream(self) -> int:
        return self.lib.lf_stream(self.h) or 0

    def set_model(self, model: Model) -> None:
        self._check(self.lib.lf_set_model(self.h, model.h), "set_model")
        self.n_dofs = model.n_dofs
        self.n_groups = model.info().n_groups

    def set_field(self, inclination: float, declination: float, field_nt: float, remanence_mode: int = 0):
        self._check(self.lib.lf_set_field(self.h, inclination, declination, field_nt, remanence_mode), "set_field")

    def set_gravity_data(self, xyz, obs=None, std=None):
        x = f64(xyz).reshape(-1, 3)
        o = f64(obs) if obs is not None else None
        s = f64(std) if std is not None else None
        self._check(self.lib.lf_set_gravity_data(self.h, len(x), _d(x), _d(o), _d(s)), "set_gravity_data")
        self.n_grav = len(x)

    def set_magnetic_data(self, xyz, obs=None, std=None):
        x = f64(xyz).reshape(-1, 3)
        o = f64(obs) if obs is not None else None
        s = f64(std) if std is not None else None
        self._check(self.lib.lf_set_magnetic_data(self.h, len(x), _d(x), _d(o), _d(s)), "set_magnetic_data")
        self.n_mag = len(x)

    def set_objective(self, alpha_mag: float = 1.0, ref_weight: float = 0.0, ref_params=None):
        rp = f64(ref_params) if ref_params is not None else None
        self._check(self.lib.lf_set_objective(self.h, alpha_mag, ref_weight, _d(rp)), "set_objective")

    def set_smoothness(self, weight: float, freedom=None):
        """SurfaceSmoothness regularisation (lf_set_smoothness); freedom per
        vertex, or None for the freedoms of the model given to set_model."""
        fr = None if freedom is None else np.ascontiguousarray(freedom, np.uint8)
        self._check(self.lib.lf_set_smoothness(self.h, float(weight), _u8(fr)), "set_smoothness")

    def tuning(self) -> Tuning:
        t = Tuning()
        self._check(self.lib.lf_get_tuning(self.h, C.byref(t)), "get_tuning")
        return t

    def set_tuning(self, fwd_target_blocks: int, grad_target_warps: int, near_tiles_per_chunk: int = 0,
                   patch_threads: Optional[int] = None, far_ratio: Optional[float] = None,
                   fwd_engine: Optional[int] = None):
        """lf_set_tuning; patch_threads / far_ratio / fwd_engine default to their
        current values."""
        cur = self.tuning()
        t = Tuning(fwd_target_blocks, grad_target_warps, near_tiles_per_chunk,
                   cur.patch_threads if patch_threads is None else patch_threads,
                   cur.far_ratio if far_ratio is None else far_ratio,
                   cur.fwd_engine if fwd_engine is None else fwd_engine)
        self._check(self.lib.lf_set_tuning(self.h, C.byref(t)), "set_tuning")

    def autotune(self, params, repeats: int = 3):
        """Times candidate launch shapes on this context's problem and keeps
        the fastest (lf_autotune); returns (Tuning, ms per evaluation)."""
        t = Tuning()
        ms = np.zeros(1)
        self._check(self.lib.lf_autotune(self.h, _d(f64(params)), repeats, C.byref(t), _d(ms)), "autotune")
        return t, float(ms[0])

    def set_station_groups(self, counts):
        """Batched bodies (lf_set_station_groups): counts[g] stations of group g;
        None turns batching off.  Set station data afterwards."""
        if counts is None:
            self._check(self.lib.lf_set_station_groups(self.h, 0, None), "set_station_groups")
            return
        c = i32(counts)
        self._check(self.lib.lf_set_station_groups(self.h, len(c), _i(c)), "set_station_groups")

    def group_objectives(self, n_groups: int) -> np.ndarray:
        out = np.zeros(n_groups)
        self._check(self.lib.lf_get_group_objectives(self.h, _d(out)), "group_objectives")
        return out

    def calibrate_data_weights(self, params, seed: int = 0):
        """lf_calibrate_data_weights: returns (alpha_mag, lambda_grav, lambda_mag)."""
        a, eg, em = np.zeros(1), np.zeros(1), np.zeros(1)
        self._check(self.lib.lf_calibrate_data_weights(self.h, _d(f64(params)), seed, _d(a), _d(eg), _d(em)),
                    "calibrate_data_weights")
        return float(a[0]), float(eg[0]), float(em[0])

    def property_inversion(self, params, density_range=(-1.0, 1.0), susceptibility_range=(0.0, 1.0),
                           remanence_range=(0.0, 100.0), remanence_component_range=(-100.0, 100.0),
                           damping=0.0, max_iterations=50, tolerance=1e-6, magnetic_per_group=1):
        """lf_property_inversion: returns (densities[G], magnetic[p G] or None);
        the context's group properties are updated as the reference updates
        its model."""
        o = _native.PropertyOptions(*density_range, *susceptibility_range, *remanence_range,
                                    *remanence_component_range, float(damping), int(max_iterations), float(tolerance))
        dens = np.zeros(self.n_groups)
        mag = np.zeros(magnetic_per_group * self.n_groups)
        self._check(self.lib.lf_property_inversion(self.h, _d(f64(params)), C.byref(o), _d(dens), _d(mag)),
                    "property_inversion")
        return dens, (mag if self.n_mag else None)

    def validate_model(self, params=None, overlap_baseline: int = 0, adjacent_overlap_baseline: int = 0,
                       freedom=None):
        """lf_validate_model: (passed, reason, worst violation)."""
        ok = C.c_int(0)
        worst = np.zeros(1)
        buf = C.create_string_buffer(256)
        fr = np.ascontiguousarray(freedom, np.uint8) if freedom is not None else None
        self._check(self.lib.lf_validate_model(self.h, _d(f64(params)) if params is not None else None,
                                               _u8(fr), int(overlap_baseline), int(adjacent_overlap_baseline),
                                               C.byref(ok), _d(worst), buf, len(buf)), "validate_model")
        return bool(ok.value), buf.value.decode(), float(worst[0])

    def smooth_gradient(self, grad, weight: float) -> np.ndarray:
        """lf_smooth_gradient: the runner's neighbour-blended gradient."""
        g = f64(grad)
        out = np.zeros(self.n_dofs)
        self._check(self.lib.lf_smooth_gradient(self.h, float(weight), _d(g), _d(out)), "smooth_gradient")
        return out

    # ---- point classification and borehole constraints ----
    def set_label_grid(self, labels, origin, spacing):
        """lf_set_label_grid: labels shaped (nz, ny, nx) of group ids (negative:
        ray casting decides); labels=None removes the grid."""
        if labels is None:
            self._check(self.lib.lf_set_label_grid(self.h, 0, 0, 0, 0.0, 0.0, 0.0, 1.0, 1.0, 1.0, None),
                        "set_label_grid")
            return
        lab = i32(labels)
        nz, ny, nx = lab.shape
        self._check(self.lib.lf_set_label_grid(self.h, nx, ny, nz, *map(float, origin), *map(float, spacing),
                                               _i(lab)), "set_label_grid")

    def set_bottom_depth(self, depth: float):
        self._check(self.lib.lf_set_bottom_depth(self.h, float(depth)), "set_bottom_depth")

    def classify_points(self, xyz, params=None) -> np.ndarray:
        """lf_classify_points: group id per point (-1 outside every mesh)."""
        x = f64(xyz).reshape(-1, 3)
        out = np.zeros(len(x), np.int32)
        self._check(self.lib.lf_classify_points(self.h, _d(f64(params)) if params is not None else None, len(x),
                                                _d(x), _i(out)), "classify_points")
        return out

    def set_constraints(self, xy, z_top, z_bottom, group, weight: float = 1e6):
        """lf_set_constraints: borehole intervals (depths positive down)."""
        xy = f64(xy).reshape(-1, 2)
        zt, zb, g = f64(z_top), f64(z_bottom), i32(group)
        self._check(self.lib.lf_set_constraints(self.h, len(xy), _d(xy), _d(zt), _d(zb), _i(g), float(weight)),
                    "set_constraints")

    def constraint_penalty(self, params) -> float:
        v = np.zeros(1)
        self._check(self.lib.lf_constraint_penalty(self.h, _d(f64(params)), _d(v)), "constraint_penalty")
        return float(v[0])

    def constraint_gradient(self, params) -> np.ndarray:
        g = np.zeros(self.n_dofs)
        self._check(self.lib.lf_constraint_gradient(self.h, _d(f64(params)), _d(g)), "constraint_gradient")
        return g

    def set_scatter_stateless(self, enabled: bool = True):
        """Every scatter from the model's given positions (lf_set_scatter_stateless)."""
        self._check(self.lib.lf_set_scatter_stateless(self.h, int(bool(enabled))), "set_scatter_stateless")

    def set_gradient_gather(self, mode: int):
        """GATHER_REFERENCE (the reference's DOF-vertex gather) or GATHER_CHAIN
        (the objective's exact derivative through the control-point
        interpolation and shared-vertex averaging); lf_set_gradient_gather."""
        self._check(self.lib.lf_set_gradient_gather(self.h, int(mode)), "set_gradient_gather")

    def set_xy_derivative(self, mode: int, step: float = 0.5):
        """XY_ANALYTIC, or XY_FORWARD_DIFFERENCE: x / y vertex derivatives of the
        objective gradient by per-facet forward differences with `step` metres
        (FP64), z analytic; lf_set_xy_derivative."""
        self._check(self.lib.lf_set_xy_derivative(self.h, int(mode), float(step)), "set_xy_derivative")

    def set_collapsed_facets(self, mode: int):
        """COLLAPSED_KEEP (the reference's forward) or COLLAPSED_DROP (facets
        collapsed onto a line contribute nothing); lf_set_collapsed_facets."""
        self._check(self.lib.lf_set_collapsed_facets(self.h, int(mode)), "set_collapsed_facets")

    def set_graph_mode(self, enabled: bool = True):
        """Replay evaluations as a captured CUDA graph (lf_set_graph_mode)."""
        self._check(self.lib.lf_set_graph_mode(self.h, int(bool(enabled))), "set_graph_mode")

    def set_precision(self, mode: int):
        self._check(self.lib.lf_set_precision(self.h, mode), "set_precision")

    def set_far_field_ratio(self, tau: float):
        self._check(self.lib.lf_set_far_field_ratio(self.h, tau), "set_far_field_ratio")

    def near_pairs(self) -> int:
        n = C.c_ulonglong(0)
        self._check(self.lib.lf_get_near_pairs(self.h, C.byref(n)), "near_pairs")
        return n.value

    def forward(self, params):
        p = f64(params)
        gz = np.zeros(self.n_grav)
        tmi = np.zeros(self.n_mag)
        self._check(self.lib.lf_forward(self.h, _d(p), _d(gz) if self.n_grav else None,
                                        _d(tmi) if self.n_mag else None), "forward")
        return gz, tmi

    def forward_gravity(self, params) -> np.ndarray:
        return self.forward(params)[0]

    def forward_magnetic(self, params) -> np.ndarray:
        return self.forward(params)[1]

    def objective_components(self, params) -> np.ndarray:
        p = f64(params)
        out = np.zeros(5)
        self._check(self.lib.lf_objective(self.h, _d(p), _d(out)), "objective")
        return out

    def objective(self, params) -> float:
        return float(self.objective_components(params)[4])

    def objective_and_gradient(self, params):
        p = f64(params)
        f = np.zeros(1)
        g = np.zeros(self.n_dofs)
        self._check(self.lib.lf_objective_grad(self.h, _d(p), _d(f), _d(g)), "objective_grad")
        return float(f[0]), g

    def jacobian(self, params, which: int = GRAVITY) -> np.ndarray:
        p = f64(params)
        n = self.n_grav if which == GRAVITY else self.n_mag
        J = np.zeros((n, self.n_dofs))
        self._check(self.lib.lf_jacobian(self.h, _d(p), which, _d(J)), "jacobian")
        return J

    def unit_response(self, params, kind: int, group: int, direction=None) -> np.ndarray:
        """Forward of one group alone with unit properties (lf_unit_response)."""
        p = f64(params)
        n = self.n_grav if kind == UNIT_GRAVITY else self.n_mag
        out = np.zeros(n)
        d = f64(direction) if direction is not None else None
        self._check(self.lib.lf_unit_response(self.h, _d(p), kind, group, _d(d), _d(out)), "unit_response")
        return out

    def positions(self, n_vertices: int) -> np.ndarray:
        out = np.zeros((n_vertices, 3))
        self._check(self.lib.lf_get_positions(self.h, _d(out)), "get_positions")
        return out

    def forward_device(self, d_params: int, d_gz: int = 0, d_tmi: int = 0):
        self._check(self.lib.lf_forward_device(self.h, d_params, d_gz or None, d_tmi or None), "forward_device")

    def objective_grad_device(self, d_params: int, d_f: int, d_grad: int):
        self._check(self.lib.lf_objective_grad_device(self.h, d_params, d_f, d_grad), "objective_grad_device")

    def lbfgsb(self, x0, lower, upper, max_iterations=500, tolerance=1e-6, history_size=10, armijo_c1=1e-4,
               line_search_max_iter=50, disable_line_search=False, initial_gamma=0.0, target_value=0.0):
        opt = LbfgsbOptions()
        self.lib.lf_lbfgsb_default_options(C.byref(opt))
        opt.max_iterations = max_iterations
        opt.tolerance = tolerance
        opt.history_size = history_size
        opt.armijo_c1 = armijo_c1
        opt.line_search_max_iter = line_search_max_iter
        opt.disable_line_search = int(disable_line_search)
        opt.initial_gamma = initial_gamma
        opt.target_value = target_value
        x0 = f64(x0)
        lo, hi = f64(lower), f64(upper)
        xo = np.zeros_like(x0)
        res = LbfgsbResult()
        self._check(self.lib.lf_lbfgsb_minimize(self.h, _d(x0), _d(lo), _d(hi), C.byref(opt), _d(xo),
                                                C.byref(res)), "lbfgsb")
        return xo, res

    def counters(self) -> Counters:
        c = Counters()
        self._check(self.lib.lf_get_counters(self.h, C.byref(c)))
        return c

    def set_profiling(self, enabled: bool):
        self._check(self.lib.lf_set_profiling(self.h, int(enabled)))

    def kernel_times(self):
        """(forward ms, forward launches, gradient ms, gradient launches)."""
        fm, gm = C.c_double(0), C.c_double(0)
        fn, gn = C.c_int(0), C.c_int(0)
        self._check(self.lib.lf_get_kernel_times(self.h, C.byref(fm), C.byref(fn), C.byref(gm), C.byref(gn)))
        return fm.value, fn.value, gm.value, gn.value

    def reset_counters(self):
        self._check(self.lib.lf_reset_counters(self.h))
