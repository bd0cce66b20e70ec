"""ctypes declarations for liblitho_gpu.so (include/litho_gpu.h)."""
from __future__ import annotations

import ctypes as C
import os

from .build import library_path

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)
_vp = C.c_void_p


class ModelInfo(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "n_groups", "n_vertices", "n_triangles", "n_dofs", "n_refs", "n_interp", "n_sync", "n_sync_entries")]


class LbfgsbOptions(C.Structure):
    _fields_ = [("max_iterations", C.c_int), ("tolerance", C.c_double), ("history_size", C.c_int),
                ("armijo_c1", C.c_double), ("line_search_max_iter", C.c_int),
                ("disable_line_search", C.c_int), ("initial_gamma", C.c_double), ("target_value", C.c_double)]


class LbfgsbResult(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("evaluations", C.c_int),
                ("gradients", C.c_int), ("final_value", C.c_double), ("message", C.c_char * 96)]


class Tuning(C.Structure):
    _fields_ = [("fwd_target_blocks", C.c_int), ("grad_target_warps", C.c_int), ("near_tiles_per_chunk", C.c_int),
                ("patch_threads", C.c_int), ("far_ratio", C.c_double), ("fwd_engine", C.c_int)]


class PropertyOptions(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "density_min", "density_max", "susceptibility_min", "susceptibility_max", "remanence_min",
        "remanence_max", "remanence_component_min", "remanence_component_max", "damping")] + [
        ("max_iterations", C.c_int), ("tolerance", C.c_double)]


class Counters(C.Structure):
    _fields_ = [("forward_pairs", C.c_uint64), ("gradient_pairs", C.c_uint64), ("launches", C.c_uint64)]


# name -> (restype, argtypes)
SIGNATURES = {
    "lf_model_create": (C.c_int, [C.POINTER(_vp)]),
    "lf_model_destroy": (None, [_vp]),
    "lf_model_add_group": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                     C.c_double, _dp, C.POINTER(C.c_int)]),
    "lf_model_set_group_mesh": (C.c_int, [_vp, C.c_int, C.c_int, _dp, _u8p, C.c_int, _ip]),
    "lf_model_set_axis_scale": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double]),
    "lf_model_set_depth_bounds": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double]),
    "lf_model_set_interior_grid": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int]),
    "lf_model_set_control_point_stride": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int)]),
    "lf_model_set_mesh_control_point_stride": (C.c_int, [_vp, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "lf_model_build_shared_vertex_sync": (C.c_int, [_vp]),
    "lf_model_apply_model_bounds": (C.c_int, [_vp, C.c_double]),
    "lf_model_get_info": (C.c_int, [_vp, C.POINTER(ModelInfo)]),
    "lf_model_assemble_parameters": (C.c_int, [_vp, _dp]),
    "lf_model_get_bounds": (C.c_int, [_vp, _dp, _dp]),
    "lf_model_apply_parameters": (C.c_int, [_vp, _dp]),
    "lf_model_get_positions": (C.c_int, [_vp, _dp]),
    "lf_model_export_tables": (C.c_int, [_vp, _dp, _ip, _ip, _ip, _ip, _u8p, _dp, _ip, _ip, _dp, _ip, _ip]),
    "lf_create": (C.c_int, [C.POINTER(_vp), C.c_int]),
    "lf_destroy": (None, [_vp]),
    "lf_last_error": (C.c_char_p, [_vp]),
    "lf_stream": (_vp, [_vp]),
    "lf_set_model": (C.c_int, [_vp, _vp]),
    "lf_set_model_tables": (C.c_int, [_vp, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int, _dp, C.c_int, _ip,
                                      _ip, C.c_int, _ip, _ip, _u8p, _dp, _ip, _ip, _dp, C.c_int, _ip, _ip]),
    "lf_set_field": (C.c_int, [_vp, C.c_double, C.c_double, C.c_double, C.c_int]),
    "lf_set_gravity_data": (C.c_int, [_vp, C.c_int, _dp, _dp, _dp]),
    "lf_set_magnetic_data": (C.c_int, [_vp, C.c_int, _dp, _dp, _dp]),
    "lf_set_objective": (C.c_int, [_vp, C.c_double, C.c_double, _dp]),
    "lf_set_precision": (C.c_int, [_vp, C.c_int]),
    "lf_set_far_field_ratio": (C.c_int, [_vp, C.c_double]),
    "lf_get_near_pairs": (C.c_int, [_vp, C.POINTER(C.c_ulonglong)]),
    "lf_forward": (C.c_int, [_vp, _dp, _dp, _dp]),
    "lf_objective": (C.c_int, [_vp, _dp, _dp]),
    "lf_objective_grad": (C.c_int, [_vp, _dp, _dp, _dp]),
    "lf_jacobian": (C.c_int, [_vp, _dp, C.c_int, _dp]),
    "lf_unit_response": (C.c_int, [_vp, _dp, C.c_int, C.c_int, _dp, _dp]),
    "lf_set_graph_mode": (C.c_int, [_vp, C.c_int]),
    "lf_set_scatter_stateless": (C.c_int, [_vp, C.c_int]),
    "lf_set_gradient_gather": (C.c_int, [_vp, C.c_int]),
    "lf_set_xy_derivative": (C.c_int, [_vp, C.c_int, C.c_double]),
    "lf_set_collapsed_facets": (C.c_int, [_vp, C.c_int]),
    "lf_calibrate_data_weights": (C.c_int, [_vp, _dp, C.c_uint, _dp, _dp, _dp]),
    "lf_mlp_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint, C.POINTER(_vp)]),
    "lf_mlp_destroy": (None, [_vp]),
    "lf_mlp_last_error": (C.c_char_p, [_vp]),
    "lf_mlp_train_step": (C.c_int, [_vp, C.c_void_p, C.c_void_p, C.c_float, C.POINTER(C.c_float)]),
    "lf_mlp_predict": (C.c_int, [_vp, C.c_void_p, C.c_int, C.c_void_p]),
    "lf_mlp_param_count": (C.c_int, [_vp, C.POINTER(C.c_size_t)]),
    "lf_mlp_get_params": (C.c_int, [_vp, C.c_void_p]),
    "lf_mlp_set_params": (C.c_int, [_vp, C.c_void_p]),
    "lf_mlp_gradients": (C.c_int, [_vp, C.c_void_p, C.c_void_p, C.POINTER(C.c_float), C.c_void_p]),
    "lf_set_station_groups": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int32)]),
    "lf_get_group_objectives": (C.c_int, [_vp, _dp]),
    "lf_set_tuning": (C.c_int, [_vp, C.c_void_p]),
    "lf_get_tuning": (C.c_int, [_vp, C.c_void_p]),
    "lf_autotune": (C.c_int, [_vp, _dp, C.c_int, C.c_void_p, _dp]),
    "lf_set_smoothness": (C.c_int, [_vp, C.c_double, C.POINTER(C.c_uint8)]),
    "lf_get_positions": (C.c_int, [_vp, _dp]),
    "lf_forward_device": (C.c_int, [_vp, _vp, _vp, _vp]),
    "lf_objective_grad_device": (C.c_int, [_vp, _vp, _vp, _vp]),
    "lf_lbfgsb_default_options": (None, [C.POINTER(LbfgsbOptions)]),
    "lf_lbfgsb_minimize": (C.c_int, [_vp, _dp, _dp, _dp, C.POINTER(LbfgsbOptions), _dp, C.POINTER(LbfgsbResult)]),
    "lf_get_counters": (C.c_int, [_vp, C.POINTER(Counters)]),
    "lf_reset_counters": (C.c_int, [_vp]),
    "lf_set_profiling": (C.c_int, [_vp, C.c_int]),
    "lf_forward_noalloc": (C.c_int, [C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, C.c_double, C.c_double, C.c_double,
                                     C.c_double, C.c_double, _vp, _vp, _vp]),
    "lf_get_kernel_times": (C.c_int, [_vp, _dp, C.POINTER(C.c_int), _dp, C.POINTER(C.c_int)]),
    "lf_read_surface": (C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp, _ip]),
    "lf_write_tsurf": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, _dp, C.c_int, _ip]),
    "lf_validate_model": (C.c_int, [_vp, _dp, _u8p, C.c_ulonglong, C.c_ulonglong, C.POINTER(C.c_int), _dp,
                                    C.c_char_p, C.c_int]),
    "lf_smooth_gradient": (C.c_int, [_vp, C.c_double, _dp, _dp]),
    "lf_smooth_gradient_device": (C.c_int, [_vp, C.c_double, _vp, _vp]),
    "lf_mlp_set_engine": (C.c_int, [_vp, C.c_int]),
    "lf_gemm_bf16": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _vp, C.c_int, _vp,
                               C.c_int, _vp, _vp, C.c_int, _vp]),
    "lf_set_device_wait_limit": (C.c_int, [C.c_longlong]),
    "lf_facet_patches": (C.c_int, [C.c_int, _dp, C.c_int, _ip, C.c_int, _ip, C.POINTER(C.c_int), _ip, _ip, _ip]),
    "lf_property_inversion": (C.c_int, [_vp, _dp, C.c_void_p, _dp, _dp]),
    "lf_set_label_grid": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_double, _ip]),
    "lf_set_bottom_depth": (C.c_int, [_vp, C.c_double]),
    "lf_classify_points": (C.c_int, [_vp, _dp, C.c_int, _dp, _ip]),
    "lf_set_constraints": (C.c_int, [_vp, C.c_int, _dp, _dp, _dp, _ip, C.c_double]),
    "lf_constraint_penalty": (C.c_int, [_vp, _dp, _dp]),
    "lf_constraint_gradient": (C.c_int, [_vp, _dp, _dp]),
}

STATUS = {0: "LF_OK", 1: "LF_EINVAL", 2: "LF_ECUDA", 3: "LF_ENOMEM", 4: "LF_ESTATE", 5: "LF_ETIMEOUT",
          6: "LF_ENUMERIC"}

_LIB = None


def load(path: str | None = None) -> C.CDLL:
    """Loads liblitho_gpu.so (building it with nvcc if it is missing).

    Raises if the library cannot be built or loaded: there is no fallback
    implementation of the hot path."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or library_path()
    if not os.path.exists(p):
        from .build import build_library
        p = build_library()
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = lib
    return lib
