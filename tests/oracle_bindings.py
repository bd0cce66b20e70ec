"""ctypes access to the test-only checkers under oracle/:

* liboracle.so          -- the C restatement of the reference path (always built)
* _ref/libref_litho.so  -- the reference's own sources compiled here (only
                           where the reference tree exists; tests that need
                           it skip otherwise)

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")
REF_SO = os.path.join(ORACLE_DIR, "_ref", "libref_litho.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)


def _d(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_dp)


def build_oracle() -> None:
    src = os.path.join(ORACLE_DIR, "litho_oracle.c")
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-C", ORACLE_DIR, "liboracle.so"], check=True, capture_output=True)


_ORACLE = None


def oracle() -> C.CDLL:
    global _ORACLE
    if _ORACLE is None:
        build_oracle()
        lib = C.CDLL(ORACLE_SO)
        lib.lo_solid_angle.restype = C.c_double
        lib.lo_solid_angle.argtypes = [_dp, _dp, _dp, _dp]
        lib.lo_line_integral_term.restype = C.c_double
        lib.lo_line_integral_term.argtypes = [_dp, _dp, _dp]
        lib.lo_face_nagy.restype = C.c_double
        lib.lo_face_nagy.argtypes = [_dp, _dp, _dp, _dp]
        lib.lo_magnetic_facet.restype = C.c_double
        lib.lo_magnetic_facet.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp]
        lib.lo_face_fd_gradient.restype = C.c_double
        lib.lo_face_fd_gradient.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        lib.lo_face_true_gradient.restype = None
        lib.lo_face_true_gradient.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double, _dp]
        lib.lo_field_unit_vector.restype = None
        lib.lo_field_unit_vector.argtypes = [C.c_double, C.c_double, _dp]
        lib.lo_group_magnetization.restype = None
        lib.lo_group_magnetization.argtypes = [C.c_double, C.c_double, _dp, C.c_int, C.c_double, C.c_double,
                                               C.c_double, _dp, _dp, _dp]
        lib.lo_scatter.restype = None
        lib.lo_scatter.argtypes = [C.c_int, _dp, _ip, _ip, _u8p, _dp, C.c_int, _ip, _ip, _dp, C.c_int, _ip, _ip, _dp]
        lib.lo_forward_gz.restype = None
        lib.lo_forward_gz.argtypes = [C.c_int, _dp, C.c_int, _ip, _ip, _dp, _dp, _dp]
        lib.lo_forward_tmi.restype = None
        lib.lo_forward_tmi.argtypes = [C.c_int, _dp, C.c_int, _ip, _ip, _dp, _dp, _dp, _dp, _dp]
        lib.lo_jacobian.restype = None
        lib.lo_jacobian.argtypes = [C.c_int, C.c_int, _dp, C.c_int, _ip, _ip, C.c_int, _dp, _dp, _dp, _dp, _dp,
                                    C.c_int, _ip, _ip, _u8p, _dp, C.c_double, _dp]
        lib.lo_chain_gather.restype = None
        lib.lo_chain_gather.argtypes = [C.c_int, _dp, C.c_int, _ip, _ip, _u8p, _dp, _ip, _ip, _dp, C.c_int, _ip, _ip,
                                        _dp]
        lib.lo_misfit.restype = C.c_double
        lib.lo_misfit.argtypes = [C.c_int, _dp, _dp, _dp]
        lib.lo_misfit_gradient.restype = None
        lib.lo_misfit_gradient.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp, C.c_double, _dp]
        lib.lo_smoothness.restype = None
        lib.lo_smoothness.argtypes = [C.c_int, _dp, _u8p, C.c_int, _ip, C.c_double, C.c_int, _ip, _ip, _u8p, _dp,
                                      _dp, _dp]
        _ORACLE = lib
    return _ORACLE


def ref_available() -> bool:
    return os.path.exists(REF_SO)


_REF = None


def ref() -> C.CDLL:
    global _REF
    if _REF is None:
        lib = C.CDLL(REF_SO)
        V = C.c_void_p
        sig = {
            "ref_new": (V, []), "ref_free": (None, [V]),
            "ref_add_group": (C.c_int, [V, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, _dp]),
            "ref_set_mesh": (C.c_int, [V, C.c_int, C.c_int, _dp, _u8p, C.c_int, _ip, _dp, C.c_double, C.c_double]),
            "ref_set_control_point_stride": (C.c_int, [V, C.c_int]),
            "ref_build_shared_sync": (None, [V]),
            "ref_apply_model_bounds": (None, [V, C.c_double]),
            "ref_dof_count": (C.c_int, [V]), "ref_vertex_count": (C.c_int, [V]),
            "ref_dof_tables": (C.c_int, [V, _ip, _ip, _u8p, _dp]),
            "ref_is_control_point": (None, [V, _u8p]),
            "ref_assemble": (None, [V, _dp]), "ref_bounds": (None, [V, _dp, _dp]),
            "ref_apply": (None, [V, _dp]), "ref_positions": (None, [V, _dp]),
            "ref_set_gravity": (None, [V, C.c_int, _dp, _dp, _dp]),
            "ref_set_magnetic": (None, [V, C.c_int, _dp, _dp, _dp, C.c_double, C.c_double, C.c_double, C.c_int]),
            "ref_set_objective": (None, [V, C.c_double, C.c_double, _dp]),
            "ref_group_magnetization": (None, [V, C.c_int, _dp, _dp]),
            "ref_forward_gz": (None, [V, _dp, _dp]), "ref_forward_tmi": (None, [V, _dp, _dp]),
            "ref_jacobian_gz": (None, [V, _dp, _dp]), "ref_jacobian_tmi": (None, [V, _dp, _dp]),
            "ref_unit_response": (None, [V, _dp, C.c_int, C.c_int, _dp, _dp]),
            "ref_set_smoothness": (None, [V, C.c_double]),
            "ref_calibrate": (C.c_double, [V, _dp]),
            "ref_smoothness_value": (C.c_double, [V, _dp]),
            "ref_smoothness_gradient": (None, [V, _dp, _dp]),
            "ref_objective": (None, [V, _dp, _dp]), "ref_gradient": (None, [V, _dp, _dp]),
            "ref_lbfgsb": (C.c_int, [V, _dp, _dp, _dp, C.c_int, C.c_double, C.c_int, _dp, _dp]),
            "ref_load_surface": (C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp, _ip]),
            "ref_export_ts": (None, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, _dp, C.c_int, _ip]),
            "ref_validate": (C.c_int, [V, C.c_ulonglong, C.c_ulonglong, _dp, C.c_char_p, C.c_int]),
            "ref_smooth_gradient": (None, [V, C.c_double, _dp, _dp]),
            "ref_property_inversion": (None, [V, _dp, _dp, C.c_int, _dp, _dp]),
            "ref_set_label_grid": (None, [V, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                          C.c_double, C.c_double, C.c_double, _ip]),
            "ref_set_bottom_depth": (None, [V, C.c_double]),
            "ref_classify": (None, [V, C.c_int, _dp, _ip]),
            "ref_set_constraints": (None, [V, C.c_int, _dp, _dp, _dp, _ip, C.c_double]),
            "ref_constraint_value": (C.c_double, [V, _dp]),
            "ref_constraint_gradient": (None, [V, _dp, _dp]),
            "ref_use_gpu": (C.c_int, [V, C.c_char_p, C.c_int, C.c_int, _ip, _ip, _dp, C.c_int, _ip, _ip]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _REF = lib
    return _REF


class RefModel:
    """The reference's LithologyModel + forwards + objective built from a
    synth.Problem (test harness over oracle/_ref)."""

    def __init__(self, problem, grav_obs=None, grav_std=None, mag_obs=None, mag_std=None, alpha_mag=1.0,
                 ref_weight=0.0, ref_params=None, remanence_mode=0, smooth_weight=0.0):
        self.lib = ref()
        self.h = self.lib.ref_new()
        for g, (rho, chi) in enumerate(zip(problem.densities, problem.susceptibilities)):
            idx = self.lib.ref_add_group(self.h, g, rho, chi, 0.0, 0.0, 0.0, None)
            assert idx == g
        scale = np.full(3, problem.axis_scale)
        lo, hi = (problem.depth_bounds if problem.depth_bounds is not None else (-10000.0, 0.0))
        for g, (V, F, fr) in enumerate(problem.meshes):
            V = np.ascontiguousarray(V, np.float64)
            F = np.ascontiguousarray(F, np.int32)
            fr = np.ascontiguousarray(np.broadcast_to(np.asarray(fr, np.uint8), (len(V),)))
            self.lib.ref_set_mesh(self.h, g, len(V), _d(V), fr.ctypes.data_as(_u8p), len(F),
                                  F.ctypes.data_as(_ip), _d(scale), lo, hi)
        if problem.cp_stride > 0:
            self.lib.ref_set_control_point_stride(self.h, problem.cp_stride)
        if len(problem.meshes) > 1:
            self.lib.ref_build_shared_sync(self.h)
        Sg = len(problem.grav_xyz)
        self.lib.ref_set_gravity(self.h, Sg, _d(problem.grav_xyz), _d(grav_obs), _d(grav_std))
        if problem.mag_xyz is not None:
            inc, dec, F0 = problem.inducing
            self.lib.ref_set_magnetic(self.h, len(problem.mag_xyz), _d(problem.mag_xyz), _d(mag_obs), _d(mag_std),
                                      inc, dec, F0, remanence_mode)
        self.lib.ref_set_objective(self.h, alpha_mag, ref_weight, _d(ref_params))
        self.lib.ref_set_smoothness(self.h, smooth_weight)
        self.np = self.lib.ref_dof_count(self.h)
        self.nv = self.lib.ref_vertex_count(self.h)
        self.Sg = Sg
        self.Sm = 0 if problem.mag_xyz is None else len(problem.mag_xyz)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_free(self.h)
            self.h = None

    def assemble(self):
        p = np.zeros(self.np)
        self.lib.ref_assemble(self.h, _d(p) if False else p.ctypes.data_as(_dp))
        return p

    def bounds(self):
        lo, hi = np.zeros(self.np), np.zeros(self.np)
        self.lib.ref_bounds(self.h, lo.ctypes.data_as(_dp), hi.ctypes.data_as(_dp))
        return lo, hi

    def apply(self, params):
        self.lib.ref_apply(self.h, _d(params))

    def positions(self):
        out = np.zeros((self.nv, 3))
        self.lib.ref_positions(self.h, out.ctypes.data_as(_dp))
        return out

    def dof_tables(self):
        nref_cap = 3 * self.nv + 8
        off = np.zeros(self.np + 1, np.int32)
        rv = np.zeros(nref_cap, np.int32)
        ra = np.zeros(nref_cap, np.uint8)
        rs = np.zeros(nref_cap)
        n = self.lib.ref_dof_tables(self.h, off.ctypes.data_as(_ip), rv.ctypes.data_as(_ip),
                                    ra.ctypes.data_as(_u8p), rs.ctypes.data_as(_dp))
        return off, rv[:n], ra[:n], rs[:n]

    def is_control_point(self):
        out = np.zeros(self.nv, np.uint8)
        self.lib.ref_is_control_point(self.h, out.ctypes.data_as(_u8p))
        return out

    def forward_gz(self, params):
        out = np.zeros(self.Sg)
        self.lib.ref_forward_gz(self.h, _d(params), out.ctypes.data_as(_dp))
        return out

    def forward_tmi(self, params):
        out = np.zeros(self.Sm)
        self.lib.ref_forward_tmi(self.h, _d(params), out.ctypes.data_as(_dp))
        return out

    def calibrate(self, params):
        """JointObjective::calibrateDataWeights; returns the new alpha_mag."""
        return float(self.lib.ref_calibrate(self.h, _d(params)))

    def smoothness(self, params):
        """SurfaceSmoothness value and DOF gradient at params."""
        g = np.zeros(self.np)
        v = self.lib.ref_smoothness_value(self.h, _d(params))
        self.lib.ref_smoothness_gradient(self.h, _d(params), g.ctypes.data_as(_dp))
        return v, g

    def validate(self, overlap_baseline=0, adjacent_baseline=0):
        """LithologyModel::validate at the current positions: (passed, reason, worst)."""
        worst = np.zeros(1)
        buf = C.create_string_buffer(256)
        ok = self.lib.ref_validate(self.h, int(overlap_baseline), int(adjacent_baseline),
                                   worst.ctypes.data_as(_dp), buf, len(buf))
        return bool(ok), buf.value.decode(), float(worst[0])

    def smooth_gradient(self, grad, weight):
        """InversionRunner::smoothGradient restated with the reference model."""
        g = np.ascontiguousarray(grad, np.float64)
        out = np.zeros(self.np)
        self.lib.ref_smooth_gradient(self.h, float(weight), _d(g), out.ctypes.data_as(_dp))
        return out

    def property_inversion(self, params, opt, max_iter, n_groups, magnetic_per_group):
        """runPropertyInversion parts A and B (restated with the reference's
        classes): (densities, magnetic parameters)."""
        o = np.ascontiguousarray(opt, np.float64)
        dens = np.zeros(n_groups)
        mag = np.zeros(magnetic_per_group * n_groups)
        self.lib.ref_property_inversion(self.h, _d(params), _d(o), int(max_iter), dens.ctypes.data_as(_dp),
                                        mag.ctypes.data_as(_dp))
        return dens, mag

    def set_label_grid(self, labels, origin, spacing):
        lab = np.ascontiguousarray(labels, np.int32)
        nz, ny, nx = lab.shape
        self.lib.ref_set_label_grid(self.h, nx, ny, nz, *map(float, origin), *map(float, spacing),
                                    lab.ctypes.data_as(_ip))

    def set_bottom_depth(self, depth):
        self.lib.ref_set_bottom_depth(self.h, float(depth))

    def classify(self, xyz):
        """classifyPoint for each row of xyz at the current positions."""
        x = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        out = np.zeros(len(x), np.int32)
        self.lib.ref_classify(self.h, len(x), _d(x), out.ctypes.data_as(_ip))
        return out

    def set_constraints(self, xy, z_top, z_bottom, group, weight=1e6):
        xy = np.ascontiguousarray(xy, np.float64).reshape(-1, 2)
        zt, zb = np.ascontiguousarray(z_top, np.float64), np.ascontiguousarray(z_bottom, np.float64)
        g = np.ascontiguousarray(group, np.int32)
        self.lib.ref_set_constraints(self.h, len(xy), _d(xy), _d(zt), _d(zb), g.ctypes.data_as(_ip), float(weight))

    def constraint_value(self, params):
        return self.lib.ref_constraint_value(self.h, _d(params))

    def constraint_gradient(self, params):
        g = np.zeros(self.np)
        self.lib.ref_constraint_gradient(self.h, _d(params), g.ctypes.data_as(_dp))
        return g

    def unit_response(self, params, kind, group, direction=None):
        out = np.zeros(self.Sg if kind == 0 else self.Sm)
        d = np.ascontiguousarray(direction, np.float64) if direction is not None else np.zeros(3)
        self.lib.ref_unit_response(self.h, _d(params), kind, group, d.ctypes.data_as(_dp), out.ctypes.data_as(_dp))
        return out

    def jacobian_gz(self, params):
        J = np.zeros((self.Sg, self.np))
        self.lib.ref_jacobian_gz(self.h, _d(params), J.ctypes.data_as(_dp))
        return J

    def jacobian_tmi(self, params):
        J = np.zeros((self.Sm, self.np))
        self.lib.ref_jacobian_tmi(self.h, _d(params), J.ctypes.data_as(_dp))
        return J

    def objective(self, params):
        out = np.zeros(5)
        self.lib.ref_objective(self.h, _d(params), out.ctypes.data_as(_dp))
        return out

    def gradient(self, params):
        g = np.zeros(self.np)
        self.lib.ref_gradient(self.h, _d(params), g.ctypes.data_as(_dp))
        return g

    def group_magnetization(self, g):
        amp = np.zeros(1)
        d = np.zeros(3)
        self.lib.ref_group_magnetization(self.h, g, amp.ctypes.data_as(_dp), d.ctypes.data_as(_dp))
        return float(amp[0]), d

    def use_gpu(self, lib_path, device=0, precision=0, tables=None):
        """Runs this model's objective on the GPU drop-in operators
        (oracle/gpu_dropin.hpp) over liblitho_gpu.so at lib_path.  `tables`
        (the library builder's tables) supplies the control-point and
        shared-vertex rows the reference keeps private; None for models
        without them.  Call after the data are set."""
        io = isrc = iw = so = sv = None
        ns = 0
        if tables is not None:
            self._keep = [np.ascontiguousarray(tables[k]) for k in
                          ("interp_off", "interp_src", "interp_w", "sync_off", "sync_vertex")]
            io, isrc, iw, so, sv = self._keep
            ns = len(so) - 1
            io, isrc, so, sv = (a.ctypes.data_as(_ip) for a in (io, isrc, so, sv))
            iw = iw.ctypes.data_as(_dp)
        st = self.lib.ref_use_gpu(self.h, str(lib_path).encode(), device, precision, io, isrc, iw, ns, so, sv)
        if st != 0:
            raise RuntimeError(f"ref_use_gpu failed: {st}")

    def lbfgsb(self, x0, lo, hi, max_iter=30, ftol=1e-6, history=10):
        x = np.zeros(self.np)
        f = np.zeros(1)
        it = self.lib.ref_lbfgsb(self.h, _d(x0), _d(lo), _d(hi), max_iter, ftol, history,
                                 x.ctypes.data_as(_dp), f.ctypes.data_as(_dp))
        return x, float(f[0]), it


class OracleModel:
    """Flat-table view of a model evaluated by the C restatement."""

    def __init__(self, tables: dict, densities, susceptibilities, inducing=(60.0, 0.0, 55000.0), remanence=None):
        self.o = oracle()
        self.t = {k: np.ascontiguousarray(v) for k, v in tables.items()}
        self.pos = np.ascontiguousarray(self.t["pos"], np.float64).copy()
        self.G = len(densities)
        self.rho = np.ascontiguousarray(densities, np.float64)
        inc, dec, F0 = inducing
        self.fdir = np.zeros(3)
        self.o.lo_field_unit_vector(inc, dec, self.fdir.ctypes.data_as(_dp))
        self.amp = np.zeros(self.G)
        self.mdir = np.zeros((self.G, 3))
        for g in range(self.G):
            a = np.zeros(1)
            d = np.zeros(3)
            self.o.lo_group_magnetization(susceptibilities[g], F0, _d(self.fdir), 0, 0.0, 0.0, 0.0, None,
                                          a.ctypes.data_as(_dp), d.ctypes.data_as(_dp))
            self.amp[g] = a[0]
            self.mdir[g] = d
        self.np = len(self.t["dof_off"]) - 1

    def _ip(self, k):
        return self.t[k].ctypes.data_as(_ip)

    def scatter(self, params):
        t = self.t
        ns = len(t["sync_off"]) - 1
        self.o.lo_scatter(self.np, _d(params), self._ip("dof_off"), self._ip("ref_vertex"),
                          t["ref_axis"].ctypes.data_as(_u8p), t["ref_scale"].ctypes.data_as(_dp), len(self.pos),
                          self._ip("interp_off"), self._ip("interp_src"), t["interp_w"].ctypes.data_as(_dp), ns,
                          self._ip("sync_off"), self._ip("sync_vertex"), self.pos.ctypes.data_as(_dp))

    def forward_gz(self, sta):
        sta = np.ascontiguousarray(sta, np.float64)
        out = np.zeros(len(sta))
        self.o.lo_forward_gz(len(sta), sta.ctypes.data_as(_dp), self.G, self._ip("grp_tri_off"), self._ip("tri"),
                             self.pos.ctypes.data_as(_dp), self.rho.ctypes.data_as(_dp), out.ctypes.data_as(_dp))
        return out

    def forward_tmi(self, sta):
        sta = np.ascontiguousarray(sta, np.float64)
        out = np.zeros(len(sta))
        self.o.lo_forward_tmi(len(sta), sta.ctypes.data_as(_dp), self.G, self._ip("grp_tri_off"), self._ip("tri"),
                              self.pos.ctypes.data_as(_dp), self.amp.ctypes.data_as(_dp),
                              self.mdir.ctypes.data_as(_dp), self.fdir.ctypes.data_as(_dp), out.ctypes.data_as(_dp))
        return out

    def smoothness(self, freedom, weight):
        """SurfaceSmoothness value and DOF gradient at the current positions
        (freedom: VertexFreedom code per global vertex)."""
        t = self.t
        fr = np.ascontiguousarray(freedom, np.uint8)
        V = self.pos.size // 3
        T = t["tri"].size // 3
        g = np.zeros(self.np)
        val = np.zeros(1)
        self.o.lo_smoothness(V, self.pos.ctypes.data_as(_dp), fr.ctypes.data_as(_u8p), T, self._ip("tri"), weight,
                             self.np, self._ip("dof_off"), self._ip("ref_vertex"),
                             t["ref_axis"].ctypes.data_as(_u8p), t["ref_scale"].ctypes.data_as(_dp),
                             val.ctypes.data_as(_dp), g.ctypes.data_as(_dp))
        return float(val[0]), g

    def forward_unit(self, sta, kind, group, direction=None, field_nt=55000.0):
        """Group `group` alone with a unit property: kind 0 density (gz), 1
        susceptibility under the inducing field, 2 magnetisation along
        `direction`, 3 the same for a remanence direction (TMI)."""
        sta = np.ascontiguousarray(sta, np.float64)
        out = np.zeros(len(sta))
        if kind == 0:
            rho = np.zeros(self.G)
            rho[group] = 1.0
            self.o.lo_forward_gz(len(sta), sta.ctypes.data_as(_dp), self.G, self._ip("grp_tri_off"),
                                 self._ip("tri"), self.pos.ctypes.data_as(_dp), rho.ctypes.data_as(_dp),
                                 out.ctypes.data_as(_dp))
            return out
        amp = np.zeros(self.G)
        mdir = np.ascontiguousarray(np.tile(self.fdir, (self.G, 1)))
        if kind == 1:
            amp[group] = field_nt / 100.0
        else:
            amp[group] = 1.0
            mdir[group] = direction
        self.o.lo_forward_tmi(len(sta), sta.ctypes.data_as(_dp), self.G, self._ip("grp_tri_off"), self._ip("tri"),
                              self.pos.ctypes.data_as(_dp), amp.ctypes.data_as(_dp), mdir.ctypes.data_as(_dp),
                              self.fdir.ctypes.data_as(_dp), out.ctypes.data_as(_dp))
        return out

    def jacobian(self, sta, kind, true_h=1e-2):
        """kind: 0 gravity FD (reference), 1 magnetic FD, 2 gravity true, 3 magnetic true."""
        sta = np.ascontiguousarray(sta, np.float64)
        J = np.zeros((len(sta), self.np))
        t = self.t
        self.o.lo_jacobian(kind, len(sta), sta.ctypes.data_as(_dp), self.G, self._ip("grp_tri_off"),
                           self._ip("tri"), len(self.pos), self.pos.ctypes.data_as(_dp),
                           self.rho.ctypes.data_as(_dp), self.amp.ctypes.data_as(_dp), self.mdir.ctypes.data_as(_dp),
                           self.fdir.ctypes.data_as(_dp), self.np, self._ip("dof_off"), self._ip("ref_vertex"),
                           t["ref_axis"].ctypes.data_as(_u8p), t["ref_scale"].ctypes.data_as(_dp), true_h,
                           J.ctypes.data_as(_dp))
        return J

    def vertex_jacobian(self, sta, kind, true_h=-3e-3):
        """Jacobian with respect to every vertex coordinate, columns 3 v + axis
        (kind 2 gravity / 3 magnetic true derivative, 0 / 1 the reference's
        per-facet forward differences)."""
        sta = np.ascontiguousarray(sta, np.float64)
        V = self.pos.size // 3
        dof_off = np.arange(3 * V + 1, dtype=np.int32)
        ref_vertex = np.repeat(np.arange(V, dtype=np.int32), 3)
        ref_axis = np.tile(np.arange(3, dtype=np.uint8), V)
        ref_scale = np.ones(3 * V)
        J = np.zeros((len(sta), 3 * V))
        t = self.t
        self.o.lo_jacobian(kind, len(sta), sta.ctypes.data_as(_dp), self.G, self._ip("grp_tri_off"),
                           self._ip("tri"), V, self.pos.ctypes.data_as(_dp), self.rho.ctypes.data_as(_dp),
                           self.amp.ctypes.data_as(_dp), self.mdir.ctypes.data_as(_dp),
                           self.fdir.ctypes.data_as(_dp), 3 * V, dof_off.ctypes.data_as(_ip),
                           ref_vertex.ctypes.data_as(_ip), ref_axis.ctypes.data_as(_u8p), _d(ref_scale), true_h,
                           J.ctypes.data_as(_dp))
        return J

    def chain_gather(self, vg):
        """Gradient with respect to the parameters from one with respect to the
        scattered positions (vg[3V]): lo_chain_gather, the adjoint of scatter."""
        t = self.t
        vg = np.array(vg, np.float64).ravel().copy()
        out = np.zeros(self.np)
        self.o.lo_chain_gather(len(self.pos), vg.ctypes.data_as(_dp), self.np, self._ip("dof_off"),
                               self._ip("ref_vertex"), t["ref_axis"].ctypes.data_as(_u8p),
                               t["ref_scale"].ctypes.data_as(_dp), self._ip("interp_off"), self._ip("interp_src"),
                               t["interp_w"].ctypes.data_as(_dp), len(t["sync_off"]) - 1, self._ip("sync_off"),
                               self._ip("sync_vertex"), out.ctypes.data_as(_dp))
        return out

    def chain_jacobian(self, sta, kind, true_h=-3e-3):
        """Derivative of the forward at the scattered positions with respect to
        the parameters through the whole scatter (DOF writes, control-point
        interpolation, shared-vertex averaging)."""
        Jv = self.vertex_jacobian(sta, kind, true_h)
        return np.stack([self.chain_gather(row) for row in Jv]) if len(Jv) else np.zeros((0, self.np))


def misfit(pred, obs, std):
    w = np.where(std > 0, 1.0 / np.where(std > 0, std, 1.0), 1.0)
    return 0.5 * np.sum((w * (obs - pred)) ** 2)


def misfit_gradient(J, pred, obs, std, alpha=1.0):
    w = np.where(std > 0, 1.0 / np.where(std > 0, std, 1.0), 1.0)
    return -alpha * J.T @ (w * w * (obs - pred))


def ref_load_surface(path):
    """The reference's loadSurfaceMesh: (xyz [n, 3], tri [m, 3]) or None."""
    lib = ref()
    nv, nt = C.c_int(0), C.c_int(0)
    if not lib.ref_load_surface(str(path).encode(), C.byref(nv), C.byref(nt), None, None):
        return None
    xyz = np.zeros((nv.value, 3))
    tri = np.zeros((nt.value, 3), np.int32)
    lib.ref_load_surface(str(path).encode(), C.byref(nv), C.byref(nt), xyz.ctypes.data_as(_dp),
                         tri.ctypes.data_as(_ip))
    return xyz, tri


def ref_export_ts(directory, base, suffix, xyz, tri):
    """The reference's InversionExporter(directory, base).exportTS(mesh, suffix)."""
    x = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
    t = np.ascontiguousarray(tri, np.int32).reshape(-1, 3)
    ref().ref_export_ts(str(directory).encode(), base.encode(), suffix.encode(), len(x), x.ctypes.data_as(_dp),
                        len(t), t.ctypes.data_as(_ip))


def _jacobian_worker(args):
    tables, densities, susceptibilities, inducing, params, sta, kind, true_h = args
    om = OracleModel(tables, densities, susceptibilities, inducing)
    om.scatter(params)
    return om.jacobian(sta, kind, true_h=true_h)


# Step of the Richardson "true" derivative used by the full-size tests: a
# negative value makes the oracle take |TRUE_H| x the station-triangle
# distance per (station, facet).  A fixed step cannot serve every facet: the
# reference's oriented line-integral form loses digits for edges nearly
# collinear with a station, which a central difference amplifies by 1/h (on
# the icosphere the fixed 1e-2 m truth is 2.3e-6 off), while facets of deep
# DOF vertices can reach within 1 m of a station, where a large fixed step
# has O((h / d)^4) truncation.  The adaptive step converges on both (5e-8 on
# the icosphere, 1e-10 on the voxel model, between factors 1e-3 and 1e-2).
TRUE_H = -3e-3


def jacobian_parallel(tables, densities, susceptibilities, inducing, params, sta, kind, procs=None,
                      true_h=TRUE_H):
    """OracleModel(...).scatter(params) then .jacobian(sta, kind), split over
    station chunks in spawned processes (spawned, not forked: the calling
    process may already hold a CUDA context).  Each process starts from the
    model's initial positions, like a fresh context evaluated once."""
    import multiprocessing as mp

    sta = np.ascontiguousarray(sta, np.float64)
    if procs is None:
        try:
            procs = len(os.sched_getaffinity(0))
        except AttributeError:
            procs = os.cpu_count() or 1
    procs = max(1, min(procs, len(sta)))
    chunks = np.array_split(np.arange(len(sta)), procs)
    jobs = [(tables, densities, susceptibilities, inducing, params, sta[c], kind, true_h) for c in chunks if len(c)]
    if len(jobs) == 1:
        return _jacobian_worker(jobs[0])
    with mp.get_context("spawn").Pool(len(jobs)) as pool:
        parts = pool.map(_jacobian_worker, jobs)
    return np.concatenate(parts, axis=0)
