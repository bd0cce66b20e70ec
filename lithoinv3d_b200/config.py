"""INI configuration of an inversion, and the settings of it that reach this
library's path.

* ``IniConfig`` reads and writes the reference's INI files with its rules
  (ini_config.cpp:29-67 ``load``, :69-80 ``save``, :96-133 the typed
  getters): ``#`` / ``;`` comment lines, ``[section]`` headers, ``key = value``
  or ``key: value`` (the first ``=``, else the first ``:``), keys and values
  trimmed, lines before the first section ignored, the last duplicate wins;
  numbers parse a leading prefix as ``std::stod`` / ``std::stoi`` do and fall
  back to the default when there is none or it is out of range; booleans are
  true for ``true`` / ``yes`` / ``1`` / ``on`` (any case) and false for any
  other non-empty value.  ``save`` writes sections and keys in sorted order
  (the reference keeps them in a ``std::map``).
* ``InversionConfig`` mirrors ``InversionConfig::fromIni`` / ``toIni``
  (ini_config_wiring.cpp:6-128 / 130-257): the same keys, defaults and enum
  spellings.  Doubles are written as ``std::to_string`` writes them
  (``%f``, six decimals).
* ``apply_to_model``, ``apply_to_context``, ``fill_uncertainties``,
  ``geometry_bounds`` and ``lbfgsb_options`` do what ``InversionRunner``
  does with the settings on the path (runner.cpp): the control-point stride
  with its fall-back to full resolution (:35-42), default data
  uncertainties (:93-102), the inducing field and remanence mode (:109-118),
  the joint magnetic weight (:117-120), the smoothness weight ``lambda``
  (:167-170), the reference-model term (:173-179, captured at the start
  parameters), the hard depth bounds around the start (:241-247), the
  eigenvalue scaling of the magnetic weight at the start (:309-312) and the
  L-BFGS-B options (:203-210).  The constraint weight ``omega`` (:185-188)
  goes to ``Context.set_constraints`` with the constraint data.

Settings that belong to parts of the reference outside this library (the
GNCG solver, EM padding, topography preparation, property-inversion
scheduling, exports) are parsed, kept and written back, and not applied;
``apply_to_context`` refuses ``solver = gncg`` rather than run L-BFGS-B in
its place.
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass, fields

import numpy as np

from .api import XY_FREE, XYZ_FREE, Z_ONLY

__all__ = ["IniConfig", "InversionConfig", "apply_to_model", "apply_to_context", "fill_uncertainties",
           "geometry_bounds", "lbfgsb_options"]

_INT_MIN, _INT_MAX = -2 ** 31, 2 ** 31 - 1
_DBL_MIN = 2.2250738585072014e-308
# the prefixes strtod accepts (after the leading blanks it skips): decimal
# with an optional exponent, hexadecimal with an optional binary exponent,
# inf / infinity, nan / nan(chars)
_STOD = re.compile(r"[+-]?(?:"
                   r"0[xX](?:[0-9a-fA-F]+\.?[0-9a-fA-F]*|\.[0-9a-fA-F]+)(?:[pP][+-]?\d+)?"
                   r"|(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?"
                   r"|[iI][nN][fF](?:[iI][nN][iI][tT][yY])?"
                   r"|[nN][aA][nN](?:\([0-9A-Za-z_]*\))?)")
_STOI = re.compile(r"[+-]?\d+")
_BLANKS = " \t\n\v\f\r"


def _stod(s: str) -> float:
    """std::stod: the longest leading number strtod reads.  ValueError when
    there is none (invalid_argument), OverflowError when strtod reports a
    range error -- overflow, or a non-zero value that underflows to a
    subnormal or zero -- (out_of_range)."""
    m = _STOD.match(s.lstrip(_BLANKS))
    if not m:
        raise ValueError(s)
    t = m.group(0)
    body = t.lstrip("+-")
    neg = t.startswith("-")
    low = body.lower()
    if low.startswith("inf"):
        return -math.inf if neg else math.inf
    if low.startswith("nan"):
        return math.nan
    if low.startswith("0x"):
        h = body
        if "p" not in low:
            h += "p0"
        v = float.fromhex(("-" if neg else "") + h)
        digits = re.sub(r"[^1-9a-fA-F]", "", body[2:].split("p")[0].split("P")[0])
    else:
        try:
            v = float(t)
        except OverflowError:
            raise OverflowError(s) from None
        digits = re.sub(r"[^1-9]", "", body.split("e")[0].split("E")[0])
    if math.isinf(v) or (digits and abs(v) < _DBL_MIN):
        raise OverflowError(s)
    return v


def _stoi(s: str) -> int:
    """std::stoi: base-10 leading integer; ValueError when there is none,
    OverflowError outside int's range."""
    m = _STOI.match(s.lstrip(_BLANKS))
    if not m:
        raise ValueError(s)
    v = int(m.group(0))
    if v < _INT_MIN or v > _INT_MAX:
        raise OverflowError(s)
    return v


def _to_string(v: float) -> str:
    """std::to_string(double): printf's %f."""
    if math.isnan(v):
        return "-nan" if math.copysign(1.0, v) < 0 else "nan"
    if math.isinf(v):
        return "-inf" if v < 0 else "inf"
    return "%f" % v


class IniConfig:
    """Sections of key -> value strings (the reference's IniConfig)."""

    def __init__(self):
        self.data: dict[str, dict[str, str]] = {}

    # -- reading and writing files --------------------------------------
    def load(self, path) -> bool:
        """Reads a file; False if it cannot be opened (the previous contents
        are then kept, as in the reference)."""
        try:
            with open(path, "rb") as fh:
                raw = fh.read()
        except OSError:
            return False
        self.loads(raw.decode("latin-1"))
        return True

    def loads(self, text: str) -> None:
        self.data = {}
        section = ""
        # std::getline splits on '\n' only; a '\r' before it is trimmed away
        for line in text.split("\n"):
            t = line.strip(_BLANKS)
            if not t or t[0] in "#;":
                continue
            if t[0] == "[":
                end = t.find("]")
                if end < 0:
                    continue
                section = t[1:end].strip(_BLANKS)
                self.data.setdefault(section, {})
                continue
            sep = t.find("=")
            if sep < 0:
                sep = t.find(":")
            if sep < 0:
                continue
            key, value = t[:sep].strip(_BLANKS), t[sep + 1:].strip(_BLANKS)
            if key and section:
                self.data.setdefault(section, {})[key] = value

    def dumps(self) -> str:
        out = []
        for sec in sorted(self.data, key=lambda s: s.encode("latin-1")):
            out.append("[%s]\n" % sec)
            kv = self.data[sec]
            for k in sorted(kv, key=lambda s: s.encode("latin-1")):
                out.append("%s = %s\n" % (k, kv[k]))
            out.append("\n")
        return "".join(out)

    def save(self, path) -> None:
        with open(path, "wb") as fh:
            fh.write(self.dumps().encode("latin-1"))

    # -- queries ---------------------------------------------------------
    def has_section(self, section: str) -> bool:
        return section in self.data

    def sections(self) -> list:
        return sorted(self.data, key=lambda s: s.encode("latin-1"))

    def get_string(self, section: str, key: str, default: str = "") -> str:
        return self.data.get(section, {}).get(key, default)

    def get_double(self, section: str, key: str, default: float = 0.0) -> float:
        s = self.get_string(section, key, "")
        if not s:
            return default
        try:
            return _stod(s)
        except (ValueError, OverflowError):
            return default

    def get_int(self, section: str, key: str, default: int = 0) -> int:
        s = self.get_string(section, key, "")
        if not s:
            return default
        try:
            return _stoi(s)
        except (ValueError, OverflowError):
            return default

    def get_bool(self, section: str, key: str, default: bool = False) -> bool:
        s = self.get_string(section, key, "").lower()
        if not s:
            return default
        return s in ("true", "yes", "1", "on")

    # -- updates ---------------------------------------------------------
    def set_string(self, section: str, key: str, value: str) -> None:
        self.data.setdefault(section, {})[key] = value

    def set_double(self, section: str, key: str, value: float) -> None:
        self.set_string(section, key, _to_string(float(value)))

    def set_int(self, section: str, key: str, value: int) -> None:
        self.set_string(section, key, str(int(value)))

    def set_bool(self, section: str, key: str, value: bool) -> None:
        self.set_string(section, key, "true" if value else "false")


# (field, section, key, kind, default) in toIni's order; "enum" values are
# the strings the INI spells (fromIni maps unknown spellings to the default)
_SPEC = [
    ("max_iterations", "inversion", "max_iterations", "int", 500),
    ("tolerance", "inversion", "tolerance", "double", 1e-6),
    ("lambda_", "inversion", "lambda", "double", 1.0),
    ("omega", "inversion", "omega", "double", 1e6),
    ("lbfgs_history", "inversion", "lbfgs_history", "int", 10),
    ("fd_step", "inversion", "fd_step", "double", 1.0),
    ("armijo_c1", "inversion", "armijo_c1", "double", 1e-4),
    ("line_search_max_iter", "inversion", "line_search_max_iter", "int", 50),
    ("disable_line_search", "inversion", "disable_line_search", "bool", False),
    ("control_point_stride", "inversion", "control_point_stride", "int", 0),
    ("enable_property_inversion", "inversion", "enable_property_inversion", "bool", False),
    ("enable_geometry_inversion", "inversion", "enable_geometry_inversion", "bool", True),
    ("property_inversion_interval", "inversion", "property_inversion_interval", "int", 50),
    ("property_inversion_max_iter", "inversion", "property_inversion_max_iter", "int", 20),
    ("property_damping", "inversion", "property_damping", "double", 0.01),
    ("vertex_freedom", "inversion", "vertex_freedom", ("z_only", "xy_free", "xyz_free"), "z_only"),
    ("solver", "inversion", "solver", "string", "lbfgsb"),
    ("mesh_boundary_mode", "inversion", "mesh_boundary_mode", "string", "free"),
    ("gncg_cg_max_iter", "inversion", "gncg_cg_max_iter", "int", 50),
    ("gncg_cg_tolerance", "inversion", "gncg_cg_tolerance", "double", 1e-6),
    ("enable_eigenvalue_scaling", "inversion", "enable_eigenvalue_scaling", "bool", True),
    ("density_min", "gravity", "density_min", "double", 1.0),
    ("density_max", "gravity", "density_max", "double", 6.0),
    ("gravity_uncertainty", "gravity", "gravity_uncertainty", "double", 0.0),
    ("magnetic_weight", "magnetic", "magnetic_weight", "double", 1.0),
    ("inclination", "magnetic", "inclination", "double", 75.0),
    ("declination", "magnetic", "declination", "double", -20.0),
    ("field_nt", "magnetic", "field_nT", "double", 55000.0),
    ("magnetic_uncertainty", "magnetic", "magnetic_uncertainty", "double", 0.0),
    ("susceptibility_min", "magnetic", "susceptibility_min", "double", 0.0),
    ("susceptibility_max", "magnetic", "susceptibility_max", "double", 1.0),
    ("remanence_min", "magnetic", "remanence_min", "double", 0.0),
    ("remanence_max", "magnetic", "remanence_max", "double", 10.0),
    ("remanence_component_min", "magnetic", "remanence_component_min", "double", -10.0),
    ("remanence_component_max", "magnetic", "remanence_component_max", "double", 10.0),
    ("remanence_mode", "magnetic", "remanence_mode", ("effective_susceptibility", "fixed_vector", "vector"),
     "effective_susceptibility"),
    ("enable_padding_group", "padding", "enable_padding_group", "bool", False),
    ("padding_density_initial", "padding", "padding_density_initial", "double", 2.67),
    ("padding_density_lower", "padding", "padding_density_lower", "double", 1.0),
    ("padding_density_upper", "padding", "padding_density_upper", "double", 6.0),
    ("padding_depth", "padding", "padding_depth", "double", -100000.0),
    ("padding_susceptibility_initial", "padding", "padding_susceptibility_initial", "double", 0.0),
    ("padding_susceptibility_lower", "padding", "padding_susceptibility_lower", "double", 0.0),
    ("padding_susceptibility_upper", "padding", "padding_susceptibility_upper", "double", 1.0),
    ("padding_conductivity_initial", "padding", "padding_conductivity_initial", "double", 1e-4),
    ("padding_conductivity_lower", "padding", "padding_conductivity_lower", "double", 1e-5),
    ("padding_conductivity_upper", "padding", "padding_conductivity_upper", "double", 1e2),
    ("topography_mode", "topography", "mode", ("none", "raw", "terrain_corrected"), "none"),
    ("dem_file", "topography", "dem_file", "string", ""),
    ("datum_elevation", "topography", "datum_elevation", "double", 0.0),
    ("bouguer_density", "topography", "bouguer_density", "double", 2.67),
    ("padding_rings", "topography", "padding_rings", "int", 0),
    ("padding_cell_size", "topography", "padding_cell_size", "double", 0.0),
    ("invert_halfspace_properties", "topography", "invert_halfspace_properties", "bool", False),
    ("projected_beyond_survey_area", "topography", "projected_beyond_survey_area",
     ("independent_flat", "projected_beyond_survey"), "independent_flat"),
    ("enable_reference_model", "regularization", "enable_reference_model", "bool", False),
    ("lambda_ref", "regularization", "lambda_ref", "double", 0.1),
    ("gradient_smoothing_weight", "regularization", "gradient_smoothing_weight", "double", 0.0),
    ("enable_depth_bounds", "bounds", "enable_depth_bounds", "bool", False),
    ("depth_bound_margin", "bounds", "depth_bound_margin", "double", 500.0),
    ("fail_on_missing_meshes", "data", "fail_on_missing_meshes", "bool", True),
    ("iteration_export_dir", "output", "iteration_export_dir", "string", ""),
    ("line_search_export_dir", "output", "line_search_export_dir", "string", ""),
]

_FREEDOM = {"z_only": Z_ONLY, "xy_free": XY_FREE, "xyz_free": XYZ_FREE}
_REMANENCE = {"effective_susceptibility": 0, "fixed_vector": 1, "vector": 2}


@dataclass
class InversionConfig:
    """The INI-settable part of the reference's InversionConfig, one field per
    key (``lambda`` is ``lambda_``; enums hold their INI spelling)."""
    max_iterations: int = 500
    tolerance: float = 1e-6
    lambda_: float = 1.0
    omega: float = 1e6
    lbfgs_history: int = 10
    fd_step: float = 1.0
    armijo_c1: float = 1e-4
    line_search_max_iter: int = 50
    disable_line_search: bool = False
    control_point_stride: int = 0
    enable_property_inversion: bool = False
    enable_geometry_inversion: bool = True
    property_inversion_interval: int = 50
    property_inversion_max_iter: int = 20
    property_damping: float = 0.01
    vertex_freedom: str = "z_only"
    solver: str = "lbfgsb"
    mesh_boundary_mode: str = "free"
    gncg_cg_max_iter: int = 50
    gncg_cg_tolerance: float = 1e-6
    enable_eigenvalue_scaling: bool = True
    density_min: float = 1.0
    density_max: float = 6.0
    gravity_uncertainty: float = 0.0
    magnetic_weight: float = 1.0
    inclination: float = 75.0
    declination: float = -20.0
    field_nt: float = 55000.0
    magnetic_uncertainty: float = 0.0
    susceptibility_min: float = 0.0
    susceptibility_max: float = 1.0
    remanence_min: float = 0.0
    remanence_max: float = 10.0
    remanence_component_min: float = -10.0
    remanence_component_max: float = 10.0
    remanence_mode: str = "effective_susceptibility"
    enable_padding_group: bool = False
    padding_density_initial: float = 2.67
    padding_density_lower: float = 1.0
    padding_density_upper: float = 6.0
    padding_depth: float = -100000.0
    padding_susceptibility_initial: float = 0.0
    padding_susceptibility_lower: float = 0.0
    padding_susceptibility_upper: float = 1.0
    padding_conductivity_initial: float = 1e-4
    padding_conductivity_lower: float = 1e-5
    padding_conductivity_upper: float = 1e2
    topography_mode: str = "none"
    dem_file: str = ""
    datum_elevation: float = 0.0
    bouguer_density: float = 2.67
    padding_rings: int = 0
    padding_cell_size: float = 0.0
    invert_halfspace_properties: bool = False
    projected_beyond_survey_area: str = "independent_flat"
    enable_reference_model: bool = False
    lambda_ref: float = 0.1
    gradient_smoothing_weight: float = 0.0
    enable_depth_bounds: bool = False
    depth_bound_margin: float = 500.0
    fail_on_missing_meshes: bool = True
    iteration_export_dir: str = ""
    line_search_export_dir: str = ""

    @classmethod
    def from_ini(cls, ini: IniConfig) -> "InversionConfig":
        """InversionConfig::fromIni."""
        cfg = cls()
        for name, sec, key, kind, default in _SPEC:
            if kind == "int":
                v = ini.get_int(sec, key, default)
            elif kind == "double":
                v = ini.get_double(sec, key, default)
            elif kind == "bool":
                v = ini.get_bool(sec, key, default)
            elif kind == "string":
                v = ini.get_string(sec, key, default)
            else:  # enum: an unknown spelling is the default
                s = ini.get_string(sec, key, default)
                v = s if s in kind else default
            setattr(cfg, name, v)
        return cfg

    @classmethod
    def from_file(cls, path) -> "InversionConfig":
        ini = IniConfig()
        if not ini.load(path):
            raise OSError("cannot open INI file %s" % path)
        return cls.from_ini(ini)

    def to_ini(self) -> IniConfig:
        """InversionConfig::toIni (the export directories only when set)."""
        ini = IniConfig()
        for name, sec, key, kind, _ in _SPEC:
            v = getattr(self, name)
            if kind == "int":
                ini.set_int(sec, key, v)
            elif kind == "double":
                ini.set_double(sec, key, v)
            elif kind == "bool":
                ini.set_bool(sec, key, v)
            elif kind == "string":
                if sec == "output" and not v:
                    continue
                ini.set_string(sec, key, v)
            else:
                ini.set_string(sec, key, v if v in kind else kind[0])
        return ini

    # the enums as this library's constants
    @property
    def freedom(self) -> int:
        """Vertex freedom for ``Model.set_group_mesh`` (``LF_Z_ONLY``,
        ``LF_XY_FREE``, ``LF_XYZ_FREE``)."""
        return _FREEDOM.get(self.vertex_freedom, Z_ONLY)

    @property
    def remanence(self) -> int:
        """``LF_REM_*`` for ``Context.set_field``."""
        return _REMANENCE.get(self.remanence_mode, 0)


def apply_to_model(model, cfg: InversionConfig) -> int:
    """The control-point stride (runner.cpp:35-42): returns the coarse DOF
    count, or 0 when the grids do not allow the stride, in which case the
    model stays at full resolution and ``cfg.control_point_stride`` is reset
    to 0 as the runner does."""
    if cfg.control_point_stride <= 0:
        return 0
    n = model.set_control_point_stride(cfg.control_point_stride)
    if n == 0:
        cfg.control_point_stride = 0
    return n


def fill_uncertainties(std, default: float) -> np.ndarray:
    """runner.cpp:93-102: with a positive default, every standard deviation
    <= 0 becomes the default; otherwise the values are kept."""
    s = np.array(std, dtype=np.float64, copy=True)
    if default > 0.0:
        s[s <= 0.0] = default
    return s


def geometry_bounds(cfg: InversionConfig, params, lower, upper):
    """The L-BFGS-B box: the model's bounds, clipped to +- depth_bound_margin
    around the start when enable_depth_bounds (runner.cpp:241-247)."""
    lo = np.array(lower, dtype=np.float64, copy=True)
    hi = np.array(upper, dtype=np.float64, copy=True)
    if cfg.enable_depth_bounds:
        p = np.asarray(params, dtype=np.float64)
        lo = np.maximum(lo, p - cfg.depth_bound_margin)
        hi = np.minimum(hi, p + cfg.depth_bound_margin)
    return lo, hi


def lbfgsb_options(cfg: InversionConfig) -> dict:
    """Keyword arguments of ``Context.lbfgsb`` (runner.cpp:203-210, with the
    iteration cap of the geometry phase)."""
    return {"max_iterations": cfg.max_iterations, "tolerance": cfg.tolerance, "history_size": cfg.lbfgs_history,
            "armijo_c1": cfg.armijo_c1, "line_search_max_iter": cfg.line_search_max_iter,
            "disable_line_search": cfg.disable_line_search}


def apply_to_context(ctx, cfg: InversionConfig, params, has_magnetic=None):
    """The objective settings of ``InversionRunner::setup`` / ``run`` on a
    context whose model and data are set: inducing field and remanence mode,
    magnetic weight, smoothness weight ``lambda``, the reference-model term
    at ``params`` (the start) when enabled, then -- with magnetic data,
    eigenvalue scaling enabled and a positive magnetic weight -- the data-weight
    calibration at ``params``, which rescales the magnetic weight.  Returns
    the calibration's (alpha_mag, lambda_grav, lambda_mag), or None."""
    if cfg.solver == "gncg":
        raise NotImplementedError("solver = gncg: this library provides the L-BFGS-B geometry optimizer only")
    p = np.asarray(params, dtype=np.float64)
    ctx.set_field(cfg.inclination, cfg.declination, cfg.field_nt, cfg.remanence)
    ref = cfg.lambda_ref if cfg.enable_reference_model else 0.0
    ctx.set_objective(cfg.magnetic_weight, ref, p if cfg.enable_reference_model else None)
    ctx.set_smoothness(cfg.lambda_)
    if has_magnetic is None:
        has_magnetic = getattr(ctx, "n_mag", 0) > 0
    if has_magnetic and cfg.enable_eigenvalue_scaling and cfg.magnetic_weight > 0.0:
        return ctx.calibrate_data_weights(p)
    return None


# every _SPEC field is a dataclass field
assert {s[0] for s in _SPEC} <= {f.name for f in fields(InversionConfig)}
