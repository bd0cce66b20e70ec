"""INI configuration (lithoinv3d_b200.config): the parser against the
reference's own IniConfig (ini_config.cpp, compiled unmodified into
oracle/_ref/ini_ref with a query driver) on a file with every parsing rule;
InversionConfig::fromIni / toIni's keys, defaults and number formats
(ini_config_wiring.cpp); and the runner's use of the settings on the path
(runner.cpp), on fakes that record the calls.  CPU only."""
import math
import os
import subprocess

import numpy as np
import pytest

from lithoinv3d_b200 import XYZ_FREE, Z_ONLY
from lithoinv3d_b200.api import XY_FREE
from lithoinv3d_b200.config import (IniConfig, InversionConfig, apply_to_context, apply_to_model,
                                    fill_uncertainties, geometry_bounds, lbfgsb_options)

REF_INI = os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "ini_ref")

# every rule the reference's loader has: comments, text before the first
# section, '=' before ':', trimming, a header without ']', a repeated section,
# number prefixes, out-of-range numbers, hexadecimal, empty values, CRLF
EDGE_INI = "\n".join([
    "; leading comment",
    "# another",
    "orphan = before any section",
    "[inversion]",
    "max_iterations = 250",
    "tolerance=1e-7",
    "lambda : 0.5",
    "omega = 2e6 # trailing text",
    "lbfgs_history =   7   ",
    "armijo_c1 = .5e-3x",
    "line_search_max_iter = 12.9",
    "disable_line_search = YES",
    "control_point_stride = 0x10",
    "vertex_freedom = xyz_free",
    "solver =",
    "   [  magnetic  ]   ",
    "inclination = -65.5",
    "declination = inf",
    "field_nT = 1e400",
    "magnetic_weight = nan",
    "remanence_mode = vector",
    "magnetic_uncertainty = 1e-400",
    "susceptibility_max = 4.9e-324",
    "remanence_min = -0x1.8p1",
    "[bad",
    "key without separator",
    "[gravity]",
    "density_min = abc",
    "density_max = +3",
    "gravity_uncertainty = 0.25\r",
    "[inversion]",
    "max_iterations = 300",
    "property_inversion_interval = 99999999999",
    "property_inversion_max_iter = -2147483648",
    "[empty]",
    "[data]",
    "fail_on_missing_meshes = off",
    "weird = a=b:c",
    "[topography]",
    "mode = Raw",
    "padding_rings = 3",
    "[output]",
    "iteration_export_dir = /tmp/out dir",
    "",
])

QUERY_KEYS = [(s, k) for s, body in [
    ("inversion", ["max_iterations", "tolerance", "lambda", "omega", "lbfgs_history", "armijo_c1",
                   "line_search_max_iter", "disable_line_search", "control_point_stride", "vertex_freedom",
                   "solver", "property_inversion_interval", "property_inversion_max_iter", "missing"]),
    ("magnetic", ["inclination", "declination", "field_nT", "magnetic_weight", "remanence_mode",
                  "magnetic_uncertainty", "susceptibility_max", "remanence_min"]),
    ("gravity", ["density_min", "density_max", "gravity_uncertainty"]),
    ("data", ["fail_on_missing_meshes", "weird"]),
    ("topography", ["mode", "padding_rings"]),
    ("output", ["iteration_export_dir"]),
    ("nosuch", ["max_iterations"]),
    ("", ["orphan"]),
] for k in body]


def _same_double(a: float, b: float) -> bool:
    return (math.isnan(a) and math.isnan(b)) or a == b


@pytest.mark.skipif(not os.path.exists(REF_INI), reason="oracle/_ref/ini_ref is built only where the reference tree is")
@pytest.mark.parametrize("eol", ["\n", "\r\n"])
def test_parser_matches_reference(tmp_path, eol):
    path = tmp_path / "edge.ini"
    path.write_bytes(EDGE_INI.replace("\n", eol).encode())
    ours = IniConfig()
    assert ours.load(path)
    queries, expect = [], []
    for sec, key in QUERY_KEYS:
        queries += ["S\t%s\t%s\tdflt" % (sec, key), "D\t%s\t%s\t-7.25" % (sec, key),
                    "I\t%s\t%s\t-7" % (sec, key), "B\t%s\t%s\t1" % (sec, key)]
        expect += [("S", ours.get_string(sec, key, "dflt")), ("D", ours.get_double(sec, key, -7.25)),
                   ("I", ours.get_int(sec, key, -7)), ("B", ours.get_bool(sec, key, True))]
    for sec in ("inversion", "magnetic", "bad", "empty", "nosuch", ""):
        queries.append("H\t%s" % sec)
        expect.append(("H", ours.has_section(sec)))
    queries.append("L")
    expect.append(("L", "\t".join(ours.sections())))
    saved = tmp_path / "ref_saved.ini"
    queries.append("W\t%s" % saved)
    expect.append(("W", "saved"))
    out = subprocess.run([REF_INI, str(path)], input="\n".join(queries) + "\n", capture_output=True, text=True,
                         check=True).stdout.split("\n")
    assert out[0] == "1"
    for q, (kind, want), got in zip(queries, expect, out[1:]):
        if kind == "D":
            assert _same_double(float(got), want), (q, got, want)
        elif kind in ("I",):
            assert int(got) == want, (q, got, want)
        elif kind in ("B", "H"):
            assert bool(int(got)) == want, (q, got, want)
        else:
            assert got == want, (q, got, want)
    # save(): sorted sections and keys, "key = value" lines, a blank line after each section
    assert saved.read_bytes() == ours.dumps().encode("latin-1")


def test_parser_rules_without_reference():
    ini = IniConfig()
    ini.loads(EDGE_INI)
    assert ini.get_string("", "orphan", "x") == "x"                       # before any section: dropped
    assert ini.get_int("inversion", "max_iterations") == 300               # repeated section: last wins
    assert ini.get_double("inversion", "lambda") == 0.5                    # ':' separator
    assert ini.get_double("inversion", "omega") == 2e6                     # numeric prefix
    assert ini.get_double("inversion", "armijo_c1") == 0.5e-3
    assert ini.get_int("inversion", "line_search_max_iter") == 12          # stoi stops at '.'
    assert ini.get_int("inversion", "control_point_stride", 9) == 0        # base 10: "0" of "0x10"
    assert ini.get_double("inversion", "control_point_stride") == 16.0     # strtod reads hexadecimal
    assert ini.get_bool("inversion", "disable_line_search") is True
    assert ini.get_string("inversion", "solver", "d") == ""                # present but empty
    assert ini.get_double("inversion", "solver", 4.0) == 4.0
    assert ini.has_section("magnetic")                                    # header trimmed
    assert ini.get_double("magnetic", "declination") == math.inf
    assert ini.get_double("magnetic", "field_nT", 55000.0) == 55000.0      # overflow -> default
    assert math.isnan(ini.get_double("magnetic", "magnetic_weight"))
    assert ini.get_double("magnetic", "magnetic_uncertainty", 1.5) == 1.5  # underflow -> default
    assert ini.get_double("magnetic", "remanence_min") == -3.0
    assert not ini.has_section("bad")                                     # header without ']'
    assert ini.get_double("gravity", "density_min", 1.0) == 1.0            # no number -> default
    assert ini.get_double("gravity", "gravity_uncertainty") == 0.25        # '\r' trimmed
    assert ini.get_int("inversion", "property_inversion_interval", 50) == 50  # out of int range
    assert ini.get_int("inversion", "property_inversion_max_iter") == -2 ** 31
    assert ini.get_bool("data", "fail_on_missing_meshes", True) is False
    assert ini.get_string("data", "weird") == "a=b:c"                      # first '=' splits
    assert ini.get_string("output", "iteration_export_dir") == "/tmp/out dir"
    assert ini.sections() == ["data", "empty", "gravity", "inversion", "magnetic", "output", "topography"]
    assert not IniConfig().load("/nonexistent/dir/file.ini")


def test_from_ini_defaults_are_the_reference_defaults():
    cfg = InversionConfig.from_ini(IniConfig())
    assert cfg == InversionConfig()
    # a sample of ini_config_wiring.cpp:9-124's defaults
    assert (cfg.max_iterations, cfg.tolerance, cfg.lambda_, cfg.omega, cfg.lbfgs_history) == (500, 1e-6, 1.0, 1e6, 10)
    assert (cfg.armijo_c1, cfg.line_search_max_iter, cfg.control_point_stride) == (1e-4, 50, 0)
    assert (cfg.inclination, cfg.declination, cfg.field_nt, cfg.magnetic_weight) == (75.0, -20.0, 55000.0, 1.0)
    assert (cfg.lambda_ref, cfg.depth_bound_margin, cfg.padding_depth) == (0.1, 500.0, -100000.0)
    assert cfg.enable_eigenvalue_scaling and cfg.enable_geometry_inversion and cfg.fail_on_missing_meshes
    assert cfg.freedom == Z_ONLY and cfg.remanence == 0 and cfg.solver == "lbfgsb"


def test_from_ini_values_and_enums():
    ini = IniConfig()
    ini.loads(EDGE_INI)
    cfg = InversionConfig.from_ini(ini)
    assert (cfg.max_iterations, cfg.tolerance, cfg.lambda_, cfg.omega, cfg.lbfgs_history) == (300, 1e-7, 0.5, 2e6, 7)
    assert cfg.line_search_max_iter == 12 and cfg.disable_line_search and cfg.control_point_stride == 0
    assert cfg.vertex_freedom == "xyz_free" and cfg.freedom == XYZ_FREE
    assert cfg.solver == ""  # fromIni keeps the empty string (getString finds the key)
    assert cfg.remanence_mode == "vector" and cfg.remanence == 2
    assert cfg.field_nt == 55000.0 and math.isnan(cfg.magnetic_weight) and cfg.declination == math.inf
    assert cfg.topography_mode == "none"  # "Raw": the comparison is case-sensitive
    assert cfg.padding_rings == 3 and not cfg.fail_on_missing_meshes
    assert cfg.iteration_export_dir == "/tmp/out dir" and cfg.line_search_export_dir == ""
    for spelled, code in (("xy_free", XY_FREE), ("z_only", Z_ONLY), ("other", Z_ONLY)):
        ini.set_string("inversion", "vertex_freedom", spelled)
        assert InversionConfig.from_ini(ini).freedom == code


def test_to_ini_text_and_round_trip():
    cfg = InversionConfig()
    text = cfg.to_ini().dumps()
    # std::to_string(double) is %f: six decimals
    assert "tolerance = 0.000001\n" in text and "omega = 1000000.000000\n" in text
    assert "padding_depth = -100000.000000\n" in text and "max_iterations = 500\n" in text
    assert "disable_line_search = false\n" in text and "vertex_freedom = z_only\n" in text
    assert "[output]" not in text  # export directories only when set
    assert text.startswith("[bounds]\ndepth_bound_margin = 500.000000\nenable_depth_bounds = false\n\n[data]\n")
    assert InversionConfig.from_ini(cfg.to_ini()) == cfg
    cfg.iteration_export_dir, cfg.remanence_mode, cfg.tolerance = "/x", "fixed_vector", 1e-7
    back = InversionConfig.from_ini(cfg.to_ini())
    assert back.iteration_export_dir == "/x" and back.remanence_mode == "fixed_vector"
    assert back.tolerance == 0.0  # 1e-7 written as 0.000000, as the reference writes it


class _FakeContext:
    def __init__(self, n_mag):
        self.n_mag = n_mag
        self.calls = []

    def set_field(self, *a):
        self.calls.append(("set_field", a))

    def set_objective(self, *a):
        self.calls.append(("set_objective", a))

    def set_smoothness(self, w):
        self.calls.append(("set_smoothness", (w,)))

    def calibrate_data_weights(self, p):
        self.calls.append(("calibrate", (p.copy(),)))
        return (2.5, 1.0, 0.4)


def test_apply_to_context_follows_the_runner():
    p = np.array([1.0, -2.0, 3.0])
    cfg = InversionConfig(inclination=60.0, declination=5.0, field_nt=50000.0, remanence_mode="fixed_vector",
                          magnetic_weight=0.7, lambda_=0.3)
    ctx = _FakeContext(n_mag=10)
    assert apply_to_context(ctx, cfg, p) == (2.5, 1.0, 0.4)
    assert [c[0] for c in ctx.calls] == ["set_field", "set_objective", "set_smoothness", "calibrate"]
    assert ctx.calls[0][1] == (60.0, 5.0, 50000.0, 1)
    assert ctx.calls[1][1] == (0.7, 0.0, None)
    assert ctx.calls[2][1] == (0.3,)
    # reference model on: its weight and the start parameters
    cfg.enable_reference_model, cfg.lambda_ref = True, 0.05
    ctx = _FakeContext(n_mag=10)
    apply_to_context(ctx, cfg, p)
    w, lam, ref = ctx.calls[1][1]
    assert (w, lam) == (0.7, 0.05) and np.array_equal(ref, p)
    # no calibration without magnetic data, with the scaling off, or with weight 0
    for n_mag, scale, mw in ((0, True, 0.7), (10, False, 0.7), (10, True, 0.0)):
        ctx = _FakeContext(n_mag)
        cfg.enable_eigenvalue_scaling, cfg.magnetic_weight = scale, mw
        assert apply_to_context(ctx, cfg, p) is None
        assert "calibrate" not in [c[0] for c in ctx.calls]
    with pytest.raises(NotImplementedError):
        apply_to_context(_FakeContext(0), InversionConfig(solver="gncg"), p)


class _FakeModel:
    def __init__(self, result):
        self.result, self.asked = result, []

    def set_control_point_stride(self, s):
        self.asked.append(s)
        return self.result


def test_apply_to_model_stride_and_fallback():
    cfg = InversionConfig(control_point_stride=4)
    m = _FakeModel(120)
    assert apply_to_model(m, cfg) == 120 and m.asked == [4] and cfg.control_point_stride == 4
    m = _FakeModel(0)  # grids unsuitable: full resolution, stride reset as runner.cpp:39-42 does
    assert apply_to_model(m, cfg) == 0 and cfg.control_point_stride == 0
    m = _FakeModel(5)
    assert apply_to_model(m, cfg) == 0 and m.asked == []


def test_bounds_uncertainties_and_optimizer_options():
    p = np.array([0.0, 10.0, -5.0])
    lo, hi = np.array([-1e9, 0.0, -1e9]), np.array([1e9, 1e9, -4.0])
    cfg = InversionConfig(enable_depth_bounds=True, depth_bound_margin=50.0)
    blo, bhi = geometry_bounds(cfg, p, lo, hi)
    assert np.array_equal(blo, [-50.0, 0.0, -55.0]) and np.array_equal(bhi, [50.0, 60.0, -4.0])
    cfg.enable_depth_bounds = False
    blo, bhi = geometry_bounds(cfg, p, lo, hi)
    assert np.array_equal(blo, lo) and np.array_equal(bhi, hi)
    s = np.array([0.0, -1.0, 0.2])
    assert np.array_equal(fill_uncertainties(s, 0.5), [0.5, 0.5, 0.2])
    assert np.array_equal(fill_uncertainties(s, 0.0), s)
    opt = lbfgsb_options(InversionConfig(max_iterations=40, tolerance=1e-5, lbfgs_history=6, armijo_c1=1e-3,
                                         line_search_max_iter=9, disable_line_search=True))
    assert opt == {"max_iterations": 40, "tolerance": 1e-5, "history_size": 6, "armijo_c1": 1e-3,
                   "line_search_max_iter": 9, "disable_line_search": True}


def test_apply_to_model_on_a_built_model():
    """The stride from the INI on a model built at full resolution gives the
    model the builder makes with that stride (same DOF count and start)."""
    from lithoinv3d_b200 import synth
    from lithoinv3d_b200.api import Model

    p = synth.voxel_contact_model(shape=(8, 8, 6), n_side=8, cp_stride=4)
    want = p.build_model()
    m = Model()
    for g, (rho, chi) in enumerate(zip(p.densities, p.susceptibilities)):
        m.add_group(g, rho, chi)
    for g, (V, F, fr) in enumerate(p.meshes):
        m.set_group_mesh(g, V, F, fr)
    full = m.n_dofs
    ini = IniConfig()
    ini.loads("[inversion]\ncontrol_point_stride = 4\n")
    cfg = InversionConfig.from_ini(ini)
    assert apply_to_model(m, cfg) > 0 and cfg.control_point_stride == 4
    m.build_shared_vertex_sync()
    assert m.n_dofs == want.n_dofs < full
    assert np.array_equal(m.assemble_parameters(), want.assemble_parameters())


@pytest.mark.skipif(not os.path.exists(REF_INI), reason="oracle/_ref/ini_ref is built only where the reference tree is")
def test_real_configs_read_as_the_reference_reads_them(tmp_path):
    """The reference's own run configurations (apps/forrestania/*.ini): every
    key of every section through both parsers, save's bytes, and fromIni's
    typed fields from the reference parser's answers."""
    root = os.environ.get("LITHO_REFERENCE")
    if not root:
        pytest.skip("LITHO_REFERENCE (the reference tree) is not set")
    import glob
    from lithoinv3d_b200.config import _SPEC

    files = sorted(glob.glob(os.path.join(root, "apps/forrestania/*.ini")))
    if not files:
        pytest.skip("reference configurations not present")
    for f in files:
        ours = IniConfig()
        assert ours.load(f)
        keys = [(s, k) for s in ours.sections() for k in ours.data[s]]
        assert keys, f
        queries = ["S\t%s\t%s\t" % sk for sk in keys]
        queries += ["%s\t%s\t%s\t%s" % ({"int": "I", "double": "D", "bool": "B"}[kind], sec, key,
                                        ("1" if default else "0") if kind == "bool" else repr(default))
                    for _, sec, key, kind, default in _SPEC if kind in ("int", "double", "bool")]
        saved = tmp_path / "saved.ini"
        queries.append("W\t%s" % saved)
        out = subprocess.run([REF_INI, f], input="\n".join(queries) + "\n", capture_output=True, text=True,
                             check=True).stdout.split("\n")
        assert out[0] == "1"
        assert out[1:1 + len(keys)] == [ours.get_string(s, k) for s, k in keys], f
        cfg = InversionConfig.from_ini(ours)
        typed = [sp for sp in _SPEC if sp[3] in ("int", "double", "bool")]
        for (name, _, _, kind, _), got in zip(typed, out[1 + len(keys):]):
            v = getattr(cfg, name)
            if kind == "double":
                assert _same_double(float(got), v), (f, name, got, v)
            else:
                assert int(got) == int(v), (f, name, got, v)
        assert saved.read_bytes() == ours.dumps().encode("latin-1"), f
