"""Host side: the YAML grammar of src/config.cpp, the geometry plugins and the
expression initial condition against the reference's own code, and the
boundary-table compiler's error behaviour."""
import ctypes as C

import numpy as np
import pytest

from oracle import bind
from tests import cases
from tests.emu import Emu

pkg = cases.pkg
N = pkg._native


def test_field_cond_grammar():
    p = pkg.config.parse_field_cond
    assert p(None).type == "neumann"
    assert p("neumann").type == "neumann"
    assert (p("dirichlet").type, p("dirichlet").value) == ("dirichlet", 0.0)
    assert p("axis_lf").type == "axis_lf"
    fc = p("v_z * r_z")
    assert (fc.type, fc.expr_str) == ("expression", "v_z * r_z")
    assert (p({"neumann": "0.5"}).type, p({"neumann": "0.5"}).value) == ("neumann", 0.5)
    assert p({"dirichlet": "1.0"}).value == 1.0
    assert p({"expr": "r_0 / r"}).expr_str == "r_0 / r"
    assert p({"type": "neumann", "gradient": "0.25"}).value == 0.25
    assert p({"type": "neumann", "value": "0.5"}).value == 0.5
    assert p({"type": "dirichlet", "value": "2"}).value == 2.0
    assert p({"type": "expression", "expr": "H_z * r_z"}).expr_str == "H_z * r_z"
    assert p({"type": "axis_lf"}).type == "axis_lf"
    for bad, msg in [("wall_tangent", "no longer a built-in preset"),
                     ("hphi_r0_over_r", "r_0 / r"),
                     ({"type": "wall_tangent"}, "no longer supported"),
                     ({"type": "magic"}, "unknown field condition type 'magic'"),
                     ({"type": "expression"}, "requires an 'expr' key"),
                     ({"foo": "1"}, "must contain one of"),
                     ({"neumann": ["1"]}, "must be a scalar number"),
                     (["x"], "field condition must be")]:
        with pytest.raises(pkg.ConfigError, match=msg):
            p(bad)


def test_yaml_loader_sections_and_faces():
    cfg = cases.reference_default_config(L=80, M=40)
    assert (cfg.gamma, cfg.beta, cfg.H_z0) == (1.67, 0.01, 0.25)
    assert cfg.adaptive_dt and cfg.cfl_number == 0.45 and cfg.dt_max == 5.0e-5
    assert (cfg.L_max, cfg.M_max, cfg.dz, cfg.dy) == (80, 40, 1.0 / 80, 1.0 / 40)
    assert cfg.geometry.type == "short_cathode_cosine"
    assert cfg.geometry.params["transition_half_width"] == "0.02"
    assert [len(f.segments) for f in cfg.faces()] == [1, 1, 3, 1]
    s = cfg.bc_m_lo.segments[2]
    assert (s.global_lo, s.global_hi, s.rho.type, s.v_r.type, s.v_r.value) == (26, -1, "axis_lf",
                                                                               "dirichlet", 0.0)
    assert cfg.bc_l_lo.segments[0].H_phi.expr_str == "r_0 / r"
    assert cfg.initial_conditions.params["H_z"] == "H_z0"
    with pytest.raises(pkg.ConfigError, match="two-element sequence"):
        pkg.SimConfig.from_yaml("boundary_conditions:\n  l_lo:\n    - range: [1]\n")
    with pytest.raises(pkg.ConfigError, match="YAML sequence"):
        pkg.SimConfig.from_yaml("boundary_conditions:\n  l_lo: {rho: neumann}\n")
    with pytest.raises(pkg.ConfigError, match="no longer supported"):
        pkg.SimConfig.from_yaml("initial_conditions:\n  type: expression\n")


@pytest.mark.skipif(not bind.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("gtype,params", [
    ("short_cathode_cosine", {}),
    ("short_cathode_cosine", {"z_center": "0.31", "transition_half_width": "0.02",
                              "r_inner_before": "0.2", "r_inner_after": "0.005", "r_outer": "0.8"}),
    ("short_cathode_parabolic", {}),
    ("villani_mpdt", {}),
    ("villani_mpdt", {"cathode_tip_half_width": "0", "anode_tip_half_width": "0.03"}),
])
def test_geometry_plugins_match_reference(gtype, params):
    L = 250
    want = bind.ref_geometry_profile(gtype, params, L, 1.0 / L)
    cfg = pkg.SimConfig(L_max=L, M_max=50)
    g = pkg.GeometryRegistry.Instance().Create(gtype, params)
    grid = pkg.Grid(cfg, g)
    for got, ref in zip(grid.profiles(), want):
        np.testing.assert_array_equal(got, ref)


def test_sine_wall_geometry():
    g = pkg.GeometryRegistry.Instance().Create("sine_wall", {"r1": "0.2", "r2": "0.8", "a": "0.3"})
    assert g.RInner(0.7) == 0.2
    assert g.ROuter(0.5) == 0.8 - 0.3 * np.sin(np.pi * 0.5)
    assert g.DrOuterDz(0.25) == -0.3 * np.pi * np.cos(np.pi * 0.25)
    with pytest.raises(pkg.geometry.GeometryError):
        pkg.GeometryRegistry.Instance().Create("sine_wall", {"a": "0.7"})
    with pytest.raises(pkg.geometry.GeometryError, match="unknown geometry type"):
        pkg.GeometryRegistry.Instance().Create("no_such", {})


@pytest.mark.skipif(not bind.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("cfg", [cases.reference_default_config(L=40, M=20),
                                 cases.channel_config(L=30, M=12, a=0.2, amp=1.7, vz=0.21)])
def test_expression_ic_matches_reference(cfg):
    case = cases.make_case(cfg)
    params = [cfg.gamma, cfg.beta, cfg.H_z0, cfg.dz, cfg.dy, case.grid.r_0]
    want = bind.ref_expression_ic(cfg.initial_conditions.params, cfg.L_max, cfg.M_max, params,
                                  *case.grid.profiles())
    np.testing.assert_array_equal(case.phys, want)


@pytest.mark.skipif(not bind.ref_available(), reason="oracle/_ref not built")
def test_expression_ic_defaults_and_leftovers_match_reference():
    """Missing fields take the reference defaults; a field reading a later one
    sees the previous cell's value, exactly as the reference's symbol table."""
    cfg = cases.channel_config(L=20, M=8, a=0.1)
    ic = {"rho": "1 + e", "v_z": "0.1 * sin(pi * z) + sqrt(r)", "H_r": "H_z * r_z + 0.5 * v_r"}
    cfg.initial_conditions = pkg.config.ICConfig(params=ic)
    case = cases.make_case(cfg)
    params = [cfg.gamma, cfg.beta, cfg.H_z0, cfg.dz, cfg.dy, case.grid.r_0]
    want = bind.ref_expression_ic(ic, cfg.L_max, cfg.M_max, params, *case.grid.profiles())
    np.testing.assert_allclose(case.phys, want, rtol=0, atol=0)


def test_expression_ic_user_vars_and_errors():
    cfg = cases.channel_config(L=12, M=6)
    geom = pkg.GeometryRegistry.Instance().Create("sine_wall", cfg.geometry.params)
    grid = pkg.Grid(cfg, geom)
    phys = pkg.ExpressionIC({"rho": "k * 2", "vars": {"k": "0.25"}}).Apply(grid, cfg)
    assert (phys[0, 1:-1, 1:-1] == 0.5).all()
    with pytest.raises(N.MpdError, match="shadows the built-in symbol"):
        pkg.ExpressionIC({"vars": {"beta": "1"}}).Apply(grid, cfg)
    with pytest.raises(N.MpdError, match="failed to compile expression for 'v_z'"):
        pkg.ExpressionIC({"v_z": "1 +"}).Apply(grid, cfg)


def _emu_error(cfg):
    case = cases.make_case(cfg)
    with pytest.raises(N.MpdError) as ei:
        Emu(case)
    return ei.value


def test_bc_compile_errors():
    cfg = cases.channel_config(L=12, M=6)
    cfg.bc_l_hi.segments = [cases.segment(rho="axis_lf")]
    e = _emu_error(cfg)
    assert e.code == N.MPD_ERR_INVALID and "only valid on the M_LO face" in str(e)
    cfg = cases.channel_config(L=12, M=6)
    cfg.bc_m_lo.segments = [cases.segment(v_r="axis_lf")]
    e = _emu_error(cfg)
    assert e.code == N.MPD_ERR_INVALID and "'v_r' has no AxisLF formula" in str(e)
    cfg = cases.channel_config(L=12, M=6)
    cfg.bc_m_hi.segments = [cases.segment(v_r=("expr", "v_z * * r_z"))]
    e = _emu_error(cfg)
    assert e.code == N.MPD_ERR_EXPR and "failed to compile BC expression for field 'v_r'" in str(e)
    cfg = cases.channel_config(L=12, M=6)
    cfg.bc_m_hi.segments = [cases.segment(v_r=("expr", "e * r_z"))]
    e = _emu_error(cfg)
    assert e.code == N.MPD_ERR_UNSUPPORTED_BC and "forward reference" in str(e)


def test_eval_expression_matches_oracle_evaluator():
    lib = N.load()
    names = (C.c_char_p * 3)(b"x", b"y", b"z")
    vals = np.array([0.3, -1.7, 2.5])
    exprs = ["x + y * z", "-x^2", "2^3^2", "min(x, y, z) + max(x, y)", "clamp(0, y, 1)",
             "atan2(y, x) / pi", "sign(y) * abs(y) % 0.5", "log10(z) + log2(z) + exp(x)",
             "((x - y) / (z + 1)) * 3.5e-2"]
    for src in exprs:
        out = C.c_double()
        rc = lib.mpd_eval_expression(src.encode(), 3, names, vals.ctypes.data_as(N.DP),
                                     C.byref(out))
        assert rc == 0, src
        x, y, z = vals
        ref = {"x + y * z": x + y * z, "-x^2": -(x ** 2), "2^3^2": 2.0 ** 9,
               "min(x, y, z) + max(x, y)": y + x, "clamp(0, y, 1)": 0.0,
               "atan2(y, x) / pi": np.arctan2(y, x) / np.pi,
               "sign(y) * abs(y) % 0.5": np.fmod(-1.0 * abs(y), 0.5),
               "log10(z) + log2(z) + exp(x)": np.log10(z) + np.log2(z) + np.exp(x),
               "((x - y) / (z + 1)) * 3.5e-2": ((x - y) / (z + 1)) * 3.5e-2}[src]
        assert out.value == pytest.approx(ref, rel=1e-15, abs=1e-300), src
