"""Simulation configuration: the reference's ``SimConfig`` and its YAML schema.

Mirrors ``include/config.hpp:119-176`` (field names and defaults) and the
loader of ``src/config.cpp:52-384`` (the per-field boundary grammar, segment
ranges, removed-preset errors).  Scalars are read as their source text (YAML
"base" loader, as yaml-cpp keeps them), so expression strings and numbers
reach the solver exactly as written.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Any

import yaml

from . import _native as N

# FieldCondType (include/field_condition.hpp:92-97)
NEUMANN, DIRICHLET, EXPRESSION, AXIS_LF = "neumann", "dirichlet", "expression", "axis_lf"
_TYPE_CODE = {NEUMANN: N.NEUMANN, DIRICHLET: N.DIRICHLET, EXPRESSION: N.EXPRESSION,
              AXIS_LF: N.AXIS_LF}
SEGMENT_FIELDS = ("rho", "v_z", "v_r", "v_phi", "e", "H_z", "H_r", "H_phi")


class ConfigError(RuntimeError):
    """A malformed configuration (the reference throws std::runtime_error)."""


@dataclasses.dataclass
class FieldCond:
    """Condition for one physical field at one segment (include/field_condition.hpp:100-105)."""
    type: str = NEUMANN
    value: float = 0.0
    expr_str: str = ""


@dataclasses.dataclass
class BCSegmentConfig:
    """One contiguous segment of a face (include/config.hpp:82-95)."""
    global_lo: int = -1
    global_hi: int = -1
    rho: FieldCond = dataclasses.field(default_factory=FieldCond)
    v_z: FieldCond = dataclasses.field(default_factory=FieldCond)
    v_r: FieldCond = dataclasses.field(default_factory=FieldCond)
    v_phi: FieldCond = dataclasses.field(default_factory=FieldCond)
    e: FieldCond = dataclasses.field(default_factory=FieldCond)
    H_z: FieldCond = dataclasses.field(default_factory=FieldCond)
    H_r: FieldCond = dataclasses.field(default_factory=FieldCond)
    H_phi: FieldCond = dataclasses.field(default_factory=FieldCond)


@dataclasses.dataclass
class BCFaceConfig:
    segments: list = dataclasses.field(default_factory=list)


@dataclasses.dataclass
class GeometryConfig:
    type: str = "short_cathode_cosine"
    params: dict = dataclasses.field(default_factory=dict)


@dataclasses.dataclass
class ICConfig:
    vtk_file: str = ""
    params: dict = dataclasses.field(default_factory=dict)


@dataclasses.dataclass
class SimConfig:
    """All tuneable parameters (include/config.hpp:119-176, same defaults)."""
    gamma: float = 1.67
    beta: float = 0.05
    H_z0: float = 0.25
    T: float = 0.5
    dt: float = 0.000025
    adaptive_dt: bool = False
    cfl_number: float = 0.5
    dt_growth_factor: float = 1.1
    dt_min: float = 1.0e-9
    dt_max: float = 1.0e-3
    L_max: int = 800
    M_max: int = 400
    convergence_threshold: float = 0.0
    check_frequency: int = 100
    output_dir: str = "output"
    run_name: str = "run"
    vtk_step: int = 100
    openmp_threads: int = 0
    mpi_dims_l: int = 0
    mpi_dims_m: int = 0
    geometry: GeometryConfig = dataclasses.field(default_factory=GeometryConfig)
    initial_conditions: ICConfig = dataclasses.field(default_factory=ICConfig)
    bc_l_lo: BCFaceConfig = dataclasses.field(default_factory=BCFaceConfig)
    bc_l_hi: BCFaceConfig = dataclasses.field(default_factory=BCFaceConfig)
    bc_m_lo: BCFaceConfig = dataclasses.field(default_factory=BCFaceConfig)
    bc_m_hi: BCFaceConfig = dataclasses.field(default_factory=BCFaceConfig)
    dz: float = 0.0
    dy: float = 0.0

    def __post_init__(self):
        self.init()

    def init(self) -> None:
        """Derived quantities (SimConfig::Init, src/config.cpp:15-18)."""
        self.dz = 1.0 / self.L_max
        self.dy = 1.0 / self.M_max

    @classmethod
    def load(cls, path: str) -> "SimConfig":
        """SimConfig::Load (src/config.cpp:261-384) from a YAML file."""
        try:
            with open(path, "r", encoding="utf-8") as fh:
                text = fh.read()
        except OSError as exc:
            raise ConfigError(f"Failed to load config file '{path}': {exc}") from exc
        return cls.from_yaml(text)

    @classmethod
    def from_yaml(cls, text: str) -> "SimConfig":
        try:
            root = yaml.load(text, Loader=yaml.BaseLoader) or {}
        except yaml.YAMLError as exc:
            raise ConfigError(f"Failed to parse config: {exc}") from exc
        cfg = cls()
        cfg.apply(root)
        return cfg

    def apply(self, root: dict) -> None:
        def sect(name):
            n = root.get(name)
            return n if isinstance(n, dict) else None

        if (n := sect("physics")) is not None:
            _set(self, n, "gamma", float)
            _set(self, n, "beta", float)
            _set(self, n, "H_z0", float)
        if (n := sect("time")) is not None:
            _set(self, n, "T", float)
            _set(self, n, "dt", float)
        if (n := sect("adaptive_dt")) is not None:
            _set(self, n, "adaptive_dt", _as_bool, key="enabled")
            _set(self, n, "cfl_number", float)
            _set(self, n, "dt_growth_factor", float, key="growth_factor")
            _set(self, n, "dt_min", float)
            _set(self, n, "dt_max", float)
        if (n := sect("grid")) is not None:
            _set(self, n, "L_max", int)
            _set(self, n, "M_max", int)
        if (n := sect("convergence")) is not None:
            _set(self, n, "convergence_threshold", float, key="threshold")
            _set(self, n, "check_frequency", int)
        if (n := sect("output")) is not None:
            _set(self, n, "output_dir", str, key="directory")
            _set(self, n, "run_name", str)
            _set(self, n, "vtk_step", int)
        if (n := sect("parallel")) is not None:
            _set(self, n, "openmp_threads", int)
            _set(self, n, "mpi_dims_l", int)
            _set(self, n, "mpi_dims_m", int)
        if (n := sect("geometry")) is not None:
            if "type" in n:
                self.geometry.type = str(n["type"])
            if "params" in n and n["params"] is not None:
                if not isinstance(n["params"], dict):
                    raise ConfigError("config: 'geometry.params' must be a YAML map")
                self.geometry.params = dict(n["params"])
        if "initial_conditions" in root and root["initial_conditions"] is not None:
            self._load_ic(root["initial_conditions"])
        if (n := sect("boundary_conditions")) is not None:
            for face in ("l_lo", "l_hi", "m_lo", "m_hi"):
                if face in n:
                    setattr(self, f"bc_{face}", parse_face(n[face]))
        self.init()

    def _load_ic(self, n: Any) -> None:
        if not isinstance(n, dict):
            raise ConfigError("config: 'initial_conditions' must be a YAML map")
        if "type" in n:
            raise ConfigError(
                "config: 'initial_conditions.type' is no longer supported — "
                "ExpressionIC is always used.\n"
                "  Remove the 'type' key.  Field expressions now live directly\n"
                "  under 'initial_conditions:', not under 'initial_conditions.params:'.")
        if "params" in n:
            raise ConfigError(
                "config: 'initial_conditions.params' is no longer supported.\n"
                "  Move field expressions one level up, directly under 'initial_conditions:'.")
        if "vtk_file" in n:
            if not isinstance(n["vtk_file"], str):
                raise ConfigError("config: 'initial_conditions.vtk_file' must be a scalar "
                                  "file-path string.")
            self.initial_conditions.vtk_file = n["vtk_file"]
        else:
            self.initial_conditions.params = dict(n)

    # -- C ABI view ------------------------------------------------------------
    def faces(self):
        """Faces in FaceBC::Face order (L_LO, L_HI, M_LO, M_HI)."""
        return (self.bc_l_lo, self.bc_l_hi, self.bc_m_lo, self.bc_m_hi)


def _as_bool(s: str) -> bool:
    v = str(s).strip().lower()
    if v in ("true", "yes", "on", "y"):
        return True
    if v in ("false", "no", "off", "n"):
        return False
    raise ConfigError(f"config: bad boolean '{s}'")


def _set(obj, node: dict, attr: str, conv, key: str | None = None) -> None:
    key = key or attr
    if key in node and node[key] is not None:
        try:
            setattr(obj, attr, conv(node[key]))
        except (TypeError, ValueError) as exc:
            raise ConfigError(f"config: bad value for '{key}': {node[key]!r}") from exc


_WALL_TANGENT_MSG = (
    "config: 'wall_tangent' is no longer a built-in preset.\n"
    "  Replace it with an expression that encodes the wall-tangent\n"
    "  condition explicitly:\n"
    "\n"
    "    On M_LO (inner wall) — uses interior-neighbour slope:\n"
    "      v_r: \"v_z_nb * r_z_nb\"\n"
    "      H_r: \"H_z_nb * r_z_nb\"\n"
    "\n"
    "    On M_HI (outer wall) — uses wall-cell slope:\n"
    "      v_r: \"v_z * r_z\"\n"
    "      H_r: \"H_z * r_z\"\n"
    "\n"
    "  Note: 'v_z' and 'H_z' here refer to the wall-cell values\n"
    "  (already evaluated earlier in the same cell's update).\n"
    "  'v_z_nb' / 'H_z_nb' refer to the interior-neighbour cell.")
_HPHI_MSG = ("config: 'hphi_r0_over_r' is no longer a built-in preset.\n"
             "  Replace it with the equivalent expression:\n"
             "\n"
             "    H_phi: \"r_0 / r\"\n"
             "\n"
             "  This enforces H_phi * r = r_0 = const (free-vortex / no-current\n"
             "  azimuthal field profile).")


def parse_field_cond(n: Any) -> FieldCond:
    """ParseFieldCond (src/config.cpp:52-202)."""
    if n is None:
        return FieldCond()
    if isinstance(n, str):
        if n == "neumann":
            return FieldCond(NEUMANN)
        if n == "dirichlet":
            return FieldCond(DIRICHLET, 0.0)
        if n == "axis_lf":
            return FieldCond(AXIS_LF)
        if n == "wall_tangent":
            raise ConfigError(_WALL_TANGENT_MSG)
        if n == "hphi_r0_over_r":
            raise ConfigError(_HPHI_MSG)
        return FieldCond(EXPRESSION, 0.0, n)
    if isinstance(n, dict):
        if "neumann" in n:
            v = n["neumann"]
            if not isinstance(v, str):
                raise ConfigError("config: 'neumann' offset must be a scalar number "
                                  "(e.g. { neumann: 0.5 })")
            return FieldCond(NEUMANN, float(v))
        if "dirichlet" in n:
            v = n["dirichlet"]
            if not isinstance(v, str):
                raise ConfigError("config: 'dirichlet' value must be a scalar number "
                                  "(e.g. { dirichlet: 1.0 })")
            return FieldCond(DIRICHLET, float(v))
        if "expr" in n and "type" not in n:
            v = n["expr"]
            if not isinstance(v, str):
                raise ConfigError("config: 'expr' value must be a scalar expression string "
                                  "(e.g. { expr: \"v_z * r_z\" })")
            return FieldCond(EXPRESSION, 0.0, v)
        if "type" in n:
            t = str(n["type"])
            if t == "neumann":
                off = 0.0
                if "gradient" in n:
                    off = float(n["gradient"])
                elif "value" in n:
                    off = float(n["value"])
                return FieldCond(NEUMANN, off)
            if t == "dirichlet":
                return FieldCond(DIRICHLET, float(n["value"]) if "value" in n else 0.0)
            if t == "axis_lf":
                return FieldCond(AXIS_LF)
            if t in ("expression", "expr"):
                if "expr" not in n:
                    raise ConfigError(
                        "config: { type: expression } requires an 'expr' key "
                        "containing the formula string\n"
                        "  Example: { type: expression, expr: \"v_z * r_z\" }")
                return FieldCond(EXPRESSION, 0.0, str(n["expr"]))
            if t == "wall_tangent":
                raise ConfigError("config: { type: wall_tangent } is no longer supported.\n"
                                  "  See the 'wall_tangent' migration note above.")
            if t == "hphi_r0_over_r":
                raise ConfigError("config: { type: hphi_r0_over_r } is no longer supported.\n"
                                  "  Use: H_phi: \"r_0 / r\"")
            raise ConfigError(
                f"config: unknown field condition type '{t}'.\n"
                "  Valid types: neumann, dirichlet, expression, axis_lf.\n"
                "  For an expression use a quoted string directly:  v_r: \"v_z * r_z\"")
        raise ConfigError("config: field condition map must contain one of: 'neumann', "
                          "'dirichlet', 'expr', or 'type'")
    raise ConfigError(
        "config: field condition must be:\n"
        "  - a keyword scalar:           neumann / dirichlet / axis_lf\n"
        "  - a quoted expression string: \"v_z * r_z\"\n"
        "  - a short map:                { dirichlet: 1.0 } / { neumann: 0.5 } / { expr: \"...\" }\n"
        "  - a verbose map:              { type: dirichlet, value: 1.0 }")


def parse_face(node: Any) -> BCFaceConfig:
    """ParseFace (src/config.cpp:212-255)."""
    face = BCFaceConfig()
    if node is None:
        return face
    if not isinstance(node, list):
        raise ConfigError("config: each boundary-condition face must be a YAML sequence "
                          "of segment maps")
    for item in node:
        if not isinstance(item, dict):
            raise ConfigError("config: each BC segment must be a YAML map")
        seg = BCSegmentConfig()
        if "range" in item:
            rng = item["range"]
            if not isinstance(rng, list) or len(rng) != 2:
                raise ConfigError(
                    "config: BC segment 'range' must be a two-element sequence "
                    "[global_lo, global_hi]  (use -1 as sentinel for face start/end)")
            seg.global_lo, seg.global_hi = int(rng[0]), int(rng[1])
        for name in SEGMENT_FIELDS:
            setattr(seg, name, parse_field_cond(item.get(name)))
        face.segments.append(seg)
    return face


def segment(range_=(-1, -1), **conds) -> BCSegmentConfig:
    """Convenience builder: ``segment((0, 235), v_r="v_z_nb * r_z_nb", rho=("dirichlet", 0.1))``.

    A string value is parsed with the YAML grammar (keyword or expression), a
    ``(kind, value)`` pair gives the kind explicitly.
    """
    seg = BCSegmentConfig(int(range_[0]), int(range_[1]))
    for name, v in conds.items():
        if name not in SEGMENT_FIELDS:
            raise ConfigError(f"unknown field '{name}'")
        if isinstance(v, FieldCond):
            fc = v
        elif isinstance(v, tuple):
            kind, val = v
            kind = EXPRESSION if kind in ("expr", EXPRESSION) else kind
            fc = FieldCond(kind, 0.0, val) if kind == EXPRESSION else FieldCond(kind, float(val))
        else:
            fc = parse_field_cond(str(v))
        setattr(seg, name, fc)
    return seg


class CConfig:
    """Keeps the ctypes mpd_config and everything it points to alive."""

    def __init__(self, cfg: SimConfig, r_0: float, precision: int, with_prev: bool):
        self._keep = []
        c = N.Config()
        c.gamma, c.beta, c.H_z0 = cfg.gamma, cfg.beta, cfg.H_z0
        c.L_max, c.M_max = cfg.L_max, cfg.M_max
        c.dz, c.dy, c.r_0 = cfg.dz, cfg.dy, r_0
        for f, face in enumerate(cfg.faces()):
            segs = (N.BCSegment * max(len(face.segments), 1))()
            for i, s in enumerate(face.segments):
                segs[i].global_lo, segs[i].global_hi = s.global_lo, s.global_hi
                for name in SEGMENT_FIELDS:
                    fc: FieldCond = getattr(s, name)
                    dst = getattr(segs[i], name)
                    dst.type = _TYPE_CODE[fc.type]
                    dst.value = float(fc.value)
                    if fc.type == EXPRESSION:
                        b = fc.expr_str.encode()
                        self._keep.append(b)
                        dst.expr = b
            self._keep.append(segs)
            c.n_segments[f] = len(face.segments)
            c.segments[f] = segs
        c.precision = precision
        c.with_prev = 1 if with_prev else 0
        self.c = c

    @property
    def ptr(self):
        import ctypes
        return ctypes.byref(self.c)


def isfinite_cfg(cfg: SimConfig) -> bool:
    return all(math.isfinite(v) for v in (cfg.gamma, cfg.beta, cfg.H_z0, cfg.dz, cfg.dy))
