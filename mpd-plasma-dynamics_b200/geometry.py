"""Channel geometry plugins and the grid's wall profiles (host side).

``IGeometry`` / ``GeometryRegistry`` keep the reference's plugin interface
(include/igeometry.hpp:16-34, include/geometry_registry.hpp:16-34,
src/geometry_registry.cpp:15-65).  The built-in plugins restate the
reference's formulas with the same operation order and libm calls, so their
profiles match the reference bit for bit; ``sine_wall`` is new
(r1 = const, r2(z) = r2 - a sin(pi z), the converging-diverging channel of the
batched and large-grid workloads).

The device never calls a plugin: ``grid_profiles`` samples it once per axial
row and the kernels rebuild r(l, m) = (1 - m_g dy) r_in(z_l) + m_g dy r_out(z_l)
on the fly (Grid::Build, src/grid.cpp:20-42).
"""
from __future__ import annotations

import abc
import math
from typing import Callable

import numpy as np


class GeometryError(RuntimeError):
    pass


class IGeometry(abc.ABC):
    """Abstract channel geometry (include/igeometry.hpp:16-34)."""

    @abc.abstractmethod
    def RInner(self, z: float) -> float: ...

    @abc.abstractmethod
    def ROuter(self, z: float) -> float: ...

    @abc.abstractmethod
    def DrInnerDz(self, z: float) -> float: ...

    @abc.abstractmethod
    def DrOuterDz(self, z: float) -> float: ...

    @abc.abstractmethod
    def Name(self) -> str: ...


def _params(node: dict | None, defaults: dict, who: str) -> dict:
    p = dict(defaults)
    if node:
        if not isinstance(node, dict):
            raise GeometryError(f"{who}: 'params' must be a YAML map")
        for k, v in node.items():
            if k in p:
                p[k] = float(v)
    return p


class ShortCathodeCosineGeometry(IGeometry):
    """src/geometries/short_cathode_cosine.cpp:10-71."""
    DEFAULTS = dict(z_center=0.31, transition_half_width=0.015, r_inner_before=0.200,
                    r_inner_after=0.005, r_outer=0.800)

    def __init__(self, node: dict | None = None):
        p = _params(node, self.DEFAULTS, "ShortCathodeCosineGeometry")
        if p["transition_half_width"] <= 0.0:
            raise GeometryError("ShortCathodeCosineGeometry: transition_half_width must be positive")
        if p["r_outer"] <= p["r_inner_before"] or p["r_outer"] <= p["r_inner_after"]:
            raise GeometryError("ShortCathodeCosineGeometry: r_outer must be greater than both "
                                "r_inner_before and r_inner_after")
        self.p = p
        self.z_start = p["z_center"] - p["transition_half_width"]
        self.z_end = p["z_center"] + p["transition_half_width"]
        self.delta_r = p["r_inner_after"] - p["r_inner_before"]
        self.inv_width = 1.0 / (self.z_end - self.z_start)

    def RInner(self, z):
        if z < self.z_start:
            return self.p["r_inner_before"]
        if z < self.z_end:
            xi = (z - self.z_start) * self.inv_width
            return self.p["r_inner_before"] + self.delta_r * 0.5 * (1.0 - math.cos(math.pi * xi))
        return self.p["r_inner_after"]

    def ROuter(self, z):
        return self.p["r_outer"]

    def DrInnerDz(self, z):
        if z < self.z_start or z >= self.z_end:
            return 0.0
        xi = (z - self.z_start) * self.inv_width
        return self.delta_r * 0.5 * math.pi * math.sin(math.pi * xi) * self.inv_width

    def DrOuterDz(self, z):
        return 0.0

    def Name(self):
        return "short_cathode_cosine"


class ShortCathodeParabolicGeometry(IGeometry):
    """src/geometries/short_cathode_parabolic.cpp:10-92."""
    DEFAULTS = dict(z_flat_end=0.3, z_throat=0.4, z_thin_start=0.478, r_flat=0.200,
                    r_thin=0.005, r_outer=0.800)

    def __init__(self, node: dict | None = None):
        p = _params(node, self.DEFAULTS, "ShortCathodeParabolicGeometry")
        if not (p["z_flat_end"] < p["z_throat"] < p["z_thin_start"]):
            raise GeometryError("ShortCathodeParabolicGeometry: requires "
                                "z_flat_end < z_throat < z_thin_start")
        if p["r_flat"] <= p["r_thin"]:
            raise GeometryError("ShortCathodeParabolicGeometry: r_flat must be greater than r_thin")
        if p["r_outer"] <= p["r_flat"]:
            raise GeometryError("ShortCathodeParabolicGeometry: r_outer must be greater than r_flat")
        self.p = p
        dz = p["z_throat"] - p["z_flat_end"]
        self.A = p["r_flat"] / (2.0 * dz * dz)
        self.z_arc_center = 2.0 * p["z_throat"] - p["z_flat_end"]

    def RInner(self, z):
        p = self.p
        if z < p["z_flat_end"]:
            return p["r_flat"]
        if z < p["z_throat"]:
            dz = z - p["z_flat_end"]
            return p["r_flat"] - self.A * dz * dz
        if z < p["z_thin_start"]:
            dz = z - self.z_arc_center
            return self.A * dz * dz
        return p["r_thin"]

    def ROuter(self, z):
        return self.p["r_outer"]

    def DrInnerDz(self, z):
        p = self.p
        if z < p["z_flat_end"] or z >= p["z_thin_start"]:
            return 0.0
        if z < p["z_throat"]:
            return -2.0 * self.A * (z - p["z_flat_end"])
        return 2.0 * self.A * (z - self.z_arc_center)

    def DrOuterDz(self, z):
        return 0.0

    def Name(self):
        return "short_cathode_parabolic"


class VillaniMPDTGeometry(IGeometry):
    """src/geometries/villani_mpdt.cpp:10-145."""
    DEFAULTS = dict(r_cathode=0.0186, z_cathode=0.518, r_inner_after=0.0002,
                    cathode_tip_half_width=0.015, r_anode=0.100, z_anode=0.392,
                    r_outer_domain=0.200, anode_tip_half_width=0.015)

    def __init__(self, node: dict | None = None):
        p = _params(node, self.DEFAULTS, "VillaniMPDTGeometry")
        checks = [
            (p["r_cathode"] <= 0.0, "r_cathode must be positive"),
            (p["r_inner_after"] <= 0.0, "r_inner_after must be positive (> 0) to avoid a 1/r "
                                        "singularity on the axis.  Use a small value such as 1 % "
                                        "of r_cathode."),
            (p["r_inner_after"] >= p["r_cathode"], "r_inner_after must be less than r_cathode "
             "(the inner radius shrinks toward the axis beyond the cathode tip)"),
            (p["r_anode"] <= p["r_cathode"], "r_anode must be greater than r_cathode"),
            (p["r_outer_domain"] <= p["r_anode"], "r_outer_domain must be greater than r_anode"),
            (p["z_anode"] <= 0.0 or p["z_anode"] >= 1.0, "z_anode must be in the open interval (0, 1)"),
            (p["z_cathode"] <= p["z_anode"], "z_cathode must be greater than z_anode (the cathode "
             "is longer than the anode in the Villani setup)"),
            (p["z_cathode"] >= 1.0, "z_cathode must be less than 1 (the cathode tip must be inside "
             "the computational domain)"),
            (p["cathode_tip_half_width"] < 0.0, "cathode_tip_half_width must be >= 0"),
            (p["anode_tip_half_width"] < 0.0, "anode_tip_half_width must be >= 0"),
        ]
        for bad, msg in checks:
            if bad:
                raise GeometryError("VillaniMPDTGeometry: " + msg)
        self.p = p
        self.c_z_start = p["z_cathode"] - p["cathode_tip_half_width"]
        self.c_z_end = p["z_cathode"] + p["cathode_tip_half_width"]
        self.c_delta_r = p["r_inner_after"] - p["r_cathode"]
        self.c_inv_width = (1.0 / (self.c_z_end - self.c_z_start)
                            if p["cathode_tip_half_width"] > 0.0 else 0.0)
        self.a_z_start = p["z_anode"] - p["anode_tip_half_width"]
        self.a_z_end = p["z_anode"] + p["anode_tip_half_width"]
        self.a_delta_r = p["r_outer_domain"] - p["r_anode"]
        self.a_inv_width = (1.0 / (self.a_z_end - self.a_z_start)
                            if p["anode_tip_half_width"] > 0.0 else 0.0)

    @staticmethod
    def _step(z, z_s, z_e, r_before, delta_r, inv_w):
        if z < z_s:
            return r_before
        if z >= z_e:
            return r_before + delta_r
        xi = (z - z_s) * inv_w
        return r_before + delta_r * 0.5 * (1.0 - math.cos(math.pi * xi))

    @staticmethod
    def _step_deriv(z, z_s, z_e, delta_r, inv_w):
        if z < z_s or z >= z_e:
            return 0.0
        xi = (z - z_s) * inv_w
        return delta_r * 0.5 * math.pi * math.sin(math.pi * xi) * inv_w

    def RInner(self, z):
        p = self.p
        if p["cathode_tip_half_width"] <= 0.0:
            return p["r_cathode"] if z < p["z_cathode"] else p["r_inner_after"]
        return self._step(z, self.c_z_start, self.c_z_end, p["r_cathode"], self.c_delta_r,
                          self.c_inv_width)

    def ROuter(self, z):
        p = self.p
        if p["anode_tip_half_width"] <= 0.0:
            return p["r_anode"] if z < p["z_anode"] else p["r_outer_domain"]
        return self._step(z, self.a_z_start, self.a_z_end, p["r_anode"], self.a_delta_r,
                          self.a_inv_width)

    def DrInnerDz(self, z):
        if self.p["cathode_tip_half_width"] <= 0.0:
            return 0.0
        return self._step_deriv(z, self.c_z_start, self.c_z_end, self.c_delta_r, self.c_inv_width)

    def DrOuterDz(self, z):
        if self.p["anode_tip_half_width"] <= 0.0:
            return 0.0
        return self._step_deriv(z, self.a_z_start, self.a_z_end, self.a_delta_r, self.a_inv_width)

    def Name(self):
        return "villani_mpdt"


class SineWallGeometry(IGeometry):
    """Straight inner electrode r1 and outer wall r2(z) = r2 - a sin(pi z).

    New plugin (no reference counterpart) for the converging-diverging
    channel sweeps; a = 0 is the straight coaxial channel.
    """
    DEFAULTS = dict(r1=0.2, r2=0.8, a=0.0)

    def __init__(self, node: dict | None = None):
        p = _params(node, self.DEFAULTS, "SineWallGeometry")
        if p["r1"] <= 0.0:
            raise GeometryError("SineWallGeometry: r1 must be positive")
        if p["r2"] - abs(p["a"]) <= p["r1"]:
            raise GeometryError("SineWallGeometry: the outer wall must stay above r1 "
                                "(need r2 - |a| > r1)")
        self.p = p

    def RInner(self, z):
        return self.p["r1"]

    def ROuter(self, z):
        return self.p["r2"] - self.p["a"] * math.sin(math.pi * z)

    def DrInnerDz(self, z):
        return 0.0

    def DrOuterDz(self, z):
        return -self.p["a"] * math.pi * math.cos(math.pi * z)

    def Name(self):
        return "sine_wall"


class GeometryRegistry:
    """Name -> factory singleton (src/geometry_registry.cpp:15-34)."""
    _instance: "GeometryRegistry | None" = None

    def __init__(self):
        self.factories: dict[str, Callable[[dict | None], IGeometry]] = {}

    @classmethod
    def Instance(cls) -> "GeometryRegistry":
        if cls._instance is None:
            cls._instance = cls()
        return cls._instance

    def RegisterGeometry(self, name: str, factory) -> None:
        self.factories.setdefault(name, factory)

    def Create(self, type_: str, params: dict | None) -> IGeometry:
        if type_ not in self.factories:
            raise GeometryError(
                f"GeometryRegistry: unknown geometry type '{type_}'.\n"
                "  Did you forget to call register_all_geometries(), or mistype the name "
                "in config.yaml?")
        return self.factories[type_](params)


def register_all_geometries() -> None:
    """RegisterAllGeometries (src/geometry_registry.cpp:40-65) + sine_wall."""
    reg = GeometryRegistry.Instance()
    reg.RegisterGeometry("short_cathode_parabolic", ShortCathodeParabolicGeometry)
    reg.RegisterGeometry("short_cathode_cosine", ShortCathodeCosineGeometry)
    reg.RegisterGeometry("villani_mpdt", VillaniMPDTGeometry)
    reg.RegisterGeometry("sine_wall", SineWallGeometry)


register_all_geometries()


class Grid:
    """Host view of Grid (include/grid.hpp:20-47) for one rank owning the domain.

    ``rin/rout/drin/drout`` hold the plugin sampled at z = (l-1) dz for
    l = 0..L_max+1 (the row profiles the device consumes); ``r``/``r_z`` are
    the full planes, built with Grid::Build's arithmetic, for host-side use.
    """

    def __init__(self, cfg, geom: IGeometry):
        L, M = cfg.L_max, cfg.M_max
        n = L + 2
        self.cfg = cfg
        self.geom = geom
        self.rin = np.empty(n)
        self.rout = np.empty(n)
        self.drin = np.empty(n)
        self.drout = np.empty(n)
        for l in range(n):
            z = (l - 1) * cfg.dz
            self.rin[l] = geom.RInner(z)
            self.rout[l] = geom.ROuter(z)
            self.drin[l] = geom.DrInnerDz(z)
            self.drout[l] = geom.DrOuterDz(z)
        self.R = self.rout - self.rin
        self.dr = self.R / M
        self.r_0 = (geom.RInner(0.0) + geom.ROuter(0.0)) / 2.0
        frac = np.arange(-1, M + 2, dtype=np.float64) * cfg.dy
        self.r = (1.0 - frac)[None, :] * self.rin[:, None] + frac[None, :] * self.rout[:, None]
        self.r_z = (1.0 - frac)[None, :] * self.drin[:, None] + frac[None, :] * self.drout[:, None]

    def profiles(self):
        return self.rin, self.rout, self.drin, self.drout
