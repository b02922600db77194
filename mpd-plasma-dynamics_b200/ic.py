"""Initial conditions (IInitialCondition, include/iinitial_condition.hpp:21-39).

``Apply`` returns the 10 physical planes (Fields member order: rho, v_z, v_r,
v_phi, e, p, P, H_z, H_r, H_phi) on the reference's (L_max+2) x (M_max+3)
index space with zero ghosts; ``GpuSolver`` uploads them and builds the
conserved state on the device (Fields::InitConservative).
"""
from __future__ import annotations

import abc
import ctypes as C

import numpy as np

from . import _native as N
from .config import CConfig, ConfigError, SimConfig

IC_FIELDS = ("rho", "v_z", "v_r", "v_phi", "H_z", "H_r", "H_phi", "e")  # evaluation order


class IInitialCondition(abc.ABC):
    @abc.abstractmethod
    def Apply(self, grid, cfg: SimConfig) -> np.ndarray: ...

    @abc.abstractmethod
    def Name(self) -> str: ...


class ExpressionIC(IInitialCondition):
    """Per-cell expression IC (src/ics/expression_ic.cpp:255-324).

    ``params`` is the ``initial_conditions`` YAML map: one scalar expression
    (or number) per field, optional ``vars`` of user constants.  Missing
    fields take the reference's defaults.  Evaluated on the host by the
    library's expression compiler: on the device, one thread per cell, when
    ``GpuSolver`` is given the IC itself (the same bits), or as one
    sequential host sweep (``Apply``), which also reproduces expressions that
    read a field evaluated after them.
    """

    def __init__(self, params: dict | None = None):
        params = params or {}
        self.exprs = {}
        for name in IC_FIELDS:
            v = params.get(name)
            if v is None:
                continue
            if isinstance(v, dict):
                raise ConfigError(
                    f"ExpressionIC: field '{name}' must be a scalar expression string or a plain "
                    "number (e.g. rho: 1.0  or  H_r: \"H_z * r_z\").\n"
                    "  Map-form entries are not supported by the expression IC.")
            self.exprs[name] = str(v)
        self.vars = {}
        uv = params.get("vars")
        if uv is not None:
            if not isinstance(uv, dict):
                raise ConfigError("ExpressionIC: 'vars' must be a YAML map of name: value pairs.")
            for k, v in uv.items():
                if isinstance(v, (dict, list)):
                    raise ConfigError(f"ExpressionIC: value for var '{k}' must be a scalar number.")
                self.vars[str(k)] = float(v)

    def _c_args(self):
        exprs = (C.c_char_p * 8)(*[self.exprs[n].encode() if n in self.exprs else None
                                   for n in IC_FIELDS])
        names = (C.c_char_p * max(len(self.vars), 1))(*[k.encode() for k in self.vars])
        vals = np.array(list(self.vars.values()) or [0.0], dtype=np.float64)
        return exprs, len(self.vars), names, vals

    def Apply(self, grid, cfg: SimConfig) -> np.ndarray:
        """The 10 physical planes on the host (one sequential sweep)."""
        lib = N.load()
        cc = CConfig(cfg, grid.r_0, N.PRECISION_EXACT, False)
        keep = [np.ascontiguousarray(a) for a in grid.profiles()]
        geo = N.Geometry(*(a.ctypes.data_as(N.DP) for a in keep))
        exprs, n_vars, names, vals = self._c_args()
        out = np.zeros((10, cfg.L_max + 2, cfg.M_max + 3))
        rc = lib.mpd_expression_ic(cc.ptr, C.byref(geo), exprs, n_vars, names,
                                   vals.ctypes.data_as(N.DP), out.ctypes.data_as(N.DP))
        N.check(rc, lib)
        return out

    def ApplyDevice(self, lib, handle) -> int:
        """Evaluate into a solver's device state (mpd_set_expression_ic); the
        status, MPD_ERR_UNSUPPORTED_IC for expressions that read a field
        evaluated after them."""
        exprs, n_vars, names, vals = self._c_args()
        return lib.mpd_set_expression_ic(handle, exprs, n_vars, names, vals.ctypes.data_as(N.DP))

    def Name(self):
        return "expression"


class ArrayIC(IInitialCondition):
    """Physical planes given directly (restarts, warm starts, tests)."""

    def __init__(self, phys10: np.ndarray):
        self.phys = np.ascontiguousarray(phys10, dtype=np.float64)

    def Apply(self, grid, cfg):
        shape = (10, cfg.L_max + 2, cfg.M_max + 3)
        if self.phys.shape != shape:
            raise ValueError(f"ArrayIC: planes have shape {self.phys.shape}, expected {shape}")
        out = np.zeros(shape)
        out[:, 1:-1, 1:-1] = self.phys[:, 1:-1, 1:-1]
        return out

    def Name(self):
        return "array"


def derived_pressures(phys: np.ndarray, gamma: float) -> None:
    """Fill p and P from the primitives in place (ExpressionIC::Apply, lines 316-321)."""
    rho, e = phys[0], phys[4]
    Hz, Hr, Hphi = phys[7], phys[8], phys[9]
    phys[5] = (gamma - 1.0) * rho * e
    phys[6] = phys[5] + 0.5 * (Hz * Hz + Hr * Hr + Hphi * Hphi)
