"""ctypes bindings of the CPU oracle — TEST INFRASTRUCTURE ONLY.

Two interchangeable back ends with the same methods:

* ``Port``  — ``oracle/_build/libmpd_oracle.so``, the plain-C restatement in
  ``oracle/mpd_oracle.c`` (always buildable: ``make -C oracle port``).
* ``Ref``   — ``oracle/_ref/libmpd_ref.so``, the reference's own translation
  units compiled with the shims in ``oracle/shim`` (``make -C oracle ref``,
  needs the reference sources; the built file travels with the tree).

A *case* is a plain dict (see ``case_arrays``) holding the hot path's inputs:
grid sizes, physics constants, wall profiles per row, the 10 initial physical
planes and the boundary segments per face.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
PORT_SO = HERE / "_build" / "libmpd_oracle.so"
REF_SO = HERE / "_ref" / "libmpd_ref.so"

FACES = {"l_lo": 0, "l_hi": 1, "m_lo": 2, "m_hi": 3}
# BCSegmentConfig field order (include/config.hpp:82-92 of the reference)
COND_FIELDS = ("rho", "v_z", "v_r", "v_phi", "e", "H_z", "H_r", "H_phi")
COND_TYPES = {"neumann": 0, "dirichlet": 1, "expr": 2, "axis_lf": 3}
# Fields physical members (include/fields.hpp:35-37)
PHYS_FIELDS = ("rho", "v_z", "v_r", "v_phi", "e", "p", "P", "H_z", "H_r", "H_phi")

_DP = C.POINTER(C.c_double)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_DP)


def build_port() -> pathlib.Path:
    if not PORT_SO.exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "port"], check=True)
    return PORT_SO


def ref_available() -> bool:
    return REF_SO.exists()


def _load(path: pathlib.Path, prefix: str) -> C.CDLL:
    lib = C.CDLL(str(path))
    vp = C.c_void_p
    p = prefix
    getattr(lib, f"{p}_new").restype = vp
    getattr(lib, f"{p}_new").argtypes = [C.c_int, C.c_int, _DP, _DP, _DP, _DP, _DP, _DP, C.c_int]
    getattr(lib, f"{p}_free").argtypes = [vp]
    getattr(lib, f"{p}_advance").argtypes = [vp, C.c_double]
    for name in ("max_wave_speed", "solution_change", "radial_symmetry"):
        f = getattr(lib, f"{p}_{name}")
        f.argtypes = [vp]
        f.restype = C.c_double
    f = getattr(lib, f"{p}_compute_dt")
    f.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]
    f.restype = C.c_double
    getattr(lib, f"{p}_save_prev").argtypes = [vp]
    getattr(lib, f"{p}_integrals").argtypes = [vp, _DP]
    getattr(lib, f"{p}_outlet").argtypes = [vp, _DP, _DP]
    getattr(lib, f"{p}_get").argtypes = [vp, C.c_int, _DP]
    getattr(lib, f"{p}_run").argtypes = [vp, _DP, _DP]
    return lib


class _Backend:
    prefix = ""
    so: pathlib.Path

    def __init__(self, case: dict):
        self.lib = _load(self.so, self.prefix)
        self.case = case
        self.L, self.M = case["L"], case["M"]
        self.rows, self.cols = self.L + 2, self.M + 3
        params = np.array([case["gamma"], case["beta"], case["H_z0"], case["dz"], case["dy"],
                           case["r_0"]], dtype=np.float64)
        prof = [np.ascontiguousarray(case[k], dtype=np.float64) for k in ("rin", "rout", "drin", "drout")]
        phys = np.ascontiguousarray(case["phys"], dtype=np.float64)
        assert phys.shape == (10, self.rows, self.cols)
        self.h = getattr(self.lib, f"{self.prefix}_new")(
            self.L, self.M, _dp(params), *(_dp(a) for a in prof), _dp(phys),
            1 if case.get("with_prev") else 0)
        for face, segs in case["bc"].items():
            for seg in segs:
                self._add_segment(FACES[face], seg)
        self._finalize()

    # -- segments -----------------------------------------------------------
    def _seg_arrays(self, seg: dict):
        types = (C.c_int * 8)()
        values = (C.c_double * 8)()
        exprs = (C.c_char_p * 8)()
        for k, name in enumerate(COND_FIELDS):
            kind, val = seg.get(name, ("neumann", 0.0))
            types[k] = COND_TYPES[kind]
            if kind == "expr":
                exprs[k] = str(val).encode()
                values[k] = 0.0
            else:
                values[k] = float(val)
        lo, hi = seg.get("range", (-1, -1))
        return int(lo), int(hi), types, values, exprs

    def _add_segment(self, face: int, seg: dict):  # pragma: no cover - overridden
        raise NotImplementedError

    def _finalize(self):
        pass

    # -- operations ---------------------------------------------------------
    def advance(self, dt: float):
        getattr(self.lib, f"{self.prefix}_advance")(self.h, float(dt))

    def max_wave_speed(self) -> float:
        return getattr(self.lib, f"{self.prefix}_max_wave_speed")(self.h)

    def compute_dt(self, cfl, growth, dt_min, dt_max, dt_current) -> float:
        return getattr(self.lib, f"{self.prefix}_compute_dt")(self.h, cfl, growth, dt_min, dt_max,
                                                             dt_current)

    def solution_change(self) -> float:
        return getattr(self.lib, f"{self.prefix}_solution_change")(self.h)

    def save_prev(self):
        getattr(self.lib, f"{self.prefix}_save_prev")(self.h)

    def radial_symmetry(self) -> float:
        return getattr(self.lib, f"{self.prefix}_radial_symmetry")(self.h)

    def integrals(self) -> np.ndarray:
        out = np.zeros(7)
        getattr(self.lib, f"{self.prefix}_integrals")(self.h, _dp(out))
        return out

    def outlet(self):
        a, b = C.c_double(), C.c_double()
        getattr(self.lib, f"{self.prefix}_outlet")(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def get(self, which: int) -> np.ndarray:
        out = np.empty((self.rows, self.cols))
        getattr(self.lib, f"{self.prefix}_get")(self.h, int(which), _dp(out))
        return out

    def conserved(self) -> np.ndarray:
        return np.stack([self.get(k) for k in range(8)])

    def physical(self) -> np.ndarray:
        return np.stack([self.get(8 + k) for k in range(10)])

    def run(self, T, dt0, adaptive, cfl, growth, dt_min, dt_max, conv_threshold=0.0,
            check_frequency=100, max_steps=1 << 40):
        run = np.array([T, dt0, 1.0 if adaptive else 0.0, cfl, growth, dt_min, dt_max,
                        conv_threshold, check_frequency, max_steps], dtype=np.float64)
        out = np.zeros(5)
        getattr(self.lib, f"{self.prefix}_run")(self.h, _dp(run), _dp(out))
        return dict(steps=int(out[0]), t=out[1], dt=out[2], converged=bool(out[3]), change=out[4])

    def close(self):
        if getattr(self, "h", None):
            getattr(self.lib, f"{self.prefix}_free")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Port(_Backend):
    prefix = "mo"
    so = PORT_SO

    def __init__(self, case: dict):
        build_port()
        super().__init__(case)

    def _add_segment(self, face, seg):
        lo, hi, types, values, exprs = self._seg_arrays(seg)
        self.lib.mo_add_segment.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int,
                                            C.POINTER(C.c_int), _DP, C.POINTER(C.c_char_p),
                                            C.c_char_p, C.c_int]
        err = C.create_string_buffer(512)
        rc = self.lib.mo_add_segment(self.h, face, lo, hi, types, values, exprs, err, 512)
        if rc != 0:
            raise RuntimeError(err.value.decode())


class Ref(_Backend):
    prefix = "ref"
    so = REF_SO

    def _add_segment(self, face, seg):
        lo, hi, types, values, exprs = self._seg_arrays(seg)
        self.lib.ref_add_segment.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int,
                                             C.POINTER(C.c_int), _DP, C.POINTER(C.c_char_p)]
        self.lib.ref_add_segment(self.h, face, lo, hi, types, values, exprs)

    def _finalize(self):
        self.lib.ref_finalize.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
        err = C.create_string_buffer(1024)
        if self.lib.ref_finalize(self.h, err, 1024) != 0:
            raise RuntimeError(err.value.decode())

    def grid_r0(self) -> float:
        self.lib.ref_grid_r0.argtypes = [C.c_void_p]
        self.lib.ref_grid_r0.restype = C.c_double
        return self.lib.ref_grid_r0(self.h)


def _kv(d: dict):
    keys = (C.c_char_p * max(len(d), 1))(*[k.encode() for k in d])
    vals = (C.c_char_p * max(len(d), 1))(*[str(v).encode() for v in d.values()])
    return keys, vals, len(d)


def ref_geometry_profile(gtype: str, params: dict, L: int, dz: float):
    """Sample the reference's own IGeometry plugin at z = (l-1)*dz."""
    lib = C.CDLL(str(REF_SO))
    n = L + 2
    out = [np.zeros(n) for _ in range(4)]
    keys, vals, nkv = _kv(params)
    err = C.create_string_buffer(512)
    lib.ref_geometry_profile.argtypes = [C.c_char_p, C.POINTER(C.c_char_p), C.POINTER(C.c_char_p),
                                         C.c_int, C.c_int, C.c_double, _DP, _DP, _DP, _DP,
                                         C.c_char_p, C.c_int]
    rc = lib.ref_geometry_profile(gtype.encode(), keys, vals, nkv, L, dz, *(_dp(a) for a in out),
                                  err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return out


def ref_expression_ic(ic: dict, L: int, M: int, params, rin, rout, drin, drout) -> np.ndarray:
    """The reference's ExpressionIC evaluated over a Grid built from the profiles."""
    lib = C.CDLL(str(REF_SO))
    keys, vals, nkv = _kv(ic)
    p = np.ascontiguousarray(params, dtype=np.float64)
    out = np.zeros((10, L + 2, M + 3))
    err = C.create_string_buffer(512)
    lib.ref_expression_ic.argtypes = [C.POINTER(C.c_char_p), C.POINTER(C.c_char_p), C.c_int,
                                      C.c_int, C.c_int, _DP, _DP, _DP, _DP, _DP, _DP, C.c_char_p,
                                      C.c_int]
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (rin, rout, drin, drout)]
    rc = lib.ref_expression_ic(keys, vals, nkv, L, M, _dp(p), *(_dp(a) for a in arrs), _dp(out),
                               err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return out
