"""ctypes bindings of the C ABI in ``include/mpd_b200.h``.

The structures mirror the header field for field.  ``load()`` opens the
in-tree ``libmpd_b200.so`` and fails loudly when it is missing: there is no
host fallback for the solver.
"""
from __future__ import annotations

import ctypes as C
import pathlib

PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG / "libmpd_b200.so"
EMU_PATH = PKG / "libmpd_emu.so"

MPD_OK = 0
MPD_ERR_INVALID = 1
MPD_ERR_CUDA = 2
MPD_ERR_NOMEM = 3
MPD_ERR_UNSUPPORTED_BC = 4
MPD_ERR_EXPR = 5
MPD_ERR_NONFINITE = 6
MPD_ERR_TIMEOUT = 7
MPD_ERR_NO_DEVICE = 8
MPD_ERR_UNSUPPORTED_IC = 9

STATUS_NAMES = {
    0: "MPD_OK", 1: "MPD_ERR_INVALID", 2: "MPD_ERR_CUDA", 3: "MPD_ERR_NOMEM",
    4: "MPD_ERR_UNSUPPORTED_BC", 5: "MPD_ERR_EXPR", 6: "MPD_ERR_NONFINITE",
    7: "MPD_ERR_TIMEOUT", 8: "MPD_ERR_NO_DEVICE", 9: "MPD_ERR_UNSUPPORTED_IC",
}

FACE_L_LO, FACE_L_HI, FACE_M_LO, FACE_M_HI = 0, 1, 2, 3
NEUMANN, DIRICHLET, EXPRESSION, AXIS_LF = 0, 1, 2, 3
ENGINE_AUTO, ENGINE_GRAPH, ENGINE_PERSISTENT = 0, 1, 2
PRECISION_EXACT, PRECISION_FAST = 0, 1
KERNEL_INTERIOR, KERNEL_RESIDUAL, KERNEL_INTERIOR_PAIR = 0, 1, 2
PHYS_FIELDS = ("rho", "v_z", "v_r", "v_phi", "e", "p", "P", "H_z", "H_r", "H_phi")

DP = C.POINTER(C.c_double)


class FieldCond(C.Structure):
    _fields_ = [("type", C.c_int), ("value", C.c_double), ("expr", C.c_char_p)]


class BCSegment(C.Structure):
    _fields_ = [("global_lo", C.c_int), ("global_hi", C.c_int),
                ("rho", FieldCond), ("v_z", FieldCond), ("v_r", FieldCond),
                ("v_phi", FieldCond), ("e", FieldCond), ("H_z", FieldCond),
                ("H_r", FieldCond), ("H_phi", FieldCond)]


class Config(C.Structure):
    _fields_ = [("gamma", C.c_double), ("beta", C.c_double), ("H_z0", C.c_double),
                ("L_max", C.c_int), ("M_max", C.c_int),
                ("dz", C.c_double), ("dy", C.c_double), ("r_0", C.c_double),
                ("n_segments", C.c_int * 4), ("segments", C.POINTER(BCSegment) * 4),
                ("precision", C.c_int), ("with_prev", C.c_int)]


class Geometry(C.Structure):
    _fields_ = [("r_inner", DP), ("r_outer", DP), ("dr_inner_dz", DP), ("dr_outer_dz", DP)]


class MonitorRecord(C.Structure):
    _fields_ = [("step", C.c_longlong), ("t", C.c_double), ("dt", C.c_double),
                ("probe", C.c_double * 5), ("integrals", C.c_double * 7),
                ("max_wave_speed", C.c_double), ("dt_cfl", C.c_double),
                ("cfl_warning", C.c_int)]


MonitorFn = C.CFUNCTYPE(None, C.POINTER(MonitorRecord), C.c_void_p)


class RunParams(C.Structure):
    _fields_ = [("T", C.c_double), ("dt", C.c_double), ("adaptive", C.c_int),
                ("cfl_number", C.c_double), ("dt_growth_factor", C.c_double),
                ("dt_min", C.c_double), ("dt_max", C.c_double),
                ("convergence_threshold", C.c_double), ("check_frequency", C.c_int),
                ("residual_tol", C.c_double), ("residual_every", C.c_int),
                ("max_steps", C.c_longlong), ("steps_per_graph", C.c_int),
                ("engine", C.c_int), ("monitor_every", C.c_int), ("monitor", MonitorFn),
                ("monitor_user", C.c_void_p)]


class RunStats(C.Structure):
    _fields_ = [("steps", C.c_longlong), ("t", C.c_double), ("dt", C.c_double),
                ("residual", C.c_double), ("change", C.c_double),
                ("max_wave_speed", C.c_double), ("converged", C.c_int), ("status", C.c_int),
                ("device_ms", C.c_double)]


class GemmDesc(C.Structure):
    _fields_ = [("M", C.c_int), ("N", C.c_int), ("K", C.c_int), ("batch", C.c_int),
                ("A", C.c_void_p), ("sam", C.c_longlong), ("sak", C.c_longlong),
                ("sab", C.c_longlong),
                ("B", C.c_void_p), ("sbn", C.c_longlong), ("sbk", C.c_longlong),
                ("sbb", C.c_longlong),
                ("C", C.c_void_p), ("scm", C.c_longlong), ("scn", C.c_longlong),
                ("scb", C.c_longlong),
                ("alpha", C.c_float), ("beta", C.c_float),
                ("work", C.c_void_p), ("work_floats", C.c_longlong)]


class MpdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


_LIB = None
_EMU = None

# (name, restype, argtypes) of every entry point declared in include/mpd_b200.h
_VP = C.c_void_p
SIGNATURES = [
    ("mpd_create", C.c_int, [C.POINTER(Config), C.POINTER(Geometry), DP, C.POINTER(_VP)]),
    ("mpd_destroy", None, [_VP]),
    ("mpd_last_error", C.c_char_p, []),
    ("mpd_advance", C.c_int, [_VP, C.c_double]),
    ("mpd_run", C.c_int, [_VP, C.POINTER(RunParams), C.POINTER(RunStats)]),
    ("mpd_max_wave_speed", C.c_int, [_VP, DP]),
    ("mpd_compute_dt", C.c_int, [_VP, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, DP]),
    ("mpd_solution_change", C.c_int, [_VP, DP]),
    ("mpd_save_prev", C.c_int, [_VP]),
    ("mpd_integrals", C.c_int, [_VP, DP]),
    ("mpd_outlet", C.c_int, [_VP, DP, DP]),
    ("mpd_radial_symmetry", C.c_int, [_VP, DP]),
    ("mpd_residual", C.c_int, [_VP, DP]),
    ("mpd_probe", C.c_int, [_VP, C.c_int, C.c_int, DP]),
    ("mpd_time", C.c_int, [_VP, DP, C.POINTER(C.c_longlong)]),
    ("mpd_download", C.c_int, [_VP, C.c_int, DP]),
    ("mpd_snapshot_async", C.c_int, [_VP, DP]),
    ("mpd_snapshot_wait", C.c_int, [_VP]),
    ("mpd_set_physical", C.c_int, [_VP, DP]),
    ("mpd_set_expression_ic", C.c_int, [_VP, C.POINTER(C.c_char_p), C.c_int,
                                        C.POINTER(C.c_char_p), DP]),
    ("mpd_get_stream", C.c_int, [_VP, C.POINTER(_VP)]),
    ("mpd_set_ring_overlap", C.c_int, [_VP, C.c_int]),
    ("mpd_ring_overlap_active", C.c_int, [_VP, C.POINTER(C.c_int)]),
    ("mpd_device_bytes", C.c_int, [_VP, C.POINTER(C.c_size_t)]),
    ("mpd_profile_kernels", C.c_int, [_VP, C.c_int, C.c_double, DP]),
    ("mpd_profile_kernel", C.c_int, [_VP, C.c_int, C.c_int, C.c_double, DP]),
    ("mpd_integrals_noalloc", C.c_int, [_VP, C.c_size_t, C.c_int, C.c_int, C.c_int, _VP, C.c_double,
                                        _VP, _VP]),
    ("mpd_batch_create", C.c_int, [C.POINTER(_VP), C.c_int, C.POINTER(_VP)]),
    ("mpd_batch_destroy", None, [_VP]),
    ("mpd_batch_capacity", C.c_int, [_VP, C.POINTER(C.c_int)]),
    ("mpd_batch_run", C.c_int, [_VP, C.POINTER(RunParams), C.c_int, C.POINTER(C.c_int),
                                C.POINTER(C.c_int), DP, C.POINTER(RunStats), DP, DP]),
    ("mpd_nn_gemm", C.c_int, [C.POINTER(GemmDesc), _VP]),
    ("mpd_nn_wait_status", C.c_int, [_VP]),
    ("mpd_nn_bias_act", C.c_int, [_VP, _VP, _VP, C.c_longlong, C.c_int, C.c_int, _VP]),
    ("mpd_nn_act_bwd", C.c_int, [_VP, _VP, _VP, C.c_longlong, _VP]),
    ("mpd_nn_colsum", C.c_int, [_VP, C.c_longlong, C.c_int, _VP, _VP, _VP]),
    ("mpd_nn_sum_parts", C.c_int, [_VP, C.c_int, C.c_longlong, _VP, C.c_int, _VP]),
    ("mpd_nn_mse", C.c_int, [_VP, _VP, C.c_longlong, _VP, _VP, _VP, _VP]),
    ("mpd_nn_adam", C.c_int, [_VP, _VP, _VP, _VP, C.c_longlong, C.c_float, C.c_float, C.c_float,
                              C.c_float, C.c_int, _VP]),
    ("mpd_remap_snapshot", C.c_int, [_VP, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _VP,
                                     _VP]),
    ("mpd_fast_math", C.c_int, [_VP, C.c_longlong, _VP, _VP, _VP]),
    ("mpd_expression_ic", C.c_int, [C.POINTER(Config), C.POINTER(Geometry), C.POINTER(C.c_char_p),
                                    C.c_int, C.POINTER(C.c_char_p), DP, DP]),
    ("mpd_eval_expression", C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_char_p), DP, DP]),
]


def _bind(lib, sigs):
    for name, res, args in sigs:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


def load() -> C.CDLL:
    """Open libmpd_b200.so (building it first if the toolkit is present)."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            from . import build  # noqa: WPS433 - build on first use in a fresh tree
            build.build_lib()
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build the CUDA extension first")
        _LIB = _bind(C.CDLL(str(LIB_PATH)), SIGNATURES)
    return _LIB


def load_emu() -> C.CDLL:
    """Open the host emulator (CPU test suite only)."""
    global _EMU
    if _EMU is None:
        if not EMU_PATH.exists():
            from . import build
            build.build_emu()
        lib = C.CDLL(str(EMU_PATH))
        lib.mpd_emu_create.restype = C.c_int
        lib.mpd_emu_create.argtypes = [C.POINTER(Config), C.POINTER(Geometry), DP, C.POINTER(_VP)]
        lib.mpd_emu_advance.restype = C.c_int
        lib.mpd_emu_advance.argtypes = [_VP, C.c_double, C.c_int]
        lib.mpd_emu_download.restype = C.c_int
        lib.mpd_emu_download.argtypes = [_VP, C.c_int, DP]
        lib.mpd_emu_wave_speed.restype = C.c_double
        lib.mpd_emu_wave_speed.argtypes = [_VP]
        lib.mpd_emu_destroy.argtypes = [_VP]
        lib.mpd_emu_last_error.restype = C.c_char_p
        _bind(lib, [s for s in SIGNATURES if s[0] in ("mpd_expression_ic", "mpd_eval_expression")])
        _EMU = lib
    return _EMU


def check(rc: int, lib=None) -> None:
    if rc != MPD_OK:
        lib = lib or load()
        err = lib.mpd_last_error() if hasattr(lib, "mpd_last_error") else lib.mpd_emu_last_error()
        raise MpdError(rc, (err or b"").decode(errors="replace"))
