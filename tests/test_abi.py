"""The C ABI library loads without a GPU and exports every symbol that
include/mpd_b200.h declares; argument errors come back as status codes."""
import ctypes as C
import pathlib
import re

import numpy as np
import pytest

from tests import cases

pkg = cases.pkg
N = pkg._native
HEADER = pathlib.Path(__file__).resolve().parent.parent / "include" / "mpd_b200.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\s*\*)\s*(mpd_\w+)\s*\(", text, re.M)))


def test_header_declarations_are_exported():
    names = declared_functions()
    assert len(names) >= 20
    lib = C.CDLL(str(N.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    bound = {s[0] for s in N.SIGNATURES}
    assert set(names) <= bound, set(names) - bound


def test_invalid_config_rejected_without_device():
    lib = N.load()
    cfg = N.Config()
    cfg.L_max, cfg.M_max, cfg.dz, cfg.dy = 2, 2, 0.5, 0.5
    h = C.c_void_p()
    rc = lib.mpd_create(C.byref(cfg), None, None, C.byref(h))
    assert rc == N.MPD_ERR_INVALID
    assert b"grid too small" in lib.mpd_last_error()
    assert lib.mpd_advance(None, 1.0) == N.MPD_ERR_INVALID


def test_no_device_reported_on_cpu_only_host(gpu_available):
    if gpu_available:
        pytest.skip("a GPU is present")
    case = cases.channel_case(L=12, M=6)
    with pytest.raises(N.MpdError) as ei:
        pkg.GpuSolver(case.cfg, case.grid, case.phys)
    assert ei.value.code == N.MPD_ERR_NO_DEVICE
