"""Wrapper of the host emulator library (libmpd_emu.so) for the CPU suite."""
from __future__ import annotations

import ctypes as C

import numpy as np

import __graft_entry__

pkg = __graft_entry__.load_package()
N = pkg._native


class Emu:
    def __init__(self, case, precision="exact"):
        self.lib = N.load_emu()
        cfg = case.cfg
        self.shape = (cfg.L_max + 2, cfg.M_max + 3)
        self._cc = pkg.config.CConfig(cfg, case.grid.r_0, pkg.solver.PRECISIONS[precision], False)
        self._prof = [np.ascontiguousarray(a) for a in case.grid.profiles()]
        geo = N.Geometry(*(a.ctypes.data_as(N.DP) for a in self._prof))
        phys = np.ascontiguousarray(case.phys)
        h = C.c_void_p()
        rc = self.lib.mpd_emu_create(self._cc.ptr, C.byref(geo), phys.ctypes.data_as(N.DP),
                                     C.byref(h))
        if rc != 0:
            raise N.MpdError(rc, self.lib.mpd_emu_last_error().decode())
        self.h = h

    def advance(self, dt, order=0):
        self.lib.mpd_emu_advance(self.h, float(dt), int(order))

    def get(self, which):
        out = np.empty(self.shape)
        self.lib.mpd_emu_download(self.h, int(which), out.ctypes.data_as(N.DP))
        return out

    def conserved(self):
        return np.stack([self.get(k) for k in range(8)])

    def physical(self):
        return np.stack([self.get(8 + k) for k in range(10)])

    def max_wave_speed(self):
        return self.lib.mpd_emu_wave_speed(self.h)

    def __del__(self):
        try:
            self.lib.mpd_emu_destroy(self.h)
        except Exception:
            pass
