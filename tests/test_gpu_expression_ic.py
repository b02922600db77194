"""ExpressionIC evaluated on the device (mpd_set_expression_ic) against the
host sweep (mpd_expression_ic), which follows src/ics/expression_ic.cpp:286-324."""
from __future__ import annotations

import numpy as np
import pytest

from tests import cases

pytestmark = pytest.mark.gpu


def _device_planes(pkg, cfg, ic):
    grid = pkg.Grid(cfg, pkg.GeometryRegistry.Instance().Create(cfg.geometry.type,
                                                               cfg.geometry.params))
    s = pkg.GpuSolver(cfg, grid, ic, precision="fast")
    try:
        return grid, s.physical()
    finally:
        s.close()


@pytest.mark.parametrize("make", [
    lambda: cases.channel_config(L=64, M=33),
    lambda: cases.channel_config(L=40, M=20, a=0.15, beta=0.3, amp=1.7, vz=0.2),
    lambda: cases.reference_default_config(L=80, M=40),
])
def test_device_ic_equals_host_sweep(pkg, make):
    cfg = make()
    ic = pkg.ExpressionIC(cfg.initial_conditions.params)
    grid, dev = _device_planes(pkg, cfg, ic)
    host = ic.Apply(grid, cfg)
    np.testing.assert_array_equal(dev, host)


def test_device_ic_user_vars_and_defaults(pkg):
    cfg = cases.channel_config(L=30, M=17)
    ic = pkg.ExpressionIC({"rho": "k * (1 + 0.5 * z) / r", "v_z": "u0 * r_z + 0.1",
                           "vars": {"k": 0.75, "u0": 2.0}})   # other fields: defaults
    grid, dev = _device_planes(pkg, cfg, ic)
    np.testing.assert_array_equal(dev, ic.Apply(grid, cfg))


def test_forward_reference_is_refused_on_device_and_swept_on_host(pkg):
    """rho reads v_z, evaluated after it: the reference's sweep sees the
    previous cell's v_z, which only the sequential host sweep reproduces."""
    cfg = cases.channel_config(L=24, M=12)
    ic = pkg.ExpressionIC({"rho": "1 + v_z", "v_z": "0.1 * r"})
    grid = pkg.Grid(cfg, pkg.GeometryRegistry.Instance().Create(cfg.geometry.type,
                                                               cfg.geometry.params))
    host = ic.Apply(grid, cfg)
    s = pkg.GpuSolver(cfg, grid, host, precision="fast")
    rc = ic.ApplyDevice(s.lib, s.h)
    assert rc == pkg._native.MPD_ERR_UNSUPPORTED_IC
    assert b"evaluated after it" in s.lib.mpd_last_error()
    s.close()
    # GpuSolver given the IC itself takes the host sweep for it
    grid2, dev = _device_planes(pkg, cfg, ic)
    np.testing.assert_array_equal(dev, host)
    assert host[0, 2, 1] != host[0, 1, 1]    # the carried value made a difference
