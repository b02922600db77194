"""The device kernels' per-cell code, compiled for the host (libmpd_emu.so),
checked against the oracle without a GPU: exact mode bit for bit, the
boundary ring free of read/write hazards, fast mode within tolerance."""
import numpy as np
import pytest

from oracle import bind
from tests import cases
from tests.emu import Emu

CONFIGS = [
    ("channel_sine", cases.channel_config(L=24, M=12, a=0.1), 1e-4),
    ("reference_default", cases.reference_default_config(L=48, M=20), 1e-6),
    ("edge_segments", cases.edge_config(), 1e-4),
]


@pytest.mark.parametrize("name,cfg,dt0", CONFIGS)
def test_exact_emulation_bitwise(name, cfg, dt0):
    case = cases.make_case(cfg)
    oracle = bind.Port(case.oracle_dict())
    emu = Emu(case, "exact")
    dt = dt0
    for step in range(30):
        oracle.advance(dt)
        emu.advance(dt, order=step % 3)
        np.testing.assert_array_equal(emu.conserved(), oracle.conserved())
        assert emu.max_wave_speed() == oracle.max_wave_speed()
        dt = oracle.compute_dt(cfg.cfl_number, cfg.dt_growth_factor, cfg.dt_min, cfg.dt_max, dt)
    np.testing.assert_array_equal(emu.physical(), oracle.physical())


def test_ring_write_order_does_not_matter():
    """Each boundary thread reads only interior cells, snapshots and its own
    cell, so any write order gives the same state (the kernel has no hazards)."""
    cfg = cases.edge_config()
    case = cases.make_case(cfg)
    emus = [Emu(case, "exact") for _ in range(3)]
    for _ in range(15):
        for order, e in enumerate(emus):
            e.advance(1e-4, order=order)
    a = emus[0].conserved()
    for e in emus[1:]:
        np.testing.assert_array_equal(e.conserved(), a)


def test_uncovered_wall_cells_hold_zero_like_the_reference():
    """A wall cell no segment covers is never written by the reference, so its
    u stays at the zero Array2D initialises it to (src/array2d.cpp:29-43)."""
    cfg = cases.channel_config(L=16, M=8)
    cfg.bc_m_lo.segments = [cases.segment((0, 5), v_r=("expr", "v_z * r_z")),
                            cases.segment((8, -1), v_r=("expr", "v_z * r_z"))]
    case = cases.make_case(cfg)
    oracle = bind.Port(case.oracle_dict())
    emu = Emu(case, "exact")
    oracle.advance(1e-4)
    emu.advance(1e-4)
    got, want = emu.conserved(), oracle.conserved()
    np.testing.assert_array_equal(got, want)
    # global l = 6, 7 (local rows 7, 8) are covered by no inner-wall segment
    assert (want[:, 7, 1] == 0).all() and (want[:, 8, 1] == 0).all()


def test_fast_emulation_within_tolerance():
    cfg = cases.channel_config(L=60, M=24, a=0.1)
    case = cases.make_case(cfg)
    oracle = bind.Port(case.oracle_dict())
    emu = Emu(case, "fast")
    dt = cfg.dt
    for _ in range(300):
        oracle.advance(dt)
        emu.advance(dt)
        dt = oracle.compute_dt(cfg.cfl_number, cfg.dt_growth_factor, cfg.dt_min, cfg.dt_max, dt)
    got, want = emu.conserved(), oracle.conserved()
    for k in range(8):
        den = np.abs(want[k]).max() or 1.0
        assert np.abs(got[k] - want[k]).max() / den <= 1e-12
