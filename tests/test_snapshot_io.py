"""Snapshot I/O on the CPU: the legacy-VTK writer's layout (IOManager::WriteVtk,
src/io_manager.cpp:218-315) round-trips through the reader."""
import numpy as np

from tests import cases

import __graft_entry__

pkg = __graft_entry__.load_package()


def test_vtk_round_trip(tmp_path):
    case = cases.channel_case(L=24, M=12, a=0.1)
    cfg, grid, phys = case.cfg, case.grid, case.phys
    path = pkg.io.write_vtk(tmp_path / "step_0000.vtk", phys, grid.r, cfg.dz, cfg.L_max, cfg.M_max)
    snap = pkg.io.read_vtk(path)
    ni, nj = cfg.L_max + 1, cfg.M_max + 1
    assert snap["dims"] == (ni, nj)
    arrays = pkg.io.snapshot_arrays(phys, grid.r, cfg.L_max, cfg.M_max)
    for name in ("Rho", "Energy", "MPI_Rank", "Hphi_times_r"):
        np.testing.assert_array_equal(snap[name], arrays[name].reshape(-1))
    for name in ("Velocity", "MagneticField"):
        np.testing.assert_array_equal(snap[name], arrays[name].reshape(-1, 3))
    # point i of row j sits at z = i dz on the r of row min(i, L-1)
    pts = snap["points"].reshape(nj, ni, 3)
    np.testing.assert_array_equal(pts[:, :, 0], np.broadcast_to(np.arange(ni) * cfg.dz, (nj, ni)))
    assert pts[3, ni - 1, 1] == grid.r[cfg.L_max, 4]
    # the reference's last point row repeats row L-1
    np.testing.assert_array_equal(snap["Rho"].reshape(nj, ni)[:, -1], phys[0, cfg.L_max, 1:cfg.M_max + 2])
