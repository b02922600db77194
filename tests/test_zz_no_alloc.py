"""mpd_integrals_noalloc: the conserved integrals for callers that cannot let
a library allocate device memory (their framework's pool owns it all).

The entry point keeps its scratch in a fixed device array instead of
cudaMalloc; this test gives it device planes the test itself owns and checks
two calls in a row, on two different states, against mpd_integrals.  The
file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from tests import cases

pytestmark = pytest.mark.gpu

pkg = cases.pkg
N = pkg._native
RTOL = 1e-13  # same tolerance as the other integral checks (summation order differs)


def device_planes(torch, solver, grid):
    """The solver's conserved state and dr, copied into test-owned device memory."""
    cons = torch.from_numpy(np.ascontiguousarray(solver.conserved())).cuda()
    dr = torch.from_numpy(np.ascontiguousarray(grid.dr)).cuda()
    return cons, dr


def test_integrals_noalloc_matches_mpd_integrals_twice():
    import torch

    lib = N.load()
    case = cases.channel_case(L=200, M=80, a=0.1)
    cfg = case.cfg
    solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision="exact")
    solver.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=40)
    want_a = solver.ComputeIntegrals()
    cons_a, dr = device_planes(torch, solver, case.grid)
    solver.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=60)
    want_b = solver.ComputeIntegrals()
    cons_b, _ = device_planes(torch, solver, case.grid)
    solver.close()
    assert not np.array_equal(want_a, want_b)

    rows, cols = cfg.L_max + 2, cfg.M_max + 3
    out_a = torch.zeros(7, dtype=torch.float64, device="cuda")
    out_b = torch.zeros(7, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    free = []
    for cons, out in ((cons_a, out_a), (cons_b, out_b)):   # two calls in a row
        rc = lib.mpd_integrals_noalloc(C.c_void_p(cons.data_ptr()), rows * cols, cols, cfg.L_max,
                                       cfg.M_max, C.c_void_p(dr.data_ptr()), cfg.dz,
                                       C.c_void_p(out.data_ptr()), stream)
        assert rc == N.MPD_OK, lib.mpd_last_error()
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
    # the first call may load the library's module (lazy loading creates the
    # fixed array then); the second must not change the device's free memory
    assert free[1] == free[0], free
    np.testing.assert_allclose(out_a.cpu().numpy(), want_a, rtol=RTOL, atol=0)
    np.testing.assert_allclose(out_b.cpu().numpy(), want_b, rtol=RTOL, atol=0)


def test_integrals_noalloc_rejects_too_many_rows():
    lib = N.load()
    dummy = C.c_void_p(16)
    rc = lib.mpd_integrals_noalloc(dummy, 10**9, 8, 9000, 4, dummy, 1e-3, dummy, None)
    assert rc == N.MPD_ERR_INVALID
    assert b"exceeds the 8192 rows" in lib.mpd_last_error()
