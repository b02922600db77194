"""Parity of the CUDA path with the oracle, through the C ABI.

Exact mode must reproduce the oracle (itself pinned bit for bit to the
reference's own build) bit for bit; fast mode must stay within 1e-12
relative L-inf per field after 1000 steps of the plain-method channel
(200 x 80, the CPU-runnable workload).
"""
import numpy as np
import pytest

from oracle import bind
from tests import cases

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-12  # relative L-inf per field after 1000 steps


def rel_linf(a, b):
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))


def step_both(solver, oracle, cfg, n, dt):
    """Advance both with the driver's adaptive dt; dt must agree bit for bit."""
    for _ in range(n):
        solver.Advance(dt)
        oracle.advance(dt)
        if cfg.adaptive_dt:
            d_gpu = solver.ComputeDt(dt)
            d_ref = oracle.compute_dt(cfg.cfl_number, cfg.dt_growth_factor, cfg.dt_min,
                                      cfg.dt_max, dt)
            assert d_gpu == d_ref
            dt = d_ref
    return dt


@pytest.mark.parametrize("name,cfg,dt0,nsteps", [
    ("channel_sine", cases.channel_config(L=24, M=12, a=0.1), 1e-4, 30),
    ("reference_default", cases.reference_default_config(L=80, M=40), 1e-6, 40),
    ("edge_segments", cases.edge_config(), 1e-4, 40),
])
def test_exact_bitwise_per_step(pkg, name, cfg, dt0, nsteps):
    case = cases.make_case(cfg)
    solver = pkg.GpuSolver(case.cfg, case.grid, case.phys, precision="exact")
    oracle = bind.Port(case.oracle_dict())
    dt = dt0
    for chunk in range(4):
        dt = step_both(solver, oracle, cfg, nsteps // 4, dt)
        np.testing.assert_array_equal(solver.conserved(), oracle.conserved())
    np.testing.assert_array_equal(solver.physical(), oracle.physical())
    solver.close()


def test_config1_exact_run_1000_steps(pkg):
    """Plain method, 200 x 80, CFL 0.4, fixed 1000 steps: graph-resident loop."""
    case = cases.channel_case(L=200, M=80)
    cfg = case.cfg
    solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision="exact")
    res = solver.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=1000, steps_per_graph=64)
    oracle = bind.Port(case.oracle_dict())
    out = oracle.run(T=1e300, dt0=cfg.dt, adaptive=True, cfl=cfg.cfl_number,
                     growth=cfg.dt_growth_factor, dt_min=cfg.dt_min, dt_max=cfg.dt_max,
                     max_steps=1000)
    assert res.steps == out["steps"] == 1000
    assert res.t == out["t"] and res.dt == out["dt"]
    np.testing.assert_array_equal(solver.conserved(), oracle.conserved())
    np.testing.assert_array_equal(solver.physical(), oracle.physical())
    solver.close()


def test_config1_fast_run_1000_steps(pkg):
    case = cases.channel_case(L=200, M=80)
    cfg = case.cfg
    solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision="fast")
    res = solver.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=1000)
    oracle = bind.Port(case.oracle_dict())
    out = oracle.run(T=1e300, dt0=cfg.dt, adaptive=True, cfl=cfg.cfl_number,
                     growth=cfg.dt_growth_factor, dt_min=cfg.dt_min, dt_max=cfg.dt_max,
                     max_steps=1000)
    assert res.steps == 1000
    assert abs(res.t - out["t"]) <= FAST_TOL * out["t"]
    got, want = solver.physical(), oracle.physical()
    for k in range(10):
        assert rel_linf(got[k], want[k]) <= FAST_TOL, bind.PHYS_FIELDS[k]
    got, want = solver.conserved(), oracle.conserved()
    for k in range(8):
        assert rel_linf(got[k], want[k]) <= FAST_TOL, f"u_{k + 1}"
    solver.close()


def test_fast_reference_default_and_edge(pkg):
    for cfg, dt0 in ((cases.reference_default_config(L=80, M=40), 1e-6), (cases.edge_config(), 1e-4)):
        case = cases.make_case(cfg)
        solver = pkg.GpuSolver(case.cfg, case.grid, case.phys, precision="fast")
        oracle = bind.Port(case.oracle_dict())
        dt = dt0
        for _ in range(200):
            solver.Advance(dt)
            oracle.advance(dt)
            dt = oracle.compute_dt(cfg.cfl_number, cfg.dt_growth_factor, cfg.dt_min, cfg.dt_max, dt)
        got, want = solver.conserved(), oracle.conserved()
        for k in range(8):
            assert rel_linf(got[k], want[k]) <= FAST_TOL
        solver.close()


def test_diagnostics_match_oracle(pkg):
    case = cases.channel_case(L=40, M=20, a=0.12)
    cfg = case.cfg
    solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision="exact", with_prev=True)
    oracle = bind.Port(case.oracle_dict(with_prev=True))
    # before any step the diagnostics read the initial condition
    assert solver.MaxWaveSpeed() == oracle.max_wave_speed()
    assert solver.CheckRadialSymmetry() == oracle.radial_symmetry()
    dt = step_both(solver, oracle, cfg, 25, 1e-4)
    assert solver.MaxWaveSpeed() == oracle.max_wave_speed()
    assert solver.ComputeDt(dt) == oracle.compute_dt(cfg.cfl_number, cfg.dt_growth_factor,
                                                     cfg.dt_min, cfg.dt_max, dt)
    assert solver.CheckRadialSymmetry() == oracle.radial_symmetry()
    mf, th = solver.outlet()
    omf, oth = oracle.outlet()
    assert (mf, th) == (omf, oth)          # serial trapezoid, same order
    np.testing.assert_allclose(solver.ComputeIntegrals(), oracle.integrals(), rtol=1e-13, atol=0)
    ch = solver.SolutionChange()
    assert abs(ch - oracle.solution_change()) <= 1e-12 * max(ch, 1e-300)
    solver.SavePrev()
    oracle.save_prev()
    step_both(solver, oracle, cfg, 5, dt)
    ch = solver.SolutionChange()
    assert abs(ch - oracle.solution_change()) <= 1e-12 * max(ch, 1e-300)
    probe = solver.probe(20, 10)
    phys = oracle.physical()
    np.testing.assert_array_equal(probe, phys[:, 21, 11])
    solver.close()


def test_run_convergence_check_matches_driver(pkg):
    """Relative-L2 convergence every check_frequency steps (src/main.cpp:233-247)."""
    case = cases.channel_case(L=32, M=16)
    cfg = case.cfg
    solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision="exact", with_prev=True)
    res = solver.run(T=1e300, dt=cfg.dt, adaptive=True, convergence_threshold=5e-3,
                     check_frequency=20, max_steps=5000, steps_per_graph=40)
    oracle = bind.Port(case.oracle_dict(with_prev=True))
    out = oracle.run(T=1e300, dt0=cfg.dt, adaptive=True, cfl=cfg.cfl_number,
                     growth=cfg.dt_growth_factor, dt_min=cfg.dt_min, dt_max=cfg.dt_max,
                     conv_threshold=5e-3, check_frequency=20, max_steps=5000)
    assert res.converged == out["converged"]
    assert res.steps == out["steps"]
    assert abs(res.change - out["change"]) <= 1e-12 * out["change"]
    np.testing.assert_array_equal(solver.conserved(), oracle.conserved())
    solver.close()


def test_t_clamp_and_residual(pkg):
    """The last step is clamped to T (src/main.cpp:221-223); residual matches numpy."""
    case = cases.channel_case(L=24, M=12)
    cfg = case.cfg
    solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision="exact")
    res = solver.run(T=0.05, dt=cfg.dt, adaptive=True)
    oracle = bind.Port(case.oracle_dict())
    out = oracle.run(T=0.05, dt0=cfg.dt, adaptive=True, cfl=cfg.cfl_number,
                     growth=cfg.dt_growth_factor, dt_min=cfg.dt_min, dt_max=cfg.dt_max)
    assert res.steps == out["steps"]
    assert res.t == out["t"]
    np.testing.assert_array_equal(solver.conserved(), oracle.conserved())
    before = solver.conserved()
    solver.Advance(1e-4)
    after = solver.conserved()
    inner = (slice(None), slice(1, -1), slice(1, -1))
    num = np.abs(after[inner] - before[inner]).reshape(8, -1).max(axis=1)
    den = np.maximum(np.abs(before[inner]).reshape(8, -1).max(axis=1), 1e-300)
    assert solver.residual() == float((num / den).max())
    solver.close()


@pytest.mark.parametrize("L,M", [(200, 80), (40, 63), (33, 95)])
def test_residual_matches_numpy(pkg, L, M):
    """The L-inf residual over row x 32-column units: ragged last units
    (M + 1 = 81, 96) and rows of exactly two units (M + 1 = 64)."""
    case = cases.channel_case(L=L, M=M)
    cfg = case.cfg
    solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision="fast")
    solver.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=30)
    before = solver.conserved()
    solver.Advance(solver.ComputeDt(cfg.dt))
    after = solver.conserved()
    inner = (slice(None), slice(1, -1), slice(1, -1))
    num = np.abs(after[inner] - before[inner]).reshape(8, -1).max(axis=1)
    den = np.maximum(np.abs(before[inner]).reshape(8, -1).max(axis=1), 1e-300)
    assert solver.residual() == float((num / den).max())
    solver.close()


def test_residual_leaves_nan_out_and_flags_it(pkg):
    """A NaN in the state: the residual's maxima skip it (NaN-ignoring
    maxima, as numpy's nanmax) and the state is flagged non-finite."""
    case = cases.channel_case(L=40, M=20)
    cfg = case.cfg
    phys = np.array(case.phys, copy=True)
    phys[0, 20, 10] = np.nan
    solver = pkg.GpuSolver(cfg, case.grid, phys, precision="fast")
    before = solver.conserved()
    solver.Advance(cfg.dt)
    after = solver.conserved()
    inner = (slice(None), slice(1, -1), slice(1, -1))
    assert np.isnan(after[inner]).any() and np.isfinite(after[inner]).any()
    with np.errstate(invalid="ignore"):
        num = np.nanmax(np.abs(after[inner] - before[inner]).reshape(8, -1), axis=1)
        den = np.maximum(np.nanmax(np.abs(before[inner]).reshape(8, -1), axis=1), 1e-300)
    assert solver.residual() == float(np.nanmax(num / den))
    res = solver.run(T=1e300, dt=cfg.dt, adaptive=False, max_steps=1)
    assert res.status == pkg._native.MPD_ERR_NONFINITE
    solver.close()


def test_restart_set_physical_and_snapshot(pkg):
    case = cases.channel_case(L=24, M=12, a=0.05)
    cfg = case.cfg
    solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision="exact")
    solver.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=50)
    phys = solver.physical()
    # restart from the downloaded physical state == a fresh solver from it
    other = pkg.GpuSolver(cfg, case.grid, phys, precision="exact")
    solver.set_physical(phys)
    for s in (solver, other):
        s.Advance(2e-4)
    np.testing.assert_array_equal(solver.conserved(), other.conserved())
    # async snapshot into pinned memory equals the synchronous download
    import torch
    buf = torch.empty((10,) + solver.shape, dtype=torch.float64).pin_memory()
    import ctypes
    lib = solver.lib
    rc = lib.mpd_snapshot_async(solver.h, ctypes.cast(ctypes.c_void_p(buf.data_ptr()),
                                                      pkg._native.DP))
    assert rc == 0
    assert lib.mpd_snapshot_wait(solver.h) == 0
    np.testing.assert_array_equal(buf.numpy(), solver.physical())
    solver.close()
    other.close()


def test_snapshot_mid_run_captures_its_step(pkg):
    """IOManager's snapshot (src/io_manager.cpp:68-77) taken while stepping
    goes on: mpd_snapshot_async at step 40 of the 200 x 80 channel (exact
    precision), then 60 more steps through the graph run loop on the solver's
    stream while the copies run on the side stream; the pinned buffer must
    hold the oracle's physical planes of step 40 bit for bit, and the state
    after step 100 must equal the oracle's too (the snapshot did not disturb
    the stepping)."""
    import torch
    case = cases.channel_case(L=200, M=80, a=0.1)
    cfg = case.cfg
    solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision="exact")
    oracle = bind.Port(case.oracle_dict())
    dt = step_both(solver, oracle, cfg, 40, cfg.dt)
    at40 = oracle.physical()
    buf = torch.empty((10,) + solver.shape, dtype=torch.float64).pin_memory()
    solver.snapshot_async(buf)
    res = solver.run(T=1e300, dt=dt, adaptive=True, max_steps=60)
    solver.snapshot_wait()
    np.testing.assert_array_equal(buf.numpy(), at40)
    assert res.steps == 60
    cases.run_oracle_steps(oracle, 60, dt, cfg)
    np.testing.assert_array_equal(solver.conserved(), oracle.conserved())
    solver.close()
    oracle.close()


def test_run_monitor_reports_match_oracle(pkg):
    """The driver loop's periodic reports from inside mpd_run
    (src/main.cpp:249-281): on the 200 x 80 channel (exact precision, adaptive
    dt) a 2500-step run reports at steps 1000 and 2000 the checkpoint cell's
    values, t, the next dt and the wave speed bit for bit as the oracle, the
    conserved integrals within 1e-13, and no CheckCfl warning; the run itself
    ends in the oracle's state."""
    case = cases.channel_case(L=200, M=80, a=0.1)
    cfg = case.cfg
    solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision="exact")
    reps = []
    res = solver.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=2500, monitor=reps.append,
                     monitor_every=1000)
    assert res.steps == 2500
    assert [r.step for r in reps] == [1000, 2000]
    oracle = bind.Port(case.oracle_dict())
    dt, t = cfg.dt, 0.0
    for rep in reps:
        for _ in range(1000):
            oracle.advance(dt)
            t += dt
            dt = oracle.compute_dt(cfg.cfl_number, cfg.dt_growth_factor, cfg.dt_min, cfg.dt_max,
                                   dt)
        phys = oracle.physical()
        assert list(rep.probe) == [phys[k][21, 41] for k in (0, 1, 3, 4, 9)]
        assert (rep.t, rep.dt) == (t, dt)
        assert rep.max_wave_speed == oracle.max_wave_speed()
        assert not rep.cfl_warning
        np.testing.assert_allclose(rep.integrals, oracle.integrals(), rtol=1e-13, atol=0)
    cases.run_oracle_steps(oracle, 500, dt, cfg)
    np.testing.assert_array_equal(solver.conserved(), oracle.conserved())
    solver.close()
    oracle.close()


def test_run_monitor_flags_cfl_warning(pkg):
    """A fixed dt above the CFL limit: every report carries CheckCfl's warning
    (src/diagnostics.cpp:112-125), with the wave speed of the state."""
    case = cases.channel_case(L=200, M=80)
    cfg = case.cfg
    solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision="fast")
    reps = []
    solver.run(T=1e300, dt=1.7e-3, adaptive=False, max_steps=1000, monitor=reps.append,
               monitor_every=500)
    assert [r.step for r in reps] == [500, 1000]
    for r in reps:
        assert r.cfl_warning and r.dt == 1.7e-3 and r.dt_cfl < 1.7e-3
        assert r.dt_cfl == cfg.cfl_number * min(cfg.dz, cfg.dy) / (r.max_wave_speed + 1e-10)
    assert reps[-1].max_wave_speed == solver.MaxWaveSpeed()
    solver.close()


def test_full_size_channel_fast_vs_oracle(pkg):
    """The 1600 x 640 channel (440 blocks of TMA strips and bands): the fast
    path through the graph run loop against the oracle's own driver loop
    (adaptive dt, CFL 0.4) over 1000 steps, every conserved and physical plane
    within 1e-12 relative L-inf, and the same simulated time.  The oracle is
    the reference's own build when present (bit-identical to the port)."""
    case = cases.channel_case(L=1600, M=640)
    cfg = case.cfg
    solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision="fast")
    res = solver.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=1000)
    assert res.steps == 1000
    oracle = (bind.Ref if bind.ref_available() else bind.Port)(case.oracle_dict())
    ran = oracle.run(1e300, cfg.dt, True, cfg.cfl_number, cfg.dt_growth_factor, cfg.dt_min,
                     cfg.dt_max, max_steps=1000)
    assert ran["steps"] == 1000
    assert abs(res.t - ran["t"]) <= 1e-12 * ran["t"]
    got, want = solver.conserved(), oracle.conserved()
    for k in range(8):
        assert rel_linf(got[k], want[k]) <= FAST_TOL, k
    got, want = solver.physical(), oracle.physical()
    for k in range(10):
        assert rel_linf(got[k], want[k]) <= FAST_TOL, k
    solver.close()
    oracle.close()


def test_bad_config_is_rejected_before_device_work(pkg):
    cfg = cases.channel_config(L=24, M=12)
    cfg.bc_l_lo.segments[0].rho = pkg.FieldCond("axis_lf")
    case_geo = pkg.Grid(cfg, pkg.GeometryRegistry.Instance().Create("sine_wall", cfg.geometry.params))
    phys = np.zeros((10, 26, 15))
    with pytest.raises(pkg._native.MpdError) as ei:
        pkg.GpuSolver(cfg, case_geo, phys)
    assert ei.value.code == pkg._native.MPD_ERR_INVALID
    assert "AxisLF condition is only valid on the M_LO face" in str(ei.value)


@pytest.mark.parametrize("name,cfg,steps,resid_every,T", [
    ("channel_200x80", cases.channel_config(L=200, M=80), 700, 25, 1e300),
    ("reference_default", cases.reference_default_config(L=80, M=40), 300, 7, 1e300),
    ("edge_segments", cases.edge_config(), 200, 1, 1e300),
    ("t_clamp", cases.channel_config(L=64, M=30, a=0.1), 100000, 10, 0.02),
    # a square grid with bands of more than ten rows per warp
    ("square_800x800", cases.channel_config(L=800, M=800, a=0.1), 60, 20, 1e300),
])
def test_persistent_engine_matches_graph_engine(pkg, name, cfg, steps, resid_every, T):
    """One cooperative launch per chunk of steps gives the graph path's bits:
    the same state, t, dt, step count and residual schedule."""
    case = cases.make_case(cfg)
    res = {}
    state = {}
    for engine in ("graph", "persistent"):
        solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision="fast")
        r = solver.run(T=T, dt=cfg.dt, adaptive=True, max_steps=steps,
                       residual_every=resid_every, engine=engine)
        res[engine] = r
        state[engine] = (solver.conserved(), solver.time(), solver.MaxWaveSpeed())
        solver.close()
    g, p = res["graph"], res["persistent"]
    assert (p.steps, p.t, p.dt, p.max_wave_speed) == (g.steps, g.t, g.dt, g.max_wave_speed)
    assert p.residual == g.residual
    np.testing.assert_array_equal(state["persistent"][0], state["graph"][0])
    assert state["persistent"][1:] == state["graph"][1:]


def test_persistent_engine_stops_on_residual(pkg):
    """residual_tol ends the persistent run at the same step as the graph run."""
    cfg = cases.channel_config(L=40, M=16)
    case = cases.make_case(cfg)
    out = []
    for engine in ("graph", "persistent"):
        solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision="fast")
        r = solver.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=200000, residual_tol=1e-5,
                       residual_every=20, engine=engine)
        out.append((r.steps, r.converged, r.residual, r.t))
        solver.close()
    assert out[0] == out[1]
    assert out[0][1] and out[0][2] <= 1e-5


def test_vtk_restart_remap_matches_oracle(pkg, tmp_path):
    """VtkIC (device bilinear remap) against the CPU restatement of
    src/ics/vtk_ic.cpp:137-239, bit for bit, onto the same grid and onto a
    finer one; then a solver starts from it."""
    from oracle import vtk_remap
    case = cases.channel_case(L=40, M=16, a=0.1)
    cfg = case.cfg
    solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision="fast")
    solver.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=300)
    phys = solver.physical()
    solver.close()
    path = pkg.io.write_vtk(tmp_path / "step_0300.vtk", phys, case.grid.r, cfg.dz, cfg.L_max,
                            cfg.M_max)
    ic = pkg.io.VtkIC(path)
    src = ic.source_fields(ic.snap)
    ni, nj = ic.snap["dims"]
    for L, M in ((40, 16), (97, 33)):
        fine = cases.channel_config(L=L, M=M, a=0.1)
        fgrid = cases.make_case(fine).grid
        got = ic.Apply(fgrid, fine)
        want = vtk_remap.remap(src, ni, nj, L, M, fine.gamma)
        np.testing.assert_array_equal(got, want)
    s2 = pkg.GpuSolver(fine, fgrid, ic, precision="fast")
    r = s2.run(T=1e300, dt=0.0, adaptive=True, max_steps=50)
    assert r.steps == 50 and r.status == 0
    s2.close()


@pytest.mark.parametrize("precision,engine", [("fast", "graph"), ("fast", "persistent"),
                                              ("exact", "graph")])
def test_blowup_is_flagged_nonfinite(pkg, precision, engine):
    """A CFL number far above 1 makes the scheme blow up; the step whose new
    state has the first Inf/NaN wave speed (overflow, or a negative energy
    before any conserved value overflows) stops the run with
    MPD_ERR_NONFINITE, the same step in every engine."""
    case = cases.channel_case(L=48, M=20, cfl=40.0)
    cfg = case.cfg
    s = pkg.GpuSolver(cfg, case.grid, case.phys, precision=precision)
    res = s.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=5000, engine=engine)
    assert res.status == pkg._native.MPD_ERR_NONFINITE
    assert 1 < res.steps < 5000
    s.close()
    if precision == "fast" and engine == "persistent":
        g = pkg.GpuSolver(cfg, case.grid, case.phys, precision="fast")
        rg = g.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=5000, engine="graph")
        assert rg.steps == res.steps
        g.close()


def test_profiling_launches_leave_the_run_unchanged(pkg):
    """mpd_profile_kernel (back-to-back timing launches of the interior kernels
    and the residual pass) between two runs: the run that follows ends in
    the same bits, dt and t as one never interrupted."""
    case = cases.channel_case(L=200, M=80, a=0.1)
    cfg = case.cfg
    a = pkg.GpuSolver(cfg, case.grid, case.phys, precision="fast")
    b = pkg.GpuSolver(cfg, case.grid, case.phys, precision="fast")
    ra = a.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=30)
    rb = b.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=30)
    for which in ("interior", "interior_pair", "residual"):
        assert b.profile_kernel(which, 5, rb.dt) > 0.0
    ra = a.run(T=1e300, dt=ra.dt, adaptive=True, max_steps=40)
    rb = b.run(T=1e300, dt=rb.dt, adaptive=True, max_steps=40)
    assert (ra.t, ra.dt) == (rb.t, rb.dt)
    np.testing.assert_array_equal(a.conserved(), b.conserved())
    a.close()
    b.close()
