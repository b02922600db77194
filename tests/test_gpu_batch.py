"""Batched solves (mpd_batch_run): every solve of a batch must take exactly the
steps, dt and residual schedule of its own GpuSolver.run and end in the same
bits, whatever the team plan."""
import numpy as np
import pytest

from tests import cases

pytestmark = pytest.mark.gpu

RUN = dict(T=1e300, adaptive=True, max_steps=300, residual_every=10)


def _configs():
    return [cases.channel_config(L=24, M=12, a=0.1),
            cases.channel_config(L=40, M=16, vz=0.2),
            cases.channel_config(L=64, M=30, beta=0.3, amp=1.5),
            cases.channel_config(L=32, M=20, a=0.05)]


def _solo(pkg, cfg, **run):
    s = pkg.build_case(cfg, precision="fast")
    r = s.run(dt=cfg.dt, engine="graph", **run)
    out = (r, s.conserved())
    s.close()
    return out


def _check(pkg, cfgs, plan, solo, **run):
    solvers = [pkg.build_case(c, precision="fast") for c in cfgs]
    batch = pkg.BatchSolver(solvers)
    res = batch.run(plan, **run)
    for i, (r, state) in enumerate(solo):
        g = res.runs[i]
        assert (g.steps, g.t, g.dt, g.max_wave_speed, g.converged) == \
            (r.steps, r.t, r.dt, r.max_wave_speed, r.converged), i
        assert g.residual == r.residual, i
        np.testing.assert_array_equal(solvers[i].conserved(), state)
    assert np.all(np.isfinite(res.solve_ms)) and res.device_ms > 0
    batch.close()
    for s in solvers:
        s.close()
    return res


@pytest.mark.parametrize("team_blocks,solve_team", [
    ([1, 1, 1, 1], [0, 1, 2, 3]),      # one-block teams (__syncthreads barriers)
    ([3, 2], [0, 1, 0, 1]),            # multi-block teams, two solves each
    ([5], [0, 0, 0, 0]),               # one team runs every solve in turn
])
def test_batch_matches_individual_runs(pkg, team_blocks, solve_team):
    cfgs = _configs()
    solo = [_solo(pkg, c, **RUN) for c in cfgs]
    plan = pkg.BatchPlan(team_blocks, solve_team)
    # 70 steps per launch: several launches, solves resumed mid-run
    _check(pkg, cfgs, plan, solo, max_steps=300, residual_every=10, steps_per_launch=70)


def test_batch_residual_stop_matches(pkg):
    cfgs = [cases.channel_config(L=40, M=16), cases.channel_config(L=24, M=12, vz=0.25)]
    run = dict(T=1e300, adaptive=True, max_steps=200000, residual_tol=1e-5, residual_every=20)
    solo = [_solo(pkg, c, **run) for c in cfgs]
    assert all(r.converged for r, _ in solo)
    _check(pkg, cfgs, pkg.BatchPlan([2, 1], [0, 1]), solo, max_steps=200000, residual_tol=1e-5,
           residual_every=20)


def test_autotuned_plan_fits_and_matches(pkg):
    cfgs = _configs() + [cases.channel_config(L=24, M=12, beta=0.5)]
    solvers = [pkg.build_case(c, precision="fast") for c in cfgs]
    batch = pkg.BatchSolver(solvers)
    tuner = pkg.Autotuner(batch.capacity, steps=50)
    plan = tuner.plan(cfgs, max_steps=300)
    assert plan.blocks <= batch.capacity
    assert len(plan.solve_team) == len(cfgs)
    assert set(plan.solve_team) == set(range(len(plan.team_blocks)))
    batch.close()
    for s in solvers:
        s.close()
    solo = [_solo(pkg, c, **RUN) for c in cfgs]
    _check(pkg, cfgs, plan, solo, max_steps=300, residual_every=10)


def test_batch_rejects_bad_plans(pkg):
    cfgs = _configs()[:2]
    solvers = [pkg.build_case(c, precision="fast") for c in cfgs]
    batch = pkg.BatchSolver(solvers)
    with pytest.raises(pkg._native.MpdError):
        batch.run(pkg.BatchPlan([batch.capacity + 1], [0, 0]))
    with pytest.raises(pkg._native.MpdError):
        batch.run(pkg.BatchPlan([1], [0, 1]))
    batch.close()
    exact = pkg.build_case(cfgs[0], precision="exact")
    with pytest.raises(pkg._native.MpdError):
        pkg.BatchSolver([exact])
    exact.close()
    for s in solvers:
        s.close()


def test_batch_matches_oracle_directly(pkg):
    """Each solve of a batch against the oracle's own driver loop (not only
    against solo GPU runs): three uneven channel grids, 400 adaptive steps in
    launches of 150, every conserved plane within 1e-12 relative L-inf and the
    same simulated time."""
    from oracle import bind
    cfgs = [cases.channel_config(L=48, M=20, a=0.1),
            cases.channel_config(L=100, M=40, vz=0.2, beta=0.3),
            cases.channel_config(L=64, M=30, amp=1.5, a=0.15)]
    solvers = [pkg.build_case(c, precision="fast") for c in cfgs]
    batch = pkg.BatchSolver(solvers)
    res = batch.run(pkg.BatchPlan([2, 1], [0, 1, 0]), T=1e300, adaptive=True, max_steps=400,
                    steps_per_launch=150)
    for i, cfg in enumerate(cfgs):
        assert res.runs[i].steps == 400
        case = cases.make_case(cfg)
        o = bind.Port(case.oracle_dict())
        ran = o.run(1e300, cfg.dt, True, cfg.cfl_number, cfg.dt_growth_factor, cfg.dt_min,
                    cfg.dt_max, max_steps=400)
        assert ran["steps"] == 400
        assert abs(res.runs[i].t - ran["t"]) <= 1e-12 * ran["t"], i
        got, want = solvers[i].conserved(), o.conserved()
        for k in range(8):
            den = np.abs(want[k]).max()
            assert np.abs(got[k] - want[k]).max() <= 1e-12 * (den if den > 0 else 1.0), (i, k)
        o.close()
    batch.close()
    for s in solvers:
        s.close()
