"""The batch autotuner's packing (Autotuner.plan) on given step-time tables:
host logic only, no GPU (the tables stand in for the measured ones)."""
import math
import types

import pytest


def _cfg(L, M):
    return types.SimpleNamespace(L_max=L, M_max=M)


def _tuner(pkg, capacity, table):
    t = pkg.Autotuner(capacity)
    t.table = dict(table)
    return t


def _makespan(plan, cfgs, table, steps):
    load = {}
    for i, team in enumerate(plan.solve_team):
        c = cfgs[i]
        us = table[(c.L_max, c.M_max)][plan.team_blocks[team]]
        load[team] = load.get(team, 0.0) + steps(c) * us
    return max(load.values())


# step times (us) that shrink with the team size, as measured shapes do
TABLE = {
    (100, 40): {1: 20.0, 2: 19.0, 4: 18.5},
    (200, 80): {1: 30.0, 2: 22.0, 4: 19.0, 8: 18.0},
    (400, 160): {1: 90.0, 2: 50.0, 4: 30.0, 8: 22.0, 16: 20.0},
    (800, 320): {1: 340.0, 2: 175.0, 4: 95.0, 8: 55.0, 16: 33.0, 32: 24.0},
}


def _batch(n_per_shape):
    return [_cfg(*k) for k in TABLE for _ in range(n_per_shape)]


def test_plan_assigns_every_solve_within_capacity(pkg):
    cfgs = _batch(16)
    plan = _tuner(pkg, 444, TABLE).plan(cfgs, max_steps=20000)
    assert len(plan.solve_team) == len(cfgs)
    assert set(plan.solve_team) == set(range(len(plan.team_blocks)))
    assert plan.blocks <= 444
    # a team runs solves of one shape only
    for team in range(len(plan.team_blocks)):
        shapes = {(cfgs[i].L_max, cfgs[i].M_max) for i, t in enumerate(plan.solve_team) if t == team}
        assert len(shapes) == 1


def test_plan_passes_plateaus_of_the_team_count(pkg):
    """16 solves on 4 teams and on 5 teams finish at the same time (4 rounds
    each); the packer must not stop there while blocks are free."""
    cfgs = _batch(16)
    plan = _tuner(pkg, 444, TABLE).plan(cfgs, max_steps=20000)
    steps = lambda c: pkg.batch.estimated_steps(c, 20000)
    span = _makespan(plan, cfgs, TABLE, steps)
    # every solve of the slowest shape on a team of its own, at least
    teams_800 = {plan.solve_team[i] for i, c in enumerate(cfgs) if c.L_max == 800}
    assert len(teams_800) == 16
    # no better than one round of the largest shape on its best team size
    assert span >= 20000 * 24.0
    assert plan.blocks > 300  # the wave is used, not left mostly idle


def test_plan_is_no_worse_than_one_block_per_solve(pkg):
    cfgs = _batch(8)
    steps = lambda c: pkg.batch.estimated_steps(c, 20000)
    plan = _tuner(pkg, 444, TABLE).plan(cfgs, max_steps=20000)
    naive = pkg.BatchPlan([1] * len(cfgs), list(range(len(cfgs))))
    assert _makespan(plan, cfgs, TABLE, steps) <= _makespan(naive, cfgs, TABLE, steps)


def test_plan_rejects_shapes_beyond_one_wave(pkg):
    cfgs = _batch(1)
    with pytest.raises(ValueError):
        _tuner(pkg, 3, TABLE).plan(cfgs, max_steps=20000)


def test_warm_estimate_plans_for_the_warm_makespan(pkg):
    """Warm solves take about 33 L steps, not the cold 4 L^2: planned with
    the warm estimate, the batch's makespan under warm step counts is no
    worse than the cold law's plan, and strictly better at a large cap."""
    cfgs = _batch(16)
    cap = 2_500_000
    warm = lambda c: pkg.batch.estimated_warm_steps(c, cap)
    assert [warm(_cfg(*k)) for k in TABLE] == [3300, 6600, 13200, 26400]
    tuner = _tuner(pkg, 444, TABLE)
    plan_cold = tuner.plan(cfgs, max_steps=cap)
    plan_warm = tuner.plan(cfgs, max_steps=cap, estimate=pkg.batch.estimated_warm_steps)
    span_cold = _makespan(plan_cold, cfgs, TABLE, warm)
    span_warm = _makespan(plan_warm, cfgs, TABLE, warm)
    assert span_warm < span_cold
