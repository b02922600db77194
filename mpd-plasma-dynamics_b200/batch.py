"""Batched steady-state solves: many solves of uneven grid sizes and
parameters in one persistent cooperative launch (``mpd_batch_run``), with
team sizes chosen by an autotuner.

The reference runs one solve per process (src/main.cpp).  Here each solve is
a ``GpuSolver`` (fast precision); a batch runs them together: team k of
``team_blocks[k]`` resident blocks runs the solves assigned to it one after
the other, each exactly as ``GpuSolver.run`` would (same steps, dt and
residual schedule, same bits).

Autotuner: for every grid shape in the batch it times a scratch solve of that
shape on a team of each candidate size (a one-team batch, CUDA events), then
packs the batch: per shape a team size and a team count, grown greedily on
the shape whose estimated finish time is latest (more teams, skipping counts
that leave the most-loaded team's share unchanged, or larger teams, whichever
shortens that finish most per block), within one cooperative wave.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math

import numpy as np

from . import _native as N
from .solver import GpuSolver, RunResult, build_case

# Team sizes the autotuner times.  Large grids keep gaining past 64 blocks
# (B200, one 800x320 solve: 50.6 us a step on 64 blocks, 33.8 on 128; 400x160:
# 25.0 and 20.0); small ones stop at their interior task count.
CANDIDATE_BLOCKS = (1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256)


@dataclasses.dataclass
class BatchPlan:
    team_blocks: list[int]
    solve_team: list[int]

    @property
    def blocks(self) -> int:
        return int(sum(self.team_blocks))


@dataclasses.dataclass
class BatchResult:
    runs: list[RunResult]
    solve_ms: np.ndarray      # per solve: first step of the batch -> its last step
    device_ms: float          # the whole batch run

    @property
    def converged(self) -> np.ndarray:
        return np.array([r.converged for r in self.runs])


def _params(T, dt, adaptive, cfl, growth, dt_min, dt_max, max_steps, residual_tol,
            residual_every, steps_per_launch) -> N.RunParams:
    p = N.RunParams()
    p.T, p.dt, p.adaptive = T, dt, int(adaptive)
    p.cfl_number, p.dt_growth_factor, p.dt_min, p.dt_max = cfl, growth, dt_min, dt_max
    p.convergence_threshold = 0.0
    p.check_frequency = 0
    p.residual_tol = residual_tol
    p.residual_every = residual_every
    p.max_steps = int(max_steps)
    p.steps_per_graph = int(steps_per_launch)
    p.engine = N.ENGINE_AUTO
    return p


class BatchSolver:
    """A batch over existing fast-precision ``GpuSolver`` objects (kept alive
    by the batch).  All solves share the run parameters of ``run``; their
    configs carry the physics, grid, geometry, initial and boundary data."""

    def __init__(self, solvers: list[GpuSolver]):
        if not solvers:
            raise ValueError("a batch needs at least one solver")
        self.lib = N.load()
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(solvers))(*[s.h.value if hasattr(s.h, "value") else s.h
                                           for s in solvers])
        h = C.c_void_p()
        N.check(self.lib.mpd_batch_create(arr, len(solvers), C.byref(h)), self.lib)
        self.h = h
        cap = C.c_int()
        N.check(self.lib.mpd_batch_capacity(self.h, C.byref(cap)), self.lib)
        self.capacity = cap.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.mpd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, plan: BatchPlan, T: float = 1e300, dt: float | None = None,
            adaptive: bool = True, max_steps: int = 200_000, residual_tol: float = 0.0,
            residual_every: int = 50, steps_per_launch: int = 0,
            dt_per_solve=None) -> BatchResult:
        """dt: initial dt of every solve (None: the first solver's config dt;
        <= 0: the CFL limit of each solve's state); dt_per_solve overrides it
        per solve."""
        cfg = self.solvers[0].cfg
        p = _params(T, cfg.dt if dt is None else dt, adaptive, cfg.cfl_number,
                    cfg.dt_growth_factor, cfg.dt_min, cfg.dt_max, max_steps, residual_tol,
                    residual_every, steps_per_launch)
        n = len(self.solvers)
        if len(plan.solve_team) != n:
            raise ValueError("plan.solve_team needs one entry per solve")
        tb = (C.c_int * len(plan.team_blocks))(*plan.team_blocks)
        st = (C.c_int * n)(*plan.solve_team)
        stats = (N.RunStats * n)()
        solve_ms = np.zeros(n)
        dev_ms = C.c_double()
        dts = None
        if dt_per_solve is not None:
            dts = np.ascontiguousarray(dt_per_solve, dtype=np.float64)
            if dts.shape != (n,):
                raise ValueError("dt_per_solve needs one entry per solve")
        rc = self.lib.mpd_batch_run(self.h, C.byref(p), len(plan.team_blocks), tb, st,
                                    dts.ctypes.data_as(N.DP) if dts is not None else None,
                                    stats, solve_ms.ctypes.data_as(N.DP), C.byref(dev_ms))
        if rc not in (N.MPD_OK, N.MPD_ERR_NONFINITE):
            N.check(rc, self.lib)
        runs = [RunResult(s.steps, s.t, s.dt, s.residual, s.change, s.max_wave_speed,
                          bool(s.converged), s.status, s.device_ms) for s in stats]
        return BatchResult(runs, solve_ms, dev_ms.value)


def estimated_steps(cfg, max_steps: int) -> int:
    """Steps a cold start of the channel needs to reach an L-inf residual of
    1e-8, capped at max_steps.  The LF scheme's numerical viscosity makes the
    slowest mode decay over ~L^2 steps: 39.5k steps at 100x40 and 158k at
    200x80 for the straight channel (measured with the oracle), so 4 L^2."""
    return int(min(max_steps, 4 * cfg.L_max ** 2))


# Steps a surrogate-warm start of the channel takes to the same residual, per
# grid row: the medians of the uneven sweep's warm solves on a B200 were
# 2,951 / 8,651 / 11,551 / 26,551 steps at L = 100 / 200 / 400 / 800, about
# 33 L (against the cold start's 4 L^2).  Only the batch plan uses it.
WARM_STEPS_PER_ROW = 33


def estimated_warm_steps(cfg, max_steps: int) -> int:
    """Steps a surrogate-warm start needs (WARM_STEPS_PER_ROW L), capped at
    max_steps: the batch plan's estimate for warm solves, which the cold law
    (estimated_steps) overstates by 10-100x, the more so the finer the grid."""
    return int(min(max_steps, WARM_STEPS_PER_ROW * cfg.L_max))


class Autotuner:
    """Team sizes per grid shape from measured step times."""

    def __init__(self, capacity: int, candidates=CANDIDATE_BLOCKS, steps: int = 200):
        self.capacity = capacity
        self.candidates = [c for c in candidates if c <= capacity]
        self.steps = steps
        self.table: dict[tuple[int, int], dict[int, float]] = {}

    def time_shape(self, cfg) -> dict[int, float]:
        """Microseconds per step of a solve of cfg's shape on each candidate team."""
        key = (cfg.L_max, cfg.M_max)
        if key in self.table:
            return self.table[key]
        s = build_case(cfg, precision="fast")
        b = BatchSolver([s])
        out = {}
        s.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=2)   # first step, warm
        for blocks in self.candidates:
            if blocks * 4 > max(1, (cfg.M_max + 29) // 30) * max(1, cfg.L_max):
                break   # more warps than interior tasks (strips x one-row bands)
            plan = BatchPlan([blocks], [0])
            b.run(plan, max_steps=10, residual_every=0)
            r = b.run(plan, max_steps=self.steps, residual_every=0)
            out[blocks] = r.device_ms * 1e3 / max(1, r.runs[0].steps)
        b.close()
        s.close()
        self.table[key] = out
        return out

    def plan(self, cfgs, max_steps: int, estimate=estimated_steps) -> BatchPlan:
        """Teams per grid shape.  estimate(cfg, max_steps): the steps a solve
        is expected to take (cold law by default; estimated_warm_steps for
        warm starts)."""
        shapes: dict[tuple[int, int], list[int]] = {}
        for i, c in enumerate(cfgs):
            shapes.setdefault((c.L_max, c.M_max), []).append(i)
        timing = {k: self.time_shape(cfgs[v[0]]) for k, v in shapes.items()}
        steps = {k: max(estimate(cfgs[i], max_steps) for i in v) for k, v in shapes.items()}
        # start: the block-efficient size (most cell-steps per block-second), one team
        state = {}
        for k, tab in timing.items():
            cells = k[0] * (k[1] + 1)
            best = max(tab, key=lambda b: cells / (tab[b] * b))
            state[k] = [best, 1]
        used = sum(b * t for b, t in state.values())
        if used > self.capacity:
            raise ValueError("the batch's shapes need more blocks than one wave holds")

        def finish(k, blocks, teams):
            return math.ceil(len(shapes[k]) / teams) * steps[k] * timing[k][blocks]

        while True:
            k = max(state, key=lambda s: finish(s, *state[s]))
            blocks, teams = state[k]
            n = len(shapes[k])
            now = finish(k, blocks, teams)
            free = self.capacity - used
            options = []
            per = math.ceil(n / teams)
            if per > 1:
                # the fewest teams that leave each at most per - 1 solves: adding
                # fewer changes nothing (ceil(n / teams) is flat in between)
                nt = math.ceil(n / (per - 1))
                if (nt - teams) * blocks <= free:
                    options.append((now - finish(k, blocks, nt), (nt - teams) * blocks,
                                    (blocks, nt)))
            for nb in timing[k]:
                if nb > blocks and (nb - blocks) * teams <= free:
                    options.append((now - finish(k, nb, teams), (nb - blocks) * teams, (nb, teams)))
            options = [o for o in options if o[0] > 0]
            if not options:
                break
            gain, cost, new = max(options, key=lambda o: o[0] / o[1])
            used += cost
            state[k] = list(new)
        team_blocks, solve_team = [], [0] * len(cfgs)
        for k, idx in shapes.items():
            blocks, teams = state[k]
            first = len(team_blocks)
            team_blocks += [blocks] * teams
            for j, i in enumerate(idx):
                solve_team[i] = first + j % teams
        return BatchPlan(team_blocks, solve_team)
