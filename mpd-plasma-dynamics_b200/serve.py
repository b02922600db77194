"""Large grid plus a serving mix: one large solve
warm-started from the surrogate's coarse prediction, remapped onto its grid
by the device bilinear remap, running in the same persistent cooperative
launch as a batch of small uneven solves admitted by a device-memory budget.

large_grid_error measures what the warm start is worth against the plain
method's steady state on a large converging-diverging channel whose cold
steady state is reachable (the 4096 x 1600 one needs ~4 L^2 = 67M steps):
per-field relative L-inf distance to the cold-started steady state of the
surrogate's remapped prediction, of the warm run after a serving cap of
steps, and of the warm run converged; the cold run's own distance after the
same cap for comparison.  When the cold start has no steady state (the
channel with a = 0.3 diverges from the uniform initial condition under this
scheme: its density grows without bound until the state is non-finite,
the reference's own arithmetic included), the distances are taken to the
steady state the plain march converges to from the prediction instead, and
the record says which reference it used.

The large solve gets a team of `big_blocks` blocks; the small ones are
admitted in draw order while their estimated device bytes fit the budget
(free device memory x `budget_frac`, less the large solve), and take the
remaining blocks of the wave in autotuned teams.
"""
from __future__ import annotations

import time

import numpy as np

from . import surrogate as S
from . import warmstart as WS
from .batch import Autotuner, BatchPlan, BatchSolver
from .io import snapshot_arrays
from .solver import GpuSolver, build_case
from .workloads import SweepParams, sweep_params


def solve_bytes(cfg) -> int:
    """Device bytes of one fast solver: 2 x 8 state planes, 10 initial
    planes, lines and profiles (pitch rounded to 32 doubles)."""
    pitch = (cfg.M_max + 3 + 31) // 32 * 32
    plane = (cfg.L_max + 2) * pitch * 8
    return 26 * plane + 64 * (cfg.L_max + cfg.M_max + 8) * 8


def upsampled_ic(tr: WS.Trained, p: SweepParams, big_cfg) -> np.ndarray:
    """The surrogate's prediction on its own grid for draw p (geometry of
    p), as snapshot points, remapped onto big_cfg's grid on the device."""
    import ctypes as C
    import torch
    from . import _native as N
    H, W = tr.net.H, tr.net.W
    L, M = H, W - 1
    small = SweepParams(L, M, p.amp, p.beta, p.vz, p.a)
    scfg = small.config()
    grid = WS.grid_of(scfg)
    pred, _ = WS.predict(tr, WS.inputs_of(small, grid)[None])
    floor = np.array([1e-3, 1e-4])
    phys = WS.planes_from_fields(pred[0].reshape(H, W, S.N_OUT), scfg, floor)
    arr = snapshot_arrays(phys, grid.r, L, M)
    v, h = arr["Velocity"].reshape(-1, 3), arr["MagneticField"].reshape(-1, 3)
    src = np.stack([arr["Rho"].reshape(-1), v[:, 0], v[:, 1], v[:, 2], h[:, 0], h[:, 1],
                    h[:, 2], arr["Energy"].reshape(-1)])
    lib = N.load()
    dsrc = torch.from_numpy(np.ascontiguousarray(src)).cuda()
    out = torch.zeros((10, big_cfg.L_max + 2, big_cfg.M_max + 3), dtype=torch.float64,
                      device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    N.check(lib.mpd_remap_snapshot(C.c_void_p(dsrc.data_ptr()), L + 1, M + 1, big_cfg.L_max,
                                   big_cfg.M_max, float(big_cfg.gamma),
                                   C.c_void_p(out.data_ptr()), stream), lib)
    return out.cpu().numpy()


def run_serving(tr: WS.Trained, big: tuple[int, int] = (4096, 1600), a_big: float = 0.3,
                n_small: int = 128, big_blocks: int = 296, max_steps: int = 20_000,
                tol: float = 1e-8, budget_frac: float = 0.8, log=print) -> dict:
    import torch
    big_p = SweepParams(big[0], big[1], 1.0, 0.1, 0.1, a_big)
    big_cfg = big_p.config()
    t0 = time.perf_counter()
    ic = upsampled_ic(tr, big_p, big_cfg)
    remap_s = time.perf_counter() - t0
    free, _ = torch.cuda.mem_get_info()
    budget = int(free * budget_frac) - solve_bytes(big_cfg)
    small_p, used = [], 0
    for i in range(n_small):
        p = sweep_params(2_000_000 + i)
        need = solve_bytes(p.config())
        if used + need > budget:
            break
        small_p.append(p)
        used += need
    log(f"admitted {len(small_p)} of {n_small} small solves ({used / 2**30:.2f} GiB of "
        f"{budget / 2**30:.2f} GiB budget)")

    out = {}
    for mode in ("warm", "cold"):
        big_s = (GpuSolver(big_cfg, WS.grid_of(big_cfg), ic, precision="fast") if mode == "warm"
                 else build_case(big_cfg, precision="fast"))
        small_cfgs = [p.config() for p in small_p]
        smalls = [build_case(c, precision="fast") for c in small_cfgs]
        batch = BatchSolver([big_s] + smalls)
        tuner = Autotuner(batch.capacity - big_blocks, steps=100)
        sub = tuner.plan(small_cfgs, max_steps=max_steps)
        plan = BatchPlan([big_blocks] + sub.team_blocks, [0] + [t + 1 for t in sub.solve_team])
        # a warm large solve starts at the CFL dt of its state; everything
        # cold starts at the workload's dt0
        dts = [0.0 if mode == "warm" else big_cfg.dt] + [c.dt for c in small_cfgs]
        res = batch.run(plan, max_steps=max_steps, residual_tol=tol, residual_every=50,
                        dt_per_solve=dts)
        r_big = res.runs[0]
        small_runs = res.runs[1:]
        conv = np.array([r.converged for r in small_runs])
        out[mode] = {
            "big_steps": r_big.steps, "big_residual": r_big.residual,
            "big_converged": r_big.converged, "device_ms": res.device_ms,
            "small_converged": int(conv.sum()),
            "small_solves_per_s": len(small_runs) / (res.device_ms * 1e-3),
            "small_p50_ms": float(np.percentile(res.solve_ms[1:], 50)),
            "small_p99_ms": float(np.percentile(res.solve_ms[1:], 99)),
            "teams": len(plan.team_blocks), "blocks": plan.blocks,
        }
        log(f"{mode}: big residual {r_big.residual:.3e} after {r_big.steps} steps; small "
            f"{int(conv.sum())}/{len(small_runs)} converged, {res.device_ms / 1e3:.1f} s")
        batch.close()
        big_s.close()
        for s in smalls:
            s.close()
    return {"big_grid": f"{big[0]}x{big[1]}", "a_big": a_big, "n_small_admitted": len(small_p),
            "budget_gib": budget / 2**30, "remap_s": remap_s, "max_steps": max_steps, **out}


def large_grid_error(tr: WS.Trained, grid: tuple[int, int] = (800, 320), a_big: float = 0.3,
                     cap: int = 20_000, max_steps: int = 8_000_000, tol: float = 1e-8,
                     log=print) -> dict:
    """See the module docstring.  Both runs use the graph engine with the
    residual every 50 steps; the warm one starts at the CFL dt of the
    remapped prediction, the cold one at the workload's dt0."""
    L, M = grid
    p = SweepParams(L, M, 1.0, 0.1, 0.1, a_big)
    cfg = p.config()

    def fields(solver):
        return WS.fields_of(solver.physical(), L, M)

    cold = build_case(cfg, precision="fast")
    c1 = cold.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=cap, residual_tol=tol,
                  residual_every=50)
    cold_cap = fields(cold)
    c2 = cold.run(T=1e300, dt=c1.dt, adaptive=True, max_steps=max_steps - c1.steps,
                  residual_tol=tol, residual_every=50)
    ref = fields(cold)
    cold.close()
    log(f"cold {L}x{M} a={a_big}: converged={c2.converged} after {c1.steps + c2.steps} steps, "
        f"residual {c2.residual:.2e}")
    ic = upsampled_ic(tr, p, cfg)
    pred = WS.fields_of(ic, L, M)
    warm = GpuSolver(cfg, WS.grid_of(cfg), ic, precision="fast")
    w1 = warm.run(T=1e300, dt=0.0, adaptive=True, max_steps=cap, residual_tol=tol,
                  residual_every=50)
    warm_cap = fields(warm)
    w2 = warm.run(T=1e300, dt=w1.dt, adaptive=True, max_steps=max_steps - w1.steps,
                  residual_tol=tol, residual_every=50)
    warm_conv = fields(warm)
    warm.close()
    log(f"warm: converged={w2.converged} after {w1.steps + w2.steps} steps")

    if not c2.converged and w2.converged:
        ref = warm_conv
        ref_name = "warm-started steady state (the cold start did not converge)"
    else:
        ref_name = "cold-started steady state"

    def per_field(x):
        return dict(zip(S.FIELDS, WS.relative_linf(x, ref).tolist()))

    return {
        "grid": f"{L}x{M}", "a": a_big, "tol": tol, "cap_steps": cap, "reference": ref_name,
        "cold_steps": int(c1.steps + c2.steps), "cold_converged": bool(c2.converged),
        "cold_status": "non-finite" if c2.status else "ok", "cold_final_residual": c2.residual,
        "cold_device_s": (c1.device_ms + c2.device_ms) * 1e-3,
        "warm_steps": int(w1.steps + w2.steps), "warm_converged": bool(w2.converged),
        "warm_device_s": (w1.device_ms + w2.device_ms) * 1e-3,
        "residual_at_cap": {"cold": c1.residual, "warm": w1.residual},
        "rel_linf_vs_cold_steady": {
            "prediction": per_field(pred),
            "warm_at_cap": per_field(warm_cap),
            "cold_at_cap": per_field(cold_cap),
            "warm_converged": per_field(warm_conv),
        },
    }
