"""Learned warm start of steady-state solves: data generation with the batched
solver, surrogate training on the GPU, and the warm-versus-cold comparison.

Pipeline:
  1. steady states of the channel for parameter draws of the sweep box
     (workloads.sweep_params on one grid), solved by BatchSolver until the
     L-inf residual is <= tol (max max_steps steps);
  2. the spectral operator (surrogate.SpectralOperator) trained on them:
     inputs = parameters + (r, z), targets = the 8 primitive fields
     normalised per field, Adam, mean squared error;
  3. held-out draws solved twice by BatchSolver: from the initial condition
     of the workload (cold) and from the surrogate's prediction (warm);
     steps to converge, solves per second and the surrogate's own L-inf error
     against the converged state are reported.  The plain time march stays
     the judge and the fallback: a warm solve is accepted only at residual
     <= tol within its step budget; a non-finite prediction, or a warm solve
     that ends non-finite or unconverged within the budget, is solved again
     from the cold initial condition (solve_warm).

On a fine grid the training data itself is generated warm (bootstrap): a
surrogate trained on a coarse grid predicts each fine training draw, the
prediction is interpolated bilinearly onto the fine grid, and the plain march
converges from it (with the same fallback).  run_pipeline does all of it in
one call; build_surrogate and evaluate split it in two.
"""
from __future__ import annotations

import dataclasses
import math
import time

import numpy as np

from . import _native as N
from . import surrogate as S
from .batch import Autotuner, BatchPlan, BatchSolver, estimated_steps, estimated_warm_steps
from .geometry import GeometryRegistry, Grid
from .ic import ArrayIC, derived_pressures
from .solver import GpuSolver, build_case
from .workloads import SweepParams, sweep_params

# physical plane index of each network field (rho, v_z, v_r, v_phi, e, H_z, H_r, H_phi)
PLANE_OF_FIELD = (0, 1, 2, 3, 4, 7, 8, 9)


def draws(seeds, grid, a_max: float = 0.2):
    return [sweep_params(int(s), grids=(grid,), a_max=a_max) for s in seeds]


def grid_of(cfg) -> Grid:
    geom = GeometryRegistry.Instance().Create(cfg.geometry.type, cfg.geometry.params)
    return Grid(cfg, geom)


def inputs_of(p: SweepParams, grid: Grid) -> np.ndarray:
    cfg = grid.cfg
    L, M = cfg.L_max, cfg.M_max
    r = grid.r[1:L + 1, 1:M + 2]
    z = (np.arange(1, L + 1) - 1) * cfg.dz
    return S.features(S.param_vector(p.amp, p.beta, p.vz, p.a), r, z)


def own_inputs(p: SweepParams) -> np.ndarray:
    """The network input of draw p on its own grid and wall."""
    return inputs_of(p, grid_of(p.config()))


def fields_of(phys10: np.ndarray, L: int, M: int) -> np.ndarray:
    """H x W x 8 network fields from the 10 physical planes."""
    return np.stack([phys10[k, 1:L + 1, 1:M + 2] for k in PLANE_OF_FIELD], axis=-1)


def planes_from_fields(f: np.ndarray, cfg, floor: np.ndarray) -> np.ndarray:
    """10 physical planes from H x W x 8 predicted fields (density and energy
    kept above `floor`), p and P derived as ExpressionIC derives them."""
    L, M = cfg.L_max, cfg.M_max
    phys = np.zeros((10, L + 2, M + 3))
    for j, k in enumerate(PLANE_OF_FIELD):
        phys[k, 1:L + 1, 1:M + 2] = f[..., j]
    phys[0] = np.maximum(phys[0], floor[0])
    phys[4] = np.maximum(phys[4], floor[1])
    derived_pressures(phys, cfg.gamma)
    return phys


@dataclasses.dataclass
class SolveSet:
    steps: np.ndarray
    converged: np.ndarray
    residual: np.ndarray
    fields: list            # H x W x 8 per solve (final state)
    device_ms: float        # sum over the batch launches
    solve_ms: np.ndarray


def solve_all(params: list[SweepParams], ics: list | None = None, max_steps=200_000, tol=1e-8,
              every=50, chunk: int = 256, tuner: Autotuner | None = None,
              estimate=None) -> SolveSet:
    """Solve every draw with the batched engine, in batches of at most `chunk`
    solves, from the workload's initial condition (the workload's dt0) or,
    with ics, from the given planes starting at their CFL dt: the LF steady
    state depends on dt, so a warm start that ramps dt up from dt0 would
    leave the steady state it was given."""
    n = len(params)
    steps = np.zeros(n, dtype=np.int64)
    conv = np.zeros(n, dtype=bool)
    res = np.full(n, np.nan)
    fields = [None] * n
    solve_ms = np.zeros(n)
    dev_ms = 0.0
    for i0 in range(0, n, chunk):
        part = params[i0:i0 + chunk]
        cfgs = [p.config() for p in part]
        solvers = []
        for k, cfg in enumerate(cfgs):
            ic = ics[i0 + k] if ics is not None else None
            if ic is None:
                solvers.append(build_case(cfg, precision="fast"))
            else:
                solvers.append(GpuSolver(cfg, grid_of(cfg), ic, precision="fast"))
        batch = BatchSolver(solvers)
        tuner = tuner or Autotuner(batch.capacity, steps=100)
        if estimate is None:
            estimate = estimated_steps if ics is None else estimated_warm_steps
        plan = tuner.plan(cfgs, max_steps=max_steps, estimate=estimate)
        out = batch.run(plan, dt=None if ics is None else 0.0, max_steps=max_steps,
                        residual_tol=tol, residual_every=every)
        dev_ms += out.device_ms
        for k, (s, r) in enumerate(zip(solvers, out.runs)):
            j = i0 + k
            steps[j], conv[j], res[j] = r.steps, r.converged, r.residual
            solve_ms[j] = out.solve_ms[k]
            fields[j] = fields_of(s.physical(), s.cfg.L_max, s.cfg.M_max)
        batch.close()
        for s in solvers:
            s.close()
    return SolveSet(steps, conv, res, fields, dev_ms, solve_ms)


def upsample_fields(f: np.ndarray, L: int, M: int) -> np.ndarray:
    """Bilinear interpolation of H x W x 8 point fields of a coarse grid
    (points at z = i / H, y = j / (W - 1)) onto the points of an L x M grid
    (z = i / L, y = j / M); rows past the coarse grid's last take its values."""
    Hc, Wc = f.shape[:2]
    zi = np.minimum(np.arange(L) * (Hc / L), Hc - 1)
    yj = np.arange(M + 1) * ((Wc - 1) / M)
    i0 = np.minimum(np.floor(zi).astype(int), Hc - 2) if Hc > 1 else np.zeros(L, int)
    j0 = np.minimum(np.floor(yj).astype(int), Wc - 2)
    wi = (zi - i0)[:, None, None]
    wj = (yj - j0)[None, :, None]
    i1 = np.minimum(i0 + 1, Hc - 1)
    a = f[i0][:, j0] * (1 - wj) + f[i0][:, j0 + 1] * wj
    b = f[i1][:, j0] * (1 - wj) + f[i1][:, j0 + 1] * wj
    return a * (1 - wi) + b * wi


def _empty_set(n: int) -> SolveSet:
    return SolveSet(np.zeros(n, dtype=np.int64), np.zeros(n, dtype=bool), np.full(n, np.nan),
                    [None] * n, 0.0, np.zeros(n))


def solve_warm(params: list[SweepParams], ics: list, max_steps=200_000, tol=1e-8, every=50,
               budget: int | None = None, chunk: int = 256) -> tuple[SolveSet, np.ndarray]:
    """Warm solves judged by the plain march: solve i starts from ics[i]
    (10 physical planes) at its CFL dt and has `budget` steps (default: half
    the cold estimate, estimated_steps) to reach the L-inf residual tol.  A
    missing (None: non-finite) prediction, and a warm solve that ends
    non-finite or unconverged within the budget, is solved again from the
    workload's initial condition with max_steps.  Returns the combined set
    (steps, device and per-solve times of both attempts added) and the mask of
    solves that fell back."""
    n = len(params)
    out = _empty_set(n)
    fell = np.array([ic is None for ic in ics])
    use = np.flatnonzero(~fell)
    if budget is None:
        budget = max(1000, estimated_steps(params[0].config(), max_steps) // 2)
    if len(use):
        w = solve_all([params[i] for i in use], ics=[ics[i] for i in use],
                      max_steps=min(budget, max_steps), tol=tol, every=every, chunk=chunk)
        out.device_ms += w.device_ms
        for k, i in enumerate(use):
            out.steps[i], out.converged[i], out.residual[i] = w.steps[k], w.converged[k], \
                w.residual[k]
            out.fields[i], out.solve_ms[i] = w.fields[k], w.solve_ms[k]
            if not w.converged[k]:
                fell[i] = True
    back = np.flatnonzero(fell)
    if len(back):
        c = solve_all([params[i] for i in back], max_steps=max_steps, tol=tol, every=every,
                      chunk=chunk)
        out.device_ms += c.device_ms
        for k, i in enumerate(back):
            out.steps[i] += c.steps[k]
            out.converged[i], out.residual[i] = c.converged[k], c.residual[k]
            out.fields[i] = c.fields[k]
            out.solve_ms[i] += c.solve_ms[k]
    return out, fell


def predicted_ics(tr: "Trained", params: list[SweepParams], grid, floor) -> tuple[list, float]:
    """Initial planes predicted by the surrogate for each draw on `grid`
    (None: each draw's own grid) — None where the prediction is not finite —
    and the inference seconds.  A surrogate trained on another (coarser)
    grid predicts on its own grid and the prediction is interpolated
    bilinearly."""
    Hs, Ws = tr.net.H, tr.net.W
    X = np.stack([own_inputs(SweepParams(Hs, Ws - 1, p.amp, p.beta, p.vz, p.a))
                  for p in params])
    pred, infer_s = predict(tr, X)
    out = []
    for p, f in zip(params, pred):
        L, M = grid if grid is not None else (p.L, p.M)
        f = f.reshape(Hs, Ws, S.N_OUT)
        if not np.all(np.isfinite(f)):
            out.append(None)
            continue
        if (Hs, Ws) != (L, M + 1):
            f = upsample_fields(f, L, M)
        out.append(planes_from_fields(f, p.config(), floor))
    return out, infer_s


@dataclasses.dataclass
class Trained:
    net: S.SpectralOperator
    norm: S.Normalizer
    losses: list
    train_s: float
    floor: np.ndarray | None = None   # lower bounds of predicted rho and e

    def save(self, path):
        p = self.net.get_params()
        floor = self.floor if self.floor is not None else np.zeros(2)
        np.savez(path, H=self.net.H, W=self.net.W, mean=self.norm.mean, std=self.norm.std,
                 const=self.norm.const, losses=np.array(self.losses), floor=floor,
                 **{f"p_{k}": v.astype(np.float32) for k, v in p.items()})

    @classmethod
    def load(cls, path, batch: int = 16) -> "Trained":
        z = np.load(path)
        params = {k[2:]: z[k] for k in z.files if k.startswith("p_")}
        net = S.SpectralOperator(int(z["H"]), int(z["W"]), batch, params=params)
        norm = S.Normalizer(z["mean"], z["std"], z["const"])
        floor = z["floor"] if "floor" in z.files else None
        return cls(net, norm, list(z["losses"]), 0.0, floor)


def train(X: np.ndarray, Y: np.ndarray, H: int, W: int, epochs: int = 40, batch: int = 16,
          lr: float = 1e-3, seed: int = 0, log=None) -> Trained:
    """X: N x P x 6 inputs, Y: N x P x 8 fields (physical units)."""
    import torch
    norm = S.Normalizer.fit(Y)
    Yn = norm.encode(Y).astype(np.float32)
    dev = torch.device("cuda")
    dX = torch.from_numpy(X.astype(np.float32)).to(dev)
    dY = torch.from_numpy(Yn).to(dev)
    net = S.SpectralOperator(H, W, batch, seed=seed)
    rng = np.random.default_rng(seed)
    N = len(X)
    nb = N // batch
    losses = []
    t0 = time.perf_counter()
    total = epochs * nb
    it = 0
    net.capture()   # forward + loss + backward replayed as one CUDA graph
    for ep in range(epochs):
        perm = torch.from_numpy(rng.permutation(N)[:nb * batch]).to(dev)
        ep_loss = 0.0
        for b in range(nb):
            idx = perm[b * batch:(b + 1) * batch]
            net.x.copy_(dX.index_select(0, idx).reshape(-1, S.N_IN))
            net.target.copy_(dY.index_select(0, idx).reshape(-1, S.N_OUT))
            rate = lr * 0.5 * (1 + math.cos(math.pi * it / total)) + 1e-5
            net.train_step(lr=rate)
            ep_loss += float(net.loss.cpu()[0]) if b == nb - 1 else 0.0
            it += 1
        losses.append(ep_loss)
        if log:
            log(f"epoch {ep} loss {ep_loss:.4e}")
    net.wait()
    return Trained(net, norm, losses, time.perf_counter() - t0)


def predict(tr: Trained, X: np.ndarray) -> tuple[np.ndarray, float]:
    """N x P x 8 fields (physical units) and the device seconds it took."""
    import torch
    net = tr.net
    B = net.B
    N = len(X)
    out = np.zeros((N, X.shape[1], S.N_OUT))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(0, N, B):
        xb = np.zeros((B,) + X.shape[1:], dtype=np.float32)
        k = min(B, N - i)
        xb[:k] = X[i:i + k]
        net.load_inputs(xb)
        y = net.forward()
        out[i:i + k] = y.cpu().numpy().reshape(B, X.shape[1], S.N_OUT)[:k]
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return tr.norm.decode(out), dt


def relative_linf(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per field max |a - b| / max |b|."""
    return np.abs(a - b).reshape(-1, S.N_OUT).max(0) / np.maximum(
        np.abs(b).reshape(-1, S.N_OUT).max(0), 1e-30)


def tight_agreement(params, cold: SolveSet, warm: SolveSet, idx, tol: float,
                    max_steps: int = 200_000) -> tuple[np.ndarray, np.ndarray]:
    """Both converged states of the solves `idx`, driven on to residual `tol`
    from where they stopped (a residual of 1e-8 per step leaves a state about
    1e-5 from the scheme's fixed point, the slowest mode decaying by ~1e-3
    per step): their relative L-inf distance per field (max over the solves)
    and the extra steps the warm ones took."""
    sub = [params[i] for i in idx]
    floor = np.zeros(2)
    def go(sset):
        ics = [planes_from_fields(sset.fields[i], params[i].config(), floor) for i in idx]
        return solve_all(sub, ics=ics, max_steps=max_steps, tol=tol)
    c, w = go(cold), go(warm)
    ok = c.converged & w.converged
    d = [relative_linf(w.fields[k], c.fields[k]) for k in np.flatnonzero(ok)]
    dist = np.stack(d).max(0) if d else np.full(S.N_OUT, np.nan)
    return dist, w.steps


def build_surrogate(n_train=2000, grid=(100, 40), epochs=40, batch=16, lr=1e-3,
                    max_steps=200_000, tol=1e-8, bootstrap=None, n_boot=2000, boot_epochs=60,
                    boot_max_steps=200_000, log=print, save: str | None = None,
                    a_max: float = 0.2) -> tuple[Trained, dict]:
    """Steps 1-2 of the module docstring: training steady states for the
    draws 0 .. n_train-1 of the sweep box on `grid`, and the network trained
    on them.  With bootstrap = a coarser (L, M), the training solves start
    from the prediction of a surrogate first built the same way on that grid
    (n_boot draws), interpolated onto `grid`.  a_max widens the draws' wall
    amplitude range beyond the sweep box's 0.2."""
    L, M = grid
    H, W = L, M + 1
    train_p = draws(range(n_train), grid, a_max)
    info: dict = {"grid": f"{L}x{M}", "n_train": n_train, "epochs": epochs, "a_max": a_max}
    t0 = time.perf_counter()
    if bootstrap and tuple(bootstrap) != tuple(grid):
        coarse, cinfo = build_surrogate(n_boot, tuple(bootstrap), boot_epochs, batch, lr,
                                        max_steps=boot_max_steps, tol=tol, log=log, a_max=a_max)
        info["bootstrap"] = cinfo
        ics, _ = predicted_ics(coarse, train_p, grid, coarse.floor)
        del coarse  # its device buffers go back to the allocator
        data, fell = solve_warm(train_p, ics, max_steps=max_steps, tol=tol, budget=max_steps)
        info["bootstrap_fallbacks"] = int(fell.sum())
    else:
        data = solve_all(train_p, max_steps=max_steps, tol=tol)
    gen_s = time.perf_counter() - t0
    keep = np.flatnonzero(data.converged)
    log(f"training solves on {L}x{M}: {len(keep)} of {n_train} converged, {gen_s:.1f} s")
    # single precision on the host too: 2000 fine-grid states are GBs; each
    # draw's r(z, y) from its own wall (its a)
    X = np.stack([own_inputs(train_p[i]).astype(np.float32) for i in keep])
    Y = np.stack([data.fields[i].reshape(H * W, S.N_OUT).astype(np.float32) for i in keep])
    data_steps_median = float(np.median(data.steps))
    data_device_s = data.device_ms * 1e-3
    del data
    tr = train(X, Y, H, W, epochs=epochs, batch=batch, lr=lr, log=log)
    tr.floor = np.array([0.05 * np.min(Y[..., 0]), 0.05 * np.min(Y[..., 4])])
    log(f"trained {epochs} epochs in {tr.train_s:.1f} s, final loss {tr.losses[-1]:.3e}")
    if save:
        tr.save(save)
    info.update({"n_train_converged": int(len(keep)), "data_gen_s": gen_s,
                 "data_steps_median": data_steps_median,
                 "data_device_s": data_device_s, "train_s": tr.train_s,
                 "final_loss": tr.losses[-1], "losses": tr.losses})
    return tr, info


def evaluate(tr: Trained, n_eval=256, grid=(100, 40), max_steps=200_000, tol=1e-8,
             plain_sample=32, warm_fraction=1.0, tight_tol: float = 1e-10,
             tight_sample: int = 16, log=print) -> dict:
    """Step 3 of the module docstring on the held-out draws 1e6 .. 1e6 +
    n_eval - 1: cold and warm batches (the warm one judged and backed by the
    plain march, solve_warm, with warm_fraction of the cold step estimate as
    its budget), the plain FP64 march one solve after another on
    `plain_sample` of them, and `tight_sample` solves converged both ways
    driven on to tight_tol."""
    L, M = grid
    H, W = L, M + 1
    eval_p = draws(range(1_000_000, 1_000_000 + n_eval), grid)
    floor = tr.floor if tr.floor is not None else np.zeros(2)
    ics, infer_s = predicted_ics(tr, eval_p, grid, floor)
    cold = solve_all(eval_p, max_steps=max_steps, tol=tol)
    budget = max(1000, int(warm_fraction * estimated_steps(eval_p[0].config(), max_steps)))
    warm, fell = solve_warm(eval_p, ics, max_steps=max_steps, tol=tol, budget=budget)
    both = cold.converged & warm.converged
    log(f"eval on {L}x{M}: cold converged {int(cold.converged.sum())}, warm converged "
        f"{int(warm.converged.sum())} of {n_eval} ({int(fell.sum())} fell back); steps cold "
        f"median {np.median(cold.steps):.0f}, warm median {np.median(warm.steps):.0f}")
    err = [relative_linf(fields_of(ics[i], L, M), cold.fields[i])
           for i in np.flatnonzero(cold.converged) if ics[i] is not None]
    err = np.stack(err) if err else np.full((1, S.N_OUT), np.nan)
    agree = [relative_linf(warm.fields[i], cold.fields[i]) for i in np.flatnonzero(both)]
    agree = np.stack(agree) if agree else None

    tight_idx = np.flatnonzero(both)[:tight_sample]
    tight = None
    if len(tight_idx) and tight_tol and tight_tol < tol:
        dist, extra = tight_agreement(eval_p, cold, warm, tight_idx, tight_tol, 4 * max_steps)
        tight = {"tol": tight_tol, "sample": int(len(tight_idx)),
                 "warm_vs_cold_rel_linf_max": dist.tolist(),
                 "extra_steps_median": float(np.median(extra))}
        log(f"driven on to residual {tight_tol:g}: warm vs cold max relative L-inf "
            f"{np.nanmax(dist):.2e} over {len(tight_idx)} solves")

    # the plain FP64 time march, one solve after another (graph engine)
    seq_ms, seq_steps, seq_conv = 0.0, 0, 0
    for p in eval_p[:plain_sample]:
        cfg = p.config()
        s = build_case(cfg, precision="fast")
        r = s.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=max_steps, residual_tol=tol,
                  residual_every=50, engine="graph")
        seq_ms += r.device_ms
        seq_steps += r.steps
        seq_conv += int(r.converged)
        s.close()
    plain_sps = plain_sample / (seq_ms * 1e-3) if plain_sample else float("nan")
    cold_sps = n_eval / (cold.device_ms * 1e-3)
    warm_sps = n_eval / (warm.device_ms * 1e-3 + infer_s)
    return {
        "n_eval": n_eval, "eval_max_steps": max_steps, "tol": tol,
        "cold_converged": int(cold.converged.sum()), "warm_converged": int(warm.converged.sum()),
        "warm_fallback_to_cold_ic": int(fell.sum()), "warm_budget_steps": budget,
        "cold_steps_mean": float(cold.steps.mean()), "warm_steps_mean": float(warm.steps.mean()),
        "cold_steps_median": float(np.median(cold.steps)),
        "warm_steps_median": float(np.median(warm.steps)),
        "cold_batch_solves_per_s": cold_sps, "warm_batch_solves_per_s": warm_sps,
        "plain_sequential_solves_per_s": plain_sps,
        "plain_sequential_sample": plain_sample, "plain_sequential_converged": seq_conv,
        "plain_sequential_steps_mean": seq_steps / max(plain_sample, 1),
        "warm_over_plain": warm_sps / plain_sps, "warm_over_cold_batch": warm_sps / cold_sps,
        "surrogate_inference_s": infer_s,
        "surrogate_rel_linf_median": np.median(err, 0).tolist(),
        "surrogate_rel_linf_max": err.max(0).tolist(),
        "warm_vs_cold_state_rel_linf_max": agree.max(0).tolist() if agree is not None else None,
        "both_converged": int(both.sum()),
        "cold_steps_both": float(cold.steps[both].mean()) if both.any() else None,
        "warm_steps_both": float(warm.steps[both].mean()) if both.any() else None,
        "warm_p50_ms": float(np.percentile(warm.solve_ms, 50)),
        "warm_p99_ms": float(np.percentile(warm.solve_ms, 99)),
        "cold_p50_ms": float(np.percentile(cold.solve_ms, 50)),
        "cold_p99_ms": float(np.percentile(cold.solve_ms, 99)),
        "tight": tight,
    }


def run_pipeline(n_train=2000, n_eval=256, grid=(100, 40), epochs=40, batch=16, lr=1e-3,
                 max_steps=200_000, tol=1e-8, plain_sample=32, log=print,
                 save: str | None = None, tight_tol: float = 1e-10, tight_sample: int = 16,
                 bootstrap=None, n_boot=2000, boot_epochs=60, warm_fraction=1.0) -> dict:
    """build_surrogate then evaluate on the same grid; returns the measurements."""
    tr, info = build_surrogate(n_train, grid, epochs, batch, lr, max_steps, tol, bootstrap,
                               n_boot, boot_epochs, log=log, save=save)
    res = evaluate(tr, n_eval, grid, max_steps, tol, plain_sample, warm_fraction, tight_tol,
                   tight_sample, log)
    return {**info, **res}


def nearest_surrogate(trs: list, L: int) -> int:
    """Index of the surrogate whose grid has the row count nearest to L (on a
    log scale; a tie goes to the finer grid)."""
    best, key = 0, None
    for k, t in enumerate(trs):
        d = (abs(np.log2(t.net.H / L)), -t.net.H)
        if key is None or d < key:
            best, key = k, d
    return best


def predicted_ics_nearest(trs: list, params: list[SweepParams]) -> tuple[list, float, list]:
    """predicted_ics over several surrogates: each draw predicted by the one
    trained nearest its grid (nearest_surrogate) and interpolated onto the
    draw's grid.  Returns the planes, the inference seconds and the index of
    the surrogate each draw used."""
    pick = [nearest_surrogate(trs, p.L) for p in params]
    ics: list = [None] * len(params)
    infer_s = 0.0
    for k, t in enumerate(trs):
        idx = [i for i, q in enumerate(pick) if q == k]
        if not idx:
            continue
        floor = t.floor if t.floor is not None else np.zeros(2)
        got, s = predicted_ics(t, [params[i] for i in idx], None, floor)
        infer_s += s
        for i, g in zip(idx, got):
            ics[i] = g
    return ics, infer_s, pick


def stratified_sample(params: list[SweepParams], k: int) -> list[int]:
    """Indices of k draws with the grid mix of the whole list: per grid, its
    share of k (largest remainders rounded up), taken as that grid's first
    draws in list order."""
    groups: dict[tuple[int, int], list[int]] = {}
    for i, p in enumerate(params):
        groups.setdefault((p.L, p.M), []).append(i)
    n = len(params)
    k = min(k, n)
    want = {g: k * len(v) / n for g, v in groups.items()}
    take = {g: int(math.floor(w)) for g, w in want.items()}
    left = k - sum(take.values())
    for g in sorted(want, key=lambda g: (take[g] - want[g], g))[:left]:
        take[g] += 1
    return sorted(i for g, v in groups.items() for i in v[:take[g]])


def sweep_comparison(tr, n: int = 256, max_steps: int = 200_000, tol: float = 1e-8,
                     plain_sample: int = 32, log=print, cold_batch: bool = True) -> dict:
    """The sweep of uneven grids (workloads.sweep_params(i), i < n) solved
    three ways, all capped at max_steps: the batched engine from the
    workload's initial condition (cold; skipped with cold_batch=False), the
    batched engine from a surrogate's prediction interpolated onto each
    draw's grid (warm, judged and backed by the plain march: solve_warm with
    the full cap as budget; tr is one Trained or a list, of which each draw
    takes the one trained nearest its grid), and the plain FP64 march one
    solve after another on plain_sample draws with the sweep's grid mix
    (stratified_sample).  Rates count all solves and converged solves."""
    trs = list(tr) if isinstance(tr, (list, tuple)) else [tr]
    params = [sweep_params(i) for i in range(n)]
    ics, infer_s, pick = predicted_ics_nearest(trs, params)
    cold = solve_all(params, max_steps=max_steps, tol=tol) if cold_batch else None
    warm, fell = solve_warm(params, ics, max_steps=max_steps, tol=tol, budget=max_steps)
    if cold is not None:
        log(f"sweep of {n}: cold converged {int(cold.converged.sum())} in "
            f"{cold.device_ms / 1e3:.1f} s")
    log(f"sweep of {n}: warm converged {int(warm.converged.sum())} in "
        f"{warm.device_ms / 1e3:.1f} s ({int(fell.sum())} fell back)")
    seq_ms, seq_conv = 0.0, 0
    plain_end = {"converged": 0, "nonfinite": 0, "capped": 0, "other": 0}
    plain_by_grid: dict[str, dict] = {}
    for i in stratified_sample(params, plain_sample):
        p = params[i]
        cfg = p.config()
        sv = build_case(cfg, precision="fast")
        r = sv.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=max_steps, residual_tol=tol,
                   residual_every=50, engine="graph")
        seq_ms += r.device_ms
        seq_conv += int(r.converged)
        end = ("converged" if r.converged else
               "nonfinite" if r.status == N.MPD_ERR_NONFINITE else
               "capped" if r.steps >= max_steps else "other")
        plain_end[end] += 1
        d = plain_by_grid.setdefault(f"{p.L}x{p.M}", {"n": 0, "converged": 0, "nonfinite": 0,
                                                      "seconds": 0.0})
        d["n"] += 1
        d["converged"] += int(r.converged)
        d["nonfinite"] += int(end == "nonfinite")
        d["seconds"] += r.device_ms * 1e-3
        sv.close()
    agree = []
    if cold is not None:
        both = cold.converged & warm.converged
        agree = [relative_linf(warm.fields[i], cold.fields[i]) for i in np.flatnonzero(both)]
    by_grid = {}
    for i, p in enumerate(params):
        d = by_grid.setdefault(f"{p.L}x{p.M}", {
            "n": 0, "cold_converged": 0, "warm_converged": 0, "cold_steps": [],
            "warm_steps": [],
            "surrogate_grid": f"{trs[pick[i]].net.H}x{trs[pick[i]].net.W - 1}"})
        d["n"] += 1
        d["warm_converged"] += int(warm.converged[i])
        d["warm_steps"].append(int(warm.steps[i]))
        if cold is not None:
            d["cold_converged"] += int(cold.converged[i])
            d["cold_steps"].append(int(cold.steps[i]))
    for d in by_grid.values():
        cs = d.pop("cold_steps")
        d["cold_steps_median"] = float(np.median(cs)) if cs else None
        d["warm_steps_median"] = float(np.median(d.pop("warm_steps")))
        if cold is None:
            d["cold_converged"] = None
    warm_s = warm.device_ms * 1e-3 + infer_s
    seq_s = seq_ms * 1e-3
    out = {
        "n": n, "max_steps": max_steps, "tol": tol, "plain_sample": plain_sample,
        "surrogate_grids": [f"{t.net.H}x{t.net.W - 1}" for t in trs],
        "warm_batch_s": warm_s, "plain_sample_s": seq_s,
        "warm_converged": int(warm.converged.sum()),
        "plain_sample_converged": seq_conv, "plain_sample_ends": plain_end,
        "plain_sample_by_grid": plain_by_grid,
        "warm_fallbacks": int(fell.sum()),
        "warm_batch_solves_per_s": n / warm_s,
        "plain_solves_per_s": plain_sample / seq_s if seq_s > 0 else None,
        "warm_batch_converged_per_s": int(warm.converged.sum()) / warm_s,
        "plain_converged_per_s": seq_conv / seq_s if seq_s > 0 else None,
        "warm_over_plain": (n / warm_s) / (plain_sample / seq_s) if seq_s > 0 else None,
        "warm_over_plain_converged": ((int(warm.converged.sum()) / warm_s) /
                                      (seq_conv / seq_s) if seq_s > 0 and seq_conv else None),
        "warm_vs_cold_state_rel_linf_max": np.stack(agree).max(0).tolist() if agree else None,
        "warm_p50_ms": float(np.percentile(warm.solve_ms, 50)),
        "warm_p99_ms": float(np.percentile(warm.solve_ms, 99)),
        "surrogate_inference_s": infer_s,
        "by_grid": by_grid,
    }
    if cold is not None:
        cold_s = cold.device_ms * 1e-3
        out.update({
            "cold_batch_s": cold_s, "cold_converged": int(cold.converged.sum()),
            "cold_batch_solves_per_s": n / cold_s,
            "cold_batch_converged_per_s": int(cold.converged.sum()) / cold_s,
            "cold_p50_ms": float(np.percentile(cold.solve_ms, 50)),
            "cold_p99_ms": float(np.percentile(cold.solve_ms, 99))})
    return out
