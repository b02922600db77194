#!/usr/bin/env python
"""Benchmark of the plain FP64 Lax-Friedrichs hot path on B200.

Workload (one "step" = one time step of Solver::Advance + the adaptive dt
update): the coaxial channel r1 = 0.2, r2 = 0.8 on the 1600 x 640 grid, IC
rho = 1, v_z = 0.1, p = beta/2, B_phi = r1/r, inlet fixed, zero-gradient
outlet, slip walls, CFL 0.4, FP64 (fast precision: reciprocal multiplies +
FMA, <= 1e-12 of the reference after 1000 steps).  Inputs are synthetic and
built on the host from the configuration.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: a single grid does not shard (one domain per GPU); N ranks run
N independent replicas and ``value`` adds their cell updates ("replicas only").
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

L_MAX, M_MAX = 1600, 640
CELLS = L_MAX * (M_MAX + 1)          # interior cell updates per step
ALG_BYTES_PER_CELL = 128             # 8 FP64 conserved values read + 8 written


def interior_cells(ring_beside: bool) -> int:
    """Cells one launch of the interior kernel updates: columns 2..M of rows
    2..L-1 when the boundary ring runs beside it (rows 1 and L are the ring
    kernel's), of rows 1..L otherwise."""
    return (L_MAX - 2 if ring_beside else L_MAX) * (M_MAX - 1)
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--cpu-child", type=str, default="", help=argparse.SUPPRESS)
    ap.add_argument("--profile", action="store_true",
                    help="lean run for ncu: warm-up, then --steps eager time steps, no extras")
    ap.add_argument("--diagnostics", action="store_true",
                    help="with --profile: then each reduction once (residual, integrals, "
                         "solution change, outlet, radial symmetry, wave speed)")
    ap.add_argument("--pair", action="store_true",
                    help="with --profile: then three launches of the two-column interior "
                         "kernel (lf_pair_kernel) on the final state")
    ap.add_argument("--precision", choices=("fast", "exact"), default="fast")
    ap.add_argument("--workload", choices=("plain", "warmstart", "batch", "surrogate", "serve",
                                           "converge", "sweep"),
                    default="plain",
                    help="plain: the 1600x640 time step (default); warmstart: surrogate-warm-"
                         "started batched steady solves vs the plain time march; batch: the "
                         "batched sweep of uneven grids; surrogate: training iterations of "
                         "the warm-start network; serve: a large warm-started grid beside a "
                         "memory-budgeted batch of small solves; converge: the 1600x640 "
                         "channel time-marched to an L-inf residual of 1e-8 (--max-steps); "
                         "sweep: the uneven sweep cold, surrogate-warm (--surrogate) and by the "
                         "plain march one solve after another")
    ap.add_argument("--n-train", type=int, default=2000)
    ap.add_argument("--n-eval", type=int, default=256)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--grid", type=str, default="100x40")
    ap.add_argument("--n-solves", type=int, default=64)
    ap.add_argument("--max-steps", type=int, default=200000)
    ap.add_argument("--surrogate", type=str, default="",
                    help="trained surrogate (.npz from --workload warmstart --save); "
                         "without it serve trains a small one first; sweep takes a "
                         "comma-separated list and predicts each draw with the one trained "
                         "nearest its grid")
    ap.add_argument("--skip-cold", action="store_true",
                    help="sweep: leave out the cold batch (warm batch and plain march only)")
    ap.add_argument("--save", type=str, default="", help="warmstart: save the surrogate here")
    ap.add_argument("--big", type=str, default="4096x1600")
    ap.add_argument("--bootstrap", type=str, default="",
                    help="warmstart: generate the training data warm from a surrogate first "
                         "trained on this coarser grid (e.g. 100x40)")
    ap.add_argument("--n-boot", type=int, default=2000)
    ap.add_argument("--a-max", type=float, default=0.2,
                    help="surrogate draws: wall amplitude range [0, a_max]")
    ap.add_argument("--skip-mix", action="store_true",
                    help="serve: only the --error-grid measurements, not the serving mix")
    ap.add_argument("--error-a", type=str, default="0.3,0.2",
                    help="serve: wall amplitudes of the --error-grid channels")
    ap.add_argument("--error-grid", type=str, default="",
                    help="serve: also measure the warm start's distance to the cold steady "
                         "state on this grid (e.g. 800x320) at a = 0.3")
    ap.add_argument("--plain-sample", type=int, default=32,
                    help="warmstart: solves of the plain march timed one after another")
    ap.add_argument("--warm-fraction", type=float, default=1.0,
                    help="warmstart: a warm solve's step budget as a fraction of the cold "
                         "estimate before it falls back to the cold start")
    ap.add_argument("--tight-tol", type=float, default=1e-10)
    ap.add_argument("--stage", choices=("all", "build", "eval"), default="all",
                    help="warmstart: build = data + training (--save), eval = the held-out "
                         "comparison with a saved surrogate (--surrogate), all = both")
    return ap.parse_args()


def workload_config():
    return {"workload": "plain FP64 LF time step, straight coaxial channel 1600x640",
            "L_max": L_MAX, "M_max": M_MAX, "cells_per_step": CELLS, "cfl": 0.4,
            "adaptive_dt": True, "geometry": "r1=0.2, r2=0.8",
            "l2": "per-step working set 138 MB (8 planes read + 8 written) > 126 MB L2, no flush",
            "parallelism": "replicas"}


PRECISION_OURS = "fast (reciprocal + FMA FP64; <= 1e-12 relative L-inf of the reference)"
PRECISION_REF = "exact (the reference's own CPU build, IEEE FP64, no FMA contraction)"


# ---------------------------------------------------------------- CPU side
def _case():
    from tests import cases
    return cases.channel_case(L=L_MAX, M=M_MAX)


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_child(spec: str) -> None:
    """Runs in a subprocess so OMP_NUM_THREADS applies: time the reference
    CPU build (or the oracle port) on the workload and print JSON.  The
    inputs come from oracle/channel.py (the reference's own geometry plugin
    and ExpressionIC), so this process never loads the product library."""
    kind, steps, warmup = spec.split(":")
    steps, warmup = int(steps), int(warmup)
    from oracle import bind, channel
    case = channel.channel_case(L_MAX, M_MAX)
    be = bind.Ref(case) if kind == "reference" else bind.Port(case)
    d = channel.DRIVER
    dt = d["dt0"]

    def step(dt):
        be.advance(dt)
        return be.compute_dt(d["cfl"], d["growth"], d["dt_min"], d["dt_max"], dt)

    for _ in range(warmup):
        dt = step(dt)
    t0 = time.perf_counter()
    per = []
    for _ in range(steps):
        s0 = time.perf_counter()
        dt = step(dt)
        per.append(time.perf_counter() - s0)
    el = time.perf_counter() - t0
    print(json.dumps({"seconds": el, "steps": steps, "per_step": per}))


def run_cpu(kind: str, steps: int, warmup: int, threads: int) -> dict:
    env = dict(os.environ)
    env.update(OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close", OMP_PLACES="cores")
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--cpu-child",
                          f"{kind}:{steps}:{warmup}"], capture_output=True, text=True, env=env,
                         timeout=1800)
    if out.returncode != 0:
        raise RuntimeError(out.stderr[-2000:])
    return json.loads(out.stdout.strip().splitlines()[-1])


def cpu_kind():
    from oracle import bind
    return "reference" if bind.ref_available() else "port"


def cpu_baseline_leg() -> dict:
    kind = cpu_kind()
    threads = os.cpu_count() or 1
    probe = run_cpu(kind, 2, 1, threads)
    per = probe["seconds"] / probe["steps"]
    steps = max(3, min(200, int(20.0 / max(per, 1e-6))))   # ~20 s of CPU work
    res = run_cpu(kind, steps, 1, threads)
    value = CELLS * res["steps"] / res["seconds"]
    return {"value": value, "unit": "cell-updates/s", "cores": threads, "kind": kind,
            "cpu_model": cpu_model(), "precision": PRECISION_REF,
            "sample": f"{res['steps']} time steps of the 1600x640 channel "
                      f"(OMP_NUM_THREADS={threads}, OMP_PROC_BIND=close)"}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_uuid: str | None):
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")
        self.uuid = device_uuid

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
               "-lms", "100"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(cmd, stdout=self.fh, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        with open(self.path) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(kernel: str = "lf_tma_kernel"):
    """DRAM bytes per launch of `kernel` from one ncu capture (profiles/traffic.json)."""
    p = ROOT / "profiles" / "traffic.json"
    try:
        d = json.loads(p.read_text())[kernel]
        return float(d["dram_bytes_per_launch"]), d.get("note", "")
    except (OSError, KeyError, ValueError, TypeError):
        return None, "no ncu capture recorded"


# ---------------------------------------------------------------- GPU side
RESID_BYTES_PER_CELL = 128  # 8 new + 8 old conserved values read per interior cell
# the interior kernel of fast steps (one point column per lane, as in the
# persistent engines); the two-column form is timed beside it
INTERIOR_KERNEL = "lf_tma_kernel"


def graph_chunk(steps: int) -> int:
    """Steps per captured CUDA graph for a timed run of `steps` steps: the
    largest divisor of `steps` up to 100, so the run launches whole graphs
    only (no launch runs past the last step); 100 when `steps` has no divisor
    of at least 10 up to 100 (the last launch then ends in early exits)."""
    if steps <= 100:
        return max(steps, 1)
    for d in range(100, 9, -1):
        if steps % d == 0:
            return d
    return 100


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", device_id=torch.device("cuda", local_rank),
                                timeout=datetime.timedelta(seconds=300))

    def max_over_ranks(x: float) -> float:
        if not dist:
            return x
        tt = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt.item())

    case = _case()
    cfg = case.cfg
    solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision="fast")
    per_graph = graph_chunk(args.steps)

    # warm-up: the exact first step, then W - 1 steps through the very graph
    # (same steps per launch, same flags) that the timed run replays, so the
    # capture and instantiation happen here and not inside the timed region
    w = max(args.warmup, 1)
    wres = solver.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=w, steps_per_graph=per_graph)
    assert wres.steps == w, wres

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local_rank).uuid)
    except Exception:
        pass
    sampler = ClockSampler(uuid)
    sampler.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    # K steps as K / per_graph launches of the captured graph, back to back;
    # device_ms is CUDA events on the solver's stream around exactly them
    res = solver.run(T=1e300, dt=wres.dt, adaptive=True, max_steps=args.steps,
                     steps_per_graph=per_graph)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    assert res.steps == args.steps, res
    t_max = max_over_ranks(res.device_ms)

    # per-launch device time of the dominant kernel and of the residual pass:
    # back-to-back launches between two events on the solver's stream
    hbm, hbm_src = measured_hbm()
    # median of five samples of 30 launches each: one sample varies by up
    # to 8 % between runs on the same GPU
    def kernel_ms(which):
        return statistics.median(solver.profile_kernel(which, 30, res.dt) for _ in range(5))

    int_ms = kernel_ms("interior")
    int2_ms = kernel_ms("interior_pair")
    resid_ms = kernel_ms("residual")
    ring_beside = solver.ring_overlap
    int_bytes = ALG_BYTES_PER_CELL * interior_cells(ring_beside)
    achieved = int_bytes / (int_ms * 1e-3) / 1e9
    resid_gbs = RESID_BYTES_PER_CELL * CELLS / (resid_ms * 1e-3) / 1e9
    traffic, traffic_note = profiled_traffic(INTERIOR_KERNEL)

    # end to end through the public API with host buffers: the initial
    # physical planes uploaded from pinned memory, the reference driver's
    # per-step pattern (Advance(dt), then ComputeDt back on the host: 8 bytes
    # each way per step), and the final physical planes read back into pinned
    # memory (IOManager's output, mpd_snapshot_async); every phase timed
    shape = (10,) + solver.shape
    h_in = torch.from_numpy(np.ascontiguousarray(case.phys)).pin_memory()
    h_out = torch.empty(shape, dtype=torch.float64).pin_memory()
    n_e2e = args.steps
    # one untimed pass of the same calls (the first upload creates the
    # solver's dense staging planes)
    solver.set_physical(h_in.numpy())
    solver.Advance(cfg.dt)
    solver.ComputeDt(cfg.dt)
    solver.snapshot_async(h_out)
    solver.snapshot_wait()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    solver.set_physical(h_in.numpy())
    t1 = time.perf_counter()
    dt = cfg.dt
    for _ in range(n_e2e):
        solver.Advance(dt)
        dt = solver.ComputeDt(dt)
    t2 = time.perf_counter()
    solver.snapshot_async(h_out)
    solver.snapshot_wait()
    t3 = time.perf_counter()
    e2e_s = max_over_ranks(t3 - t0)
    phases = {"upload_ms": 1e3 * (t1 - t0), "steps_ms": 1e3 * (t2 - t1),
              "download_ms": 1e3 * (t3 - t2)}
    # IOManager's snapshot beside stepping: 200 graph steps alone, the same
    # with a snapshot of the 10 physical planes issued first (its device ->
    # pinned host copy runs on the solver's side stream), and the snapshot
    # alone
    solver.run(T=1e300, dt=dt, adaptive=True, max_steps=200, steps_per_graph=100)
    alone = solver.run(T=1e300, dt=dt, adaptive=True, max_steps=200, steps_per_graph=100)
    t0s = time.perf_counter()
    solver.snapshot_async(h_out)
    both = solver.run(T=1e300, dt=alone.dt, adaptive=True, max_steps=200, steps_per_graph=100)
    solver.snapshot_wait()
    both_wall = time.perf_counter() - t0s
    t0s = time.perf_counter()
    solver.snapshot_async(h_out)
    solver.snapshot_wait()
    snap_alone = time.perf_counter() - t0s
    snapshot = {"steps": 200, "steps_ms": alone.device_ms, "steps_with_snapshot_ms": both.device_ms,
                "snapshot_alone_ms": 1e3 * snap_alone, "both_wall_ms": 1e3 * both_wall,
                "bytes": int(h_out.numel() * 8)}
    plane = solver.shape[0] * solver.shape[1] * 8
    h2d = (10 * plane + 8 * n_e2e) / n_e2e          # IC planes + dt per step
    d2h = (10 * plane + 8 * n_e2e) / n_e2e          # output planes + dt per step
    solver.close()

    line = None
    if rank == 0:
        cpu = None
        if world == 1:
            try:
                cpu = cpu_baseline_leg()
            except Exception as exc:  # noqa: BLE001 - report, do not fail the bench
                cpu = {"value": None, "unit": "cell-updates/s", "cores": os.cpu_count(),
                       "kind": cpu_kind(), "sample": f"failed: {exc}"[:300]}
        value = world * CELLS * args.steps / (t_max * 1e-3)
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "precision": PRECISION_OURS,
            "config": workload_config(),
            "timing": f"CUDA events on the solver stream around {args.steps // per_graph} "
                      f"back-to-back launches of one captured graph of {per_graph} steps "
                      f"(2 kernels per step), built during warm-up; max over ranks",
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic,
                         "traffic_note": traffic_note,
                         "kernel": INTERIOR_KERNEL, "kernel_ms": int_ms,
                         "pair_kernel_ms": int2_ms,
                         "alg_bytes_per_launch": int_bytes,
                         "ring_beside_interior": ring_beside,
                         "kernel_timing": "median of 5 samples of 30 back-to-back launches between two CUDA events",
                         "peak_source": hbm_src},
            "residual_kernel": {"kernel": "residual_kernel", "ms": resid_ms,
                                "achieved": resid_gbs, "unit": "GB/s", "peak": hbm,
                                "frac": resid_gbs / hbm,
                                "traffic": profiled_traffic("residual_kernel")[0],
                                "alg_bytes_per_launch": RESID_BYTES_PER_CELL * CELLS,
                                "how": "median of 5 samples of 30 back-to-back launches between two CUDA events"},
            "cpu_baseline": cpu,
            "e2e": {"value": world * CELLS * n_e2e / e2e_s, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": n_e2e, "phases_ms_rank0": phases,
                    "how": "set_physical from pinned host planes, K x (Advance, ComputeDt), "
                           "snapshot of the 10 physical planes into pinned host memory; "
                           "host wall clock, max over ranks; upload and download amortised "
                           "over the K steps"},
            "snapshot_overlap": snapshot,
            "gpu_launches": 2 * args.steps,
            "clocks": clocks,
        }
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return line


def run_warmstart(args):
    """Learned warm start (the sweep box on one grid): steady states from the
    batched solver train the surrogate (on a fine grid, optionally
    bootstrapped from a coarse surrogate's interpolated predictions);
    held-out draws are then solved cold and warm by the batched solver (warm
    solves judged and backed by the plain march), and a sample of them one
    after another by the plain FP64 time march (graph engine).  value =
    warm-start batch solves/s (surrogate inference included)."""
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    WS = pkg.warmstart
    L, M = (int(v) for v in args.grid.split("x"))
    boot = tuple(int(v) for v in args.bootstrap.split("x")) if args.bootstrap else None
    log = lambda m: print(m, file=sys.stderr, flush=True)  # noqa: E731
    info = {}
    if args.stage == "eval":
        tr = WS.Trained.load(args.surrogate)
    else:
        tr, info = WS.build_surrogate(args.n_train, (L, M), args.epochs, max_steps=args.max_steps,
                                      bootstrap=boot, n_boot=args.n_boot, log=log,
                                      save=args.save or None)
        info.pop("losses", None)
        if args.stage == "build":
            return {"metric": "learned warm start: surrogate built", "value": info["train_s"],
                    "unit": "s", "higher_is_better": False, "n_gpus": 1,
                    "data": "synthetic (sweep-box draws, numpy default_rng(seed))",
                    "config": {"workload": f"learned warm start, training on {L}x{M}",
                               "bootstrap": args.bootstrap or None}, **info}
    res = WS.evaluate(tr, args.n_eval, (L, M), args.max_steps, plain_sample=args.plain_sample,
                      warm_fraction=args.warm_fraction, tight_tol=args.tight_tol, log=log)
    return {
        "metric": "steady solves/s, warm-start batch (residual <= 1e-8)",
        "value": res["warm_batch_solves_per_s"], "unit": "solves/s", "n_gpus": 1,
        "higher_is_better": True, "dtype": "f64 solver, bf16/f32 surrogate",
        "data": "synthetic (sweep-box draws, numpy default_rng(seed))",
        "config": {"workload": f"learned warm start, channel sweep box on {L}x{M}",
                   "n_train": args.n_train, "n_eval": args.n_eval, "epochs": args.epochs,
                   "bootstrap": args.bootstrap or None,
                   "surrogate": "4 spectral layers, 64 channels, 8 modes per axis"},
        "vs_baseline": None, **info, **res}


def run_converge(args):
    """The 1600x640 channel time-marched from its initial condition until the
    L-inf residual is <= 1e-8 (evaluated every 50 steps) or --max-steps; the
    reference's CPU time for the same number of steps is extrapolated from a
    bounded sample of its per-step time, and labelled as such."""
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    case = _case()
    cfg = case.cfg
    solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision=args.precision)
    res = solver.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=args.max_steps,
                     residual_tol=1e-8, residual_every=50)
    solver.close()
    secs = res.device_ms * 1e-3
    cpu = cpu_baseline_leg()
    cpu_secs = CELLS * res.steps / cpu["value"] if cpu.get("value") else None
    return {
        "metric": "time to L-inf residual 1e-8, 1600x640 channel", "value": secs, "unit": "s",
        "higher_is_better": False, "n_gpus": 1, "dtype": "f64", "vs_baseline": None,
        "data": "synthetic", "config": workload_config(),
        "steps": res.steps, "converged": bool(res.converged), "residual": res.residual,
        "status": res.status, "t": res.t,
        "cell_updates_per_s": CELLS * res.steps / secs,
        "cpu_baseline": cpu,
        "cpu_seconds_extrapolated": cpu_secs,
        "cpu_extrapolation": "reference CPU per-step time on a bounded sample x the GPU's steps",
    }


def run_serve(args):
    """The serving mix, bounded: a large converging-diverging
    channel warm-started from the surrogate (coarse prediction remapped on
    the device) in one persistent launch beside small sweep solves admitted by
    a device-memory budget; the same mix cold for comparison.  With
    --error-grid, the per-field distance to the cold steady state on a large
    grid where that state is reachable.  Without --surrogate a surrogate is
    first built on --grid from draws whose wall amplitude reaches --a-max
    (the large channel's a = 0.3 lies outside the sweep box)."""
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    WS = pkg.warmstart
    log = lambda m: print(m, file=sys.stderr, flush=True)  # noqa: E731
    info = {}
    if args.surrogate:
        tr = WS.Trained.load(args.surrogate)
    else:
        L, M = (int(v) for v in args.grid.split("x"))
        tr, info = WS.build_surrogate(args.n_train, (L, M), args.epochs,
                                      max_steps=args.max_steps, log=log,
                                      save=args.save or None, a_max=args.a_max)
        info.pop("losses", None)
    bL, bM = (int(v) for v in args.big.split("x"))
    res = {} if args.skip_mix else pkg.serve.run_serving(
        tr, big=(bL, bM), n_small=args.n_solves, max_steps=min(args.max_steps, args.steps),
        log=log)
    err = None
    if args.error_grid:
        eL, eM = (int(v) for v in args.error_grid.split("x"))
        err = [pkg.serve.large_grid_error(tr, (eL, eM), a_big=float(a),
                                          cap=min(args.max_steps, args.steps), log=log)
               for a in args.error_a.split(",")]
    return {"metric": "serving mix: small solves/s beside a warm-started large grid",
            "value": res["warm"]["small_solves_per_s"] if res else None, "unit": "solves/s",
            "higher_is_better": True, "n_gpus": 1, "dtype": "f64", "vs_baseline": None,
            "data": "synthetic (sweep-box draws)",
            "config": {"workload": f"large channel {args.big} a=0.3 + {args.n_solves} small",
                       "steps_cap": min(args.max_steps, args.steps),
                       "surrogate_a_max": info.get("a_max")},
            "surrogate": info, **res, "large_grid_error": err}


def run_sweep(args):
    """The warm-start comparison on the parameter sweep of uneven grids:
    batched cold (unless --skip-cold), batched surrogate-warm (--surrogate:
    each draw predicted by the surrogate trained nearest its grid,
    interpolated onto the draw's grid) and the plain FP64 march one solve
    after another (--plain-sample of the draws), all capped at --max-steps.
    value = warm batch solves/s."""
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    WS = pkg.warmstart
    log = lambda m: print(m, file=sys.stderr, flush=True)  # noqa: E731
    trs = [WS.Trained.load(p) for p in args.surrogate.split(",") if p]
    res = WS.sweep_comparison(trs, args.n_solves, args.max_steps, plain_sample=args.plain_sample,
                              log=log, cold_batch=not args.skip_cold)
    return {"metric": "steady solves/s, warm-start batch on the uneven sweep",
            "value": res["warm_batch_solves_per_s"], "unit": "solves/s",
            "higher_is_better": True, "n_gpus": 1, "dtype": "f64 solver, bf16/f32 surrogate",
            "data": "synthetic (sweep-box draws, numpy default_rng(i))", "vs_baseline": None,
            "config": {"workload": "sweep grids {100x40,200x80,400x160,800x320}",
                       "n_solves": args.n_solves, "max_steps": args.max_steps,
                       "surrogate": args.surrogate}, **res}


def run_surrogate(args):
    """Training iterations of the warm-start network (forward, MSE, backward,
    Adam) on random inputs: grid --grid, batch 16; --warmup untimed, --steps
    timed with CUDA events, eagerly and as the captured CUDA graph the
    training loop replays."""
    import numpy as np
    import torch
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    S = pkg.surrogate
    L, M = (int(v) for v in args.grid.split("x"))
    H, W, B = L, M + 1, 16
    net = S.SpectralOperator(H, W, B, seed=0)
    rng = np.random.default_rng(0)
    net.load_inputs(rng.standard_normal((B, H * W, S.N_IN)))
    net.target.copy_(torch.from_numpy(rng.standard_normal((B * H * W, S.N_OUT))
                                      .astype(np.float32)))

    def timed(n):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n):
            net.train_step()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / max(n, 1)

    for _ in range(args.warmup):
        net.train_step()
    net.wait()
    eager_ms = timed(args.steps)
    net.capture()
    for _ in range(args.warmup):
        net.train_step()
    ms = timed(args.steps)
    net.wait()
    P, Q, Cw = H * W, net.Q, S.WIDTH
    # multiply-adds of one forward pass per sample; backward ~ 2x
    fwd = P * S.N_IN * Cw + S.LAYERS * (2 * Q * P * Cw + Q * Cw * Cw + P * Cw * Cw) + \
        P * Cw * S.HIDDEN + P * S.HIDDEN * S.N_OUT
    flops = 2 * 3 * fwd * B
    return {"metric": "surrogate training iteration", "value": ms, "unit": "ms",
            "higher_is_better": False, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "dtype": "bf16 operands, f32 accumulate", "data": "synthetic (random)",
            "config": {"workload": f"spectral operator on {L}x{M}, batch {B}",
                       "parameters": net.nparam},
            "vs_baseline": None, "eager_ms": eager_ms, "gemm_flops_per_iteration": flops,
            "achieved_tflops": flops / (ms * 1e-3) / 1e12}


def run_batch(args, rank=0, world=1, local_rank=0):
    """The batched sweep: n solves per GPU drawn from the sweep box (uneven
    grids), autotuned teams, one persistent cooperative launch per GPU, cold
    start.  With N GPUs (one process each) the N x n draws shard by solve,
    balanced by estimated cost; nothing crosses GPUs while solving, the
    results are gathered on rank 0 and the time is the slowest rank's."""
    import numpy as np
    import torch
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", device_id=torch.device("cuda", local_rank))
    n_total = args.n_solves * world
    params = [pkg.workloads.sweep_params(i) for i in range(n_total)]
    cfgs = [p.config() for p in params]
    info = {}

    def run_share(idx):
        sub = [cfgs[i] for i in idx]
        solvers = [pkg.build_case(c, precision="fast") for c in sub]
        batch = pkg.BatchSolver(solvers)
        tuner = pkg.Autotuner(batch.capacity, steps=100)
        plan = tuner.plan(sub, max_steps=args.max_steps)
        res = batch.run(plan, max_steps=args.max_steps, residual_tol=1e-8, residual_every=50)
        info["plan"], info["table"] = plan, tuner.table
        batch.close()
        for s in solvers:
            s.close()
        return res.runs, res.solve_ms, res.device_ms

    if world > 1:
        costs = [pkg.sharding.solve_cost(c, args.max_steps) for c in cfgs]
        merged = pkg.sharding.run_sharded(costs, run_share)
        dist.barrier()
        dist.destroy_process_group()
        if rank != 0:
            return None
        runs, solve_ms, device_ms = merged.runs, merged.solve_ms, merged.device_ms
    else:
        runs, solve_ms, device_ms = run_share(list(range(n_total)))
    plan = info["plan"]
    converged = int(sum(bool(r.converged) for r in runs))
    cells = sum(c.L_max * (c.M_max + 1) * r.steps for c, r in zip(cfgs, runs))
    return {
        "metric": "batched steady solves: solves/s", "unit": "solves/s", "n_gpus": world,
        "value": n_total / (device_ms * 1e-3), "higher_is_better": True,
        "scaling": "weak", "dtype": "f64", "data": "synthetic (sweep-box draws, numpy default_rng(i))",
        "config": {"workload": "batched sweep, grids {100x40,200x80,400x160,800x320}",
                   "n_solves": n_total, "n_solves_per_gpu": args.n_solves,
                   "max_steps": args.max_steps,
                   "teams_rank0": len(plan.team_blocks), "blocks_rank0": plan.blocks,
                   "sharding": "by solve, cost-balanced" if world > 1 else "none"},
        "vs_baseline": None,
        "cell_updates_per_s": cells / (device_ms * 1e-3),
        "converged": converged,
        "p50_solve_ms": float(np.percentile(solve_ms, 50)),
        "p99_solve_ms": float(np.percentile(solve_ms, 99)),
        "device_ms": device_ms,
        "plan_rank0": {"team_blocks": plan.team_blocks},
        "autotune_us_per_step": {f"{k[0]}x{k[1]}": v for k, v in info["table"].items()},
    }


def run_profile(args):
    """Lean run for profilers: the exact first step, --warmup graph steps, then
    --steps eagerly launched steps (interior + boundary kernel each)."""
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    case = _case()
    cfg = case.cfg
    solver = pkg.GpuSolver(cfg, case.grid, case.phys, precision=args.precision,
                           with_prev=args.diagnostics)
    # one graph of exactly --warmup steps, so no launch in the profile is an
    # early exit of a graph that ran past the step limit
    w = max(args.warmup, 1)
    solver.run(T=1e300, dt=cfg.dt, adaptive=True, max_steps=w, steps_per_graph=w)
    dt = solver.ComputeDt(cfg.dt)
    for _ in range(args.steps):
        solver.Advance(dt)
    t, step = solver.time()
    out = {"profile_steps": args.steps, "step": step, "t": t}
    if args.pair:
        out["pair_ms"] = solver.profile_kernel("interior_pair", 3, dt)
    if args.diagnostics:
        out["residual"] = solver.residual()
        out["integrals"] = [float(x) for x in solver.ComputeIntegrals()]
        out["change"] = solver.SolutionChange()
        out["mass_flux"], out["thrust"] = solver.outlet()
        out["radial"] = solver.CheckRadialSymmetry()
        solver.set_physical(solver.physical())  # a state with no fused wave speed
        out["wave_speed"] = solver.MaxWaveSpeed()
    solver.close()
    print(json.dumps(out))


def run_reference(args, rank, world):
    """The reference's own CPU implementation of the step (oracle/_ref: its
    translation units compiled unchanged; the oracle port if that build is
    absent) on all host threads, same workload, metric and config as our arm.
    Its inputs come from oracle/channel.py, so no process of this arm loads
    the product library.  Under torchrun only rank 0 runs."""
    if rank != 0:
        return None
    threads = os.cpu_count() or 1
    kind = cpu_kind()
    probe = run_cpu(kind, 1, 0, threads)
    per = max(probe["seconds"], 1e-6)
    steps = max(1, min(args.steps, int(150.0 / per)))   # bounded: a few minutes at most
    warm = max(0, min(args.warmup, int(30.0 / per)))
    res = run_cpu(kind, steps, warm, threads)
    value = CELLS * res["steps"] / res["seconds"]
    return {
        "impl": "reference", "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
        "n_gpus": world, "steps": res["steps"], "warmup": warm,
        "ms_per_step": 1e3 * res["seconds"] / res["steps"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "precision": PRECISION_REF,
        "config": workload_config(),
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": threads, "kind": kind,
                         "cpu_model": cpu_model(),
                         "sample": f"{res['steps']} of the requested {args.steps} time steps "
                                   f"(OMP_NUM_THREADS={threads}, OMP_PROC_BIND=close)"},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    args = parse()
    if args.cpu_child:
        cpu_child(args.cpu_child)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.profile:
        run_profile(args)
        return
    if args.workload == "batch":
        line = run_batch(args, rank, world, local_rank)
        if line is not None:
            print(json.dumps(line))
        return
    if args.workload != "plain":
        if rank == 0:
            runner = {"warmstart": run_warmstart, "surrogate": run_surrogate,
                      "serve": run_serve, "converge": run_converge,
                      "sweep": run_sweep}[args.workload]
            line = runner(args)
            print(json.dumps(line))
        return
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    else:
        line = run_ours(args, rank, world, local_rank)
    if line is not None:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
