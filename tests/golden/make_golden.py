"""Generate the golden fixtures in tests/golden/ from the reference's own code.

Run here, where the reference sources exist:  python tests/golden/make_golden.py
It builds oracle/_ref/libmpd_ref.so (oracle/Makefile: the reference's own
solver/fields/face_bc/per_field_bc/diagnostics/... translation units with
single-rank MPI, YAML-node and exprtk-API shims) and records, per case:

* the inputs: wall profiles (the reference's IGeometry plugin where one
  exists, else the sine-wall profile), the initial planes from the
  reference's ExpressionIC, and the boundary segments;
* the outputs of the reference's Solver::Advance driven by its driver loop
  (adaptive dt through Diagnostics::ComputeDt): all 18 planes after a few
  step counts, plus dt, t, integrals, outlet, wave speed, solution change.

The 1000-step config-1 case stores SHA-256 digests of the planes instead of
the planes themselves to keep the fixture small.
"""
from __future__ import annotations

import hashlib
import json
import os
import pathlib
import subprocess
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import bind  # noqa: E402
from tests import cases  # noqa: E402


def plane_digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def ref_inputs(cfg, use_ref_geometry: bool):
    """Profiles and IC from the reference's own plugins."""
    case = cases.make_case(cfg)
    d = case.oracle_dict(with_prev=True)
    if use_ref_geometry:
        rin, rout, drin, drout = bind.ref_geometry_profile(
            cfg.geometry.type, {k: v for k, v in cfg.geometry.params.items()}, cfg.L_max, cfg.dz)
        d.update(rin=rin, rout=rout, drin=drin, drout=drout, r_0=(rin[1] + rout[1]) / 2.0)
    params = [cfg.gamma, cfg.beta, cfg.H_z0, cfg.dz, cfg.dy, d["r_0"]]
    ic = {k: v for k, v in cfg.initial_conditions.params.items()}
    d["phys"] = bind.ref_expression_ic(ic, cfg.L_max, cfg.M_max, params, d["rin"], d["rout"],
                                       d["drin"], d["drout"])
    return d


def record(name, cfg, use_ref_geometry, checkpoints, digest_only=False):
    d = ref_inputs(cfg, use_ref_geometry)
    ref = bind.Ref(d)
    out = {"L": cfg.L_max, "M": cfg.M_max, "rin": d["rin"], "rout": d["rout"],
           "drin": d["drin"], "drout": d["drout"], "r_0": d["r_0"], "phys0": d["phys"]}
    dt = cfg.dt
    step = 0
    meta = {"name": name, "checkpoints": checkpoints, "bc": d["bc"], "gamma": cfg.gamma,
            "beta": cfg.beta, "H_z0": cfg.H_z0, "dt0": cfg.dt, "cfl": cfg.cfl_number,
            "growth": cfg.dt_growth_factor, "dt_min": cfg.dt_min, "dt_max": cfg.dt_max,
            "adaptive": cfg.adaptive_dt, "results": {}}
    t = 0.0
    for cp in checkpoints:
        while step < cp:
            ref.advance(dt)
            t += dt
            step += 1
            dt = ref.compute_dt(cfg.cfl_number, cfg.dt_growth_factor, cfg.dt_min, cfg.dt_max, dt)
        cons = np.stack([ref.get(k) for k in range(8)])
        phys = np.stack([ref.get(8 + k) for k in range(10)])
        res = {"dt_next": dt, "t": t, "integrals": list(ref.integrals()),
               "outlet": list(ref.outlet()), "max_wave_speed": ref.max_wave_speed(),
               "radial_symmetry": ref.radial_symmetry(), "solution_change": ref.solution_change(),
               "digests": [plane_digest(a) for a in list(cons) + list(phys)]}
        meta["results"][str(cp)] = res
        if not digest_only:
            out[f"cons_{cp}"] = cons
            out[f"phys_{cp}"] = phys
    np.savez_compressed(HERE / f"{name}.npz", **out)
    (HERE / f"{name}.json").write_text(json.dumps(meta, indent=1, default=float))
    print("wrote", name)


def main():
    ref = os.environ.get("MPD_REFERENCE", "/root/reference")  # the reference source tree
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), f"REF={ref}", "ref"], check=True)
    record("channel_sine_24x12", cases.channel_config(L=24, M=12, a=0.1), False, [1, 10, 100])
    record("reference_default_40x20", cases.reference_default_config(L=40, M=20), True,
           [1, 10, 60])
    record("edge_segments_20x9", cases.edge_config(), False, [1, 10, 60])
    record("config1_channel_200x80", cases.channel_config(L=200, M=80), False, [1000],
           digest_only=True)


if __name__ == "__main__":
    main()
