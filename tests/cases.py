"""Shared test cases: a SimConfig, its grid and initial planes, and the same
inputs in the oracle's dict form (oracle/bind.py)."""
from __future__ import annotations

import dataclasses

import numpy as np

import __graft_entry__

pkg = __graft_entry__.load_package()
SimConfig = pkg.SimConfig
segment = pkg.segment


@dataclasses.dataclass
class Case:
    cfg: object
    grid: object
    phys: np.ndarray

    def oracle_dict(self, with_prev: bool = False) -> dict:
        cfg, grid = self.cfg, self.grid
        bc = {}
        for name, face in zip(("l_lo", "l_hi", "m_lo", "m_hi"), cfg.faces()):
            segs = []
            for s in face.segments:
                d = {"range": (s.global_lo, s.global_hi)}
                for f in pkg.config.SEGMENT_FIELDS:
                    fc = getattr(s, f)
                    kind = {"neumann": "neumann", "dirichlet": "dirichlet",
                            "expression": "expr", "axis_lf": "axis_lf"}[fc.type]
                    d[f] = (kind, fc.expr_str if kind == "expr" else fc.value)
                segs.append(d)
            bc[name] = segs
        return dict(L=cfg.L_max, M=cfg.M_max, gamma=cfg.gamma, beta=cfg.beta, H_z0=cfg.H_z0,
                    dz=cfg.dz, dy=cfg.dy, r_0=grid.r_0, rin=grid.rin, rout=grid.rout,
                    drin=grid.drin, drout=grid.drout, phys=self.phys, bc=bc,
                    with_prev=with_prev)


def make_case(cfg) -> Case:
    geom = pkg.GeometryRegistry.Instance().Create(cfg.geometry.type, cfg.geometry.params)
    grid = pkg.Grid(cfg, geom)
    phys = pkg.ExpressionIC(cfg.initial_conditions.params).Apply(grid, cfg)
    return Case(cfg, grid, phys)


def channel_config(L=200, M=80, a=0.0, beta=0.1, amp=1.0, vz=0.1, gamma=5.0 / 3.0,
                   adaptive=True, cfl=0.4) -> object:
    """The straight / sine-wall coaxial channel of the plain-method workloads
    (mpd_b200.workloads.channel_config)."""
    return pkg.workloads.channel_config(L=L, M=M, a=a, beta=beta, amp=amp, vz=vz, gamma=gamma,
                                        adaptive=adaptive, cfl=cfl)


def channel_case(**kw) -> Case:
    return make_case(channel_config(**kw))


def reference_default_config(L=80, M=40) -> object:
    """The reference's own config.yaml (thin-electrode cosine geometry, three
    inner-wall segments ending in the AxisLF axis region), ranges scaled to L."""
    cfg = SimConfig.from_yaml(f"""
physics: {{gamma: 1.67, beta: 0.01, H_z0: 0.25}}
time: {{T: 6, dt: 1.0e-7}}
adaptive_dt: {{enabled: true, cfl_number: 0.45, growth_factor: 1.10, dt_min: 1.0e-10, dt_max: 5.0e-5}}
grid: {{L_max: {L}, M_max: {M}}}
geometry:
  type: short_cathode_cosine
  params: {{z_center: 0.31, transition_half_width: 0.02, r_inner_before: 0.200,
            r_inner_after: 0.005, r_outer: 0.800}}
initial_conditions:
  rho: 0.1
  v_z: 0.1
  v_r: 0.1
  v_phi: 0.0
  H_z: H_z0
  H_r: "H_z * r_z"
  H_phi: "(1 - 0.9 * z) * r_0 / r"
  e: "beta / (2 * (gamma - 1))"
boundary_conditions:
  l_lo:
    - {{rho: neumann, v_z: {{dirichlet: 0.0}}, v_r: neumann, v_phi: neumann, e: neumann,
       H_z: "H_z0", H_r: {{dirichlet: 0.0}}, H_phi: "r_0 / r"}}
  l_hi:
    - {{rho: neumann, v_z: neumann, v_r: neumann, v_phi: neumann, e: neumann, H_z: neumann,
       H_r: neumann, H_phi: neumann}}
  m_hi:
    - {{rho: neumann, v_z: neumann, v_r: "v_z * r_z", v_phi: neumann, e: neumann,
       H_z: neumann, H_r: "H_z * r_z", H_phi: neumann}}
  m_lo:
    - {{range: [0, {int(235 * L / 800)}], rho: neumann, v_z: neumann, v_r: "v_z_nb * r_z_nb",
       v_phi: neumann, e: neumann, H_z: neumann, H_r: "H_z_nb * r_z_nb", H_phi: neumann}}
    - {{range: [{int(236 * L / 800)}, {int(263 * L / 800)}], rho: {{dirichlet: 0.1}},
       v_z: neumann, v_r: neumann, v_phi: {{dirichlet: 0.0}}, e: "beta / (2 * (gamma - 1))",
       H_z: neumann, H_r: "H_z_nb * r_z_nb", H_phi: neumann}}
    - {{range: [{int(264 * L / 800)}, -1], rho: axis_lf, v_z: axis_lf, v_r: {{dirichlet: 0.0}},
       v_phi: {{dirichlet: 0.0}}, e: axis_lf, H_z: axis_lf, H_r: {{dirichlet: 0.0}},
       H_phi: {{dirichlet: 0.0}}}}
""")
    return cfg


def edge_config(L=20, M=9) -> object:
    """Boundary layouts the reference allows but rarely sees: overlapping
    segments, gaps that no segment covers, Neumann offsets, expressions over
    *_nb / dr / z / pi and math functions, AxisLF next to a Dirichlet v_z."""
    cfg = channel_config(L=L, M=M, a=0.15, beta=0.2, amp=1.5, vz=0.2)
    cfg.geometry = pkg.config.GeometryConfig("sine_wall", {"r1": 0.2, "r2": 0.8, "a": 0.15})
    cfg.bc_l_lo.segments = [
        segment((0, 4), rho=("dirichlet", 1.0), v_z=("dirichlet", 0.2), e=("neumann", 0.01)),
        segment((3, -1), rho=("expr", "1 + 0.1 * sin(pi * r)"), v_z=("expr", "0.2 * (1 - z)"),
                H_phi=("expr", "1.5 * 0.2 / r"), e=("expr", "beta / (2 * (gamma - 1))")),
    ]
    cfg.bc_l_hi.segments = [segment((0, M - 2)), segment((M - 1, M - 1), v_r=("dirichlet", 0.0))]
    cfg.bc_m_hi.segments = [segment((1, -1), v_r=("expr", "v_z * r_z"),
                                    H_r=("expr", "H_z * r_z + 0 * dr"))]
    cfg.bc_m_lo.segments = [
        segment((0, 6), v_r=("expr", "v_z_nb * r_z_nb"), H_r=("expr", "H_z_nb * r_z_nb")),
        segment((5, 12), rho="axis_lf", v_z=("dirichlet", 0.15), e="axis_lf", H_z="axis_lf",
                v_r=("dirichlet", 0.0), v_phi=("dirichlet", 0.0), H_r=("dirichlet", 0.0)),
        segment((13, -1), rho="axis_lf", v_z="axis_lf", e="axis_lf", H_z="axis_lf",
                v_r=("dirichlet", 0.0), v_phi=("dirichlet", 0.0), H_r=("dirichlet", 0.0),
                H_phi=("expr", "max(H_phi_nb, 0.1) * r_nb / r")),
    ]
    cfg.init()
    return cfg


def run_oracle_steps(o, n, dt0, cfg):
    """Fixed-step or adaptive stepping with the reference driver's dt update."""
    dt = dt0
    for _ in range(n):
        o.advance(dt)
        if cfg.adaptive_dt:
            dt = o.compute_dt(cfg.cfl_number, cfg.dt_growth_factor, cfg.dt_min, cfg.dt_max, dt)
    return dt
