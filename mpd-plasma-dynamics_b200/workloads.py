"""The plain-method workloads as configurations: the coaxial channel and the
parameter sweep of the batched steady-state solves.

Channel: z in [0, 1]; inner electrode r1 = 0.2; outer wall
r2(z) = 0.8 - a sin(pi z); grid L x M in (z, y) mapped by
r = (1 - y) r1 + y r2(z).  Fields rho, v_z, v_r, v_phi, B_z, B_r, B_phi and
specific internal energy with gamma = 5/3.  Initial condition rho = 1,
v_z = vz, v_r = v_phi = 0, p = beta/2 (e = beta / (2 (gamma - 1))),
B_phi = amp r1 / r, B_z = B_r = 0.  Inlet (l_lo) fixed at the initial values,
zero-gradient outlet (l_hi), slip walls (m_lo / m_hi: zero gradient except
v_r = v_z r_z and H_r = H_z r_z).  CFL 0.4, adaptive dt (growth 1.1,
dt_min 1e-12, dt_max 1, dt0 1e-5).

Sweep: solve i draws from numpy.random.default_rng(i): the grid uniformly
from {100x40, 200x80, 400x160, 800x320}, amp ~ U[0.5, 2],
beta ~ logU[0.05, 1], vz ~ U[0.05, 0.3], a ~ U[0, 0.2].
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .config import GeometryConfig, ICConfig, SimConfig, segment

SWEEP_GRIDS = ((100, 40), (200, 80), (400, 160), (800, 320))


def channel_config(L=200, M=80, a=0.0, beta=0.1, amp=1.0, vz=0.1, gamma=5.0 / 3.0,
                   adaptive=True, cfl=0.4) -> SimConfig:
    cfg = SimConfig(gamma=gamma, beta=beta, H_z0=0.0, L_max=L, M_max=M,
                    adaptive_dt=adaptive, cfl_number=cfl, dt_growth_factor=1.1,
                    dt_min=1e-12, dt_max=1.0, dt=1e-5, T=1e300)
    cfg.geometry = GeometryConfig("sine_wall", {"r1": 0.2, "r2": 0.8, "a": a})
    hphi = "0.2 / r" if amp == 1.0 else f"{amp!r} * 0.2 / r"
    e_expr = "beta / (2 * (gamma - 1))"
    cfg.initial_conditions = ICConfig(params={
        "rho": "1", "v_z": repr(vz), "v_r": "0", "v_phi": "0", "H_z": "0", "H_r": "0",
        "H_phi": hphi, "e": e_expr})
    cfg.bc_l_lo.segments = [segment(rho=("dirichlet", 1.0), v_z=("dirichlet", vz),
                                    v_r=("dirichlet", 0.0), v_phi=("dirichlet", 0.0),
                                    H_z=("dirichlet", 0.0), H_r=("dirichlet", 0.0),
                                    e=("expr", e_expr), H_phi=("expr", hphi))]
    cfg.bc_l_hi.segments = [segment()]
    wall = dict(v_r=("expr", "v_z * r_z"), H_r=("expr", "H_z * r_z"))
    cfg.bc_m_lo.segments = [segment(**wall)]
    cfg.bc_m_hi.segments = [segment(**wall)]
    cfg.init()
    return cfg


@dataclasses.dataclass(frozen=True)
class SweepParams:
    L: int
    M: int
    amp: float
    beta: float
    vz: float
    a: float

    def config(self) -> SimConfig:
        return channel_config(L=self.L, M=self.M, a=self.a, beta=self.beta, amp=self.amp,
                              vz=self.vz)

    def vector(self) -> np.ndarray:
        """(amp, beta, vz, a): the surrogate's parameter vector."""
        return np.array([self.amp, self.beta, self.vz, self.a])


def sweep_params(i: int, grids=SWEEP_GRIDS, a_max: float = 0.2) -> SweepParams:
    """Draw i of the sweep box; a_max widens the wall-amplitude range (the
    serving mix's large channel has a = 0.3, outside the sweep box)."""
    rng = np.random.default_rng(i)
    L, M = grids[int(rng.integers(len(grids)))]
    amp = float(rng.uniform(0.5, 2.0))
    beta = float(math.exp(rng.uniform(math.log(0.05), math.log(1.0))))
    vz = float(rng.uniform(0.05, 0.3))
    a = float(rng.uniform(0.0, a_max))
    return SweepParams(L, M, amp, beta, vz, a)
