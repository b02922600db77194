"""The plain-method channel workload as an oracle case, built without the
product package — TEST INFRASTRUCTURE ONLY.

bench.py's CPU legs (the reference arm and the ``cpu_baseline`` leg) time the
reference's own code and must not load the product library, so their inputs
come from here instead of from the package's config front end:

* with the reference build present (``oracle/_ref``): the wall profiles from
  the reference's own IGeometry plugin — ``short_cathode_cosine`` with equal
  inner radii is the straight channel r1 = 0.2, r2 = 0.8
  (src/geometries/short_cathode_cosine.cpp:44-67) — and the initial planes
  from its ExpressionIC over its Grid (src/ics/expression_ic.cpp:255-324,
  src/grid.cpp:20-42);
* without it: the same closed forms in numpy, in the same IEEE operations
  (Grid::Build's r = (1 - frac) r_in + frac r_out, ExpressionIC's p and P).

Boundaries: inlet (l_lo) fixed at the initial values, zero-gradient outlet
(l_hi), slip walls (m_lo / m_hi: zero gradient except v_r = v_z r_z and
H_r = H_z r_z).  The dict layout is oracle/bind.py's case.
"""
from __future__ import annotations

import numpy as np

from . import bind

GAMMA = 5.0 / 3.0
# driver-loop constants of the channel workload (adaptive dt)
DRIVER = dict(dt0=1e-5, cfl=0.4, growth=1.1, dt_min=1e-12, dt_max=1.0)


def _exprs(amp: float):
    hphi = "0.2 / r" if amp == 1.0 else f"{amp!r} * 0.2 / r"
    return hphi, "beta / (2 * (gamma - 1))"


def _bc(vz: float, amp: float) -> dict:
    hphi, e_expr = _exprs(amp)
    neu = ("neumann", 0.0)
    inlet = {"range": (-1, -1), "rho": ("dirichlet", 1.0), "v_z": ("dirichlet", vz),
             "v_r": ("dirichlet", 0.0), "v_phi": ("dirichlet", 0.0), "e": ("expr", e_expr),
             "H_z": ("dirichlet", 0.0), "H_r": ("dirichlet", 0.0), "H_phi": ("expr", hphi)}
    outlet = {"range": (-1, -1), **{f: neu for f in bind.COND_FIELDS}}
    wall = {"range": (-1, -1), **{f: neu for f in bind.COND_FIELDS},
            "v_r": ("expr", "v_z * r_z"), "H_r": ("expr", "H_z * r_z")}
    return {"l_lo": [inlet], "l_hi": [outlet], "m_lo": [wall], "m_hi": [dict(wall)]}


def _profiles_numpy(L: int):
    n = L + 2
    return np.full(n, 0.2), np.full(n, 0.8), np.zeros(n), np.zeros(n)


def _ic_numpy(L, M, dy, beta, vz, amp, rin, rout) -> np.ndarray:
    rows, cols = L + 2, M + 3
    frac = np.arange(-1, M + 2, dtype=np.float64) * dy
    r = (1.0 - frac)[None, :] * rin[:, None] + frac[None, :] * rout[:, None]
    phys = np.zeros((10, rows, cols))
    inner = (slice(1, rows - 1), slice(1, cols - 1))
    rho = np.ones((rows, cols))
    hphi = (0.2 / r) if amp == 1.0 else (amp * 0.2 / r)
    e = np.full((rows, cols), beta / (2.0 * (GAMMA - 1.0)))
    p = (GAMMA - 1.0) * rho * e
    P = p + 0.5 * (0.0 * 0.0 + 0.0 * 0.0 + hphi * hphi)
    planes = {0: rho, 1: np.full((rows, cols), vz), 4: e, 5: p, 6: P, 9: hphi}
    for k, v in planes.items():
        phys[k][inner] = v[inner]
    return phys


def channel_case(L: int = 1600, M: int = 640, beta: float = 0.1, vz: float = 0.1,
                 amp: float = 1.0, use_reference: bool | None = None) -> dict:
    """Oracle case dict of the straight coaxial channel on an L x M grid."""
    dz, dy = 1.0 / L, 1.0 / M
    if use_reference is None:
        use_reference = bind.ref_available()
    if use_reference:
        rin, rout, drin, drout = bind.ref_geometry_profile(
            "short_cathode_cosine", {"z_center": 0.5, "transition_half_width": 0.1,
                                     "r_inner_before": 0.2, "r_inner_after": 0.2,
                                     "r_outer": 0.8}, L, dz)
    else:
        rin, rout, drin, drout = _profiles_numpy(L)
    r_0 = (rin[1] + rout[1]) / 2.0
    if use_reference:
        hphi, e_expr = _exprs(amp)
        ic = {"rho": "1", "v_z": repr(vz), "v_r": "0", "v_phi": "0", "H_z": "0", "H_r": "0",
              "H_phi": hphi, "e": e_expr}
        phys = bind.ref_expression_ic(ic, L, M, [GAMMA, beta, 0.0, dz, dy, r_0],
                                      rin, rout, drin, drout)
    else:
        phys = _ic_numpy(L, M, dy, beta, vz, amp, rin, rout)
    return dict(L=L, M=M, gamma=GAMMA, beta=beta, H_z0=0.0, dz=dz, dy=dy, r_0=r_0, rin=rin,
                rout=rout, drin=drin, drout=drout, phys=phys, bc=_bc(vz, amp),
                with_prev=False)
