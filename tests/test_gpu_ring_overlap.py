"""The boundary ring beside the interior kernel (bc_overlap_kernel) against
the ring after it (bc_kernel reading the central cells the interior stored,
the fast path's default): the ring-beside form recomputes those cells from
the step's input state with the interior warp's own operations, so every
plane, dt and t must agree bit for bit, through the graph loop and through
the per-call Advance / ComputeDt pattern, and the ring-beside form is
checked against the oracle here as well."""
import numpy as np
import pytest

from oracle import bind
from tests import cases

pytestmark = pytest.mark.gpu

CASES = [
    ("channel_400x160", lambda: cases.channel_config(L=400, M=160, a=0.1), 1e-5),
    ("reference_default", lambda: cases.reference_default_config(L=80, M=40), 1e-6),
    ("edge_segments", lambda: cases.edge_config(), 1e-4),
    ("channel_6x9", lambda: cases.channel_config(L=6, M=9, a=0.1), 1e-4),
]


def _pair(pkg, cfg):
    case = cases.make_case(cfg)
    beside = pkg.GpuSolver(case.cfg, case.grid, case.phys, precision="fast")
    after = pkg.GpuSolver(case.cfg, case.grid, case.phys, precision="fast")
    beside.ring_overlap = True
    after.ring_overlap = False
    assert beside.ring_overlap and not after.ring_overlap
    return case, beside, after


@pytest.mark.parametrize("name,make,dt0", CASES)
def test_graph_run_bitwise(pkg, name, make, dt0):
    case, beside, after = _pair(pkg, make())
    for n, per in ((150, 50), (97, 97)):
        a = beside.run(T=1e300, dt=dt0, adaptive=True, max_steps=n, steps_per_graph=per)
        b = after.run(T=1e300, dt=dt0, adaptive=True, max_steps=n, steps_per_graph=per)
        assert (a.steps, a.dt, a.t) == (b.steps, b.dt, b.t)
        np.testing.assert_array_equal(beside.conserved(), after.conserved())
        dt0 = a.dt
    np.testing.assert_array_equal(beside.physical(), after.physical())
    beside.close()
    after.close()


@pytest.mark.parametrize("name,make,dt0", CASES[1:3])
def test_per_call_steps_bitwise_and_near_oracle(pkg, name, make, dt0):
    case, beside, after = _pair(pkg, make())
    oracle = bind.Port(case.oracle_dict())
    cfg = case.cfg
    dt = dt0
    for _ in range(60):
        beside.Advance(dt)
        after.Advance(dt)
        oracle.advance(dt)
        d1, d2 = beside.ComputeDt(dt), after.ComputeDt(dt)
        assert d1 == d2
        dt = d1 if cfg.adaptive_dt else dt
    got = beside.conserved()
    np.testing.assert_array_equal(got, after.conserved())
    want = oracle.conserved()
    for k in range(8):
        den = max(np.abs(want[k]).max(), 1e-300)
        assert np.abs(got[k] - want[k]).max() / den <= 1e-12
    beside.close()
    after.close()
    oracle.close()


def test_switching_mid_run_keeps_the_bits(pkg):
    """Alternating the two forms between runs gives the same state as either alone."""
    case, beside, after = _pair(pkg, cases.channel_config(L=200, M=80, a=0.05))
    dt = case.cfg.dt
    for i in range(6):
        beside.ring_overlap = i % 2 == 0
        a = beside.run(T=1e300, dt=dt, adaptive=True, max_steps=40, steps_per_graph=20)
        b = after.run(T=1e300, dt=dt, adaptive=True, max_steps=40, steps_per_graph=20)
        assert a.dt == b.dt
        dt = a.dt
    np.testing.assert_array_equal(beside.conserved(), after.conserved())
    beside.close()
    after.close()
