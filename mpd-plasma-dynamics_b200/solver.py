"""``GpuSolver``: the drop-in for the reference's ``Solver`` on one B200.

Method names follow the reference classes they replace (Solver::Advance,
Diagnostics::ComputeDt / MaxWaveSpeed / SolutionChange / GetMassFlux /
GetThrust, Fields::SavePrev, Verification::ComputeIntegrals /
CheckRadialSymmetry), and ``run`` is the graph-resident form of the driver
loop of src/main.cpp:191-282.  All state lives on the device; everything is a
call through the C ABI of include/mpd_b200.h.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _native as N
from .config import CConfig, SimConfig
from .geometry import GeometryRegistry, Grid
from .ic import ArrayIC, ExpressionIC, IInitialCondition

PRECISIONS = {"exact": N.PRECISION_EXACT, "fast": N.PRECISION_FAST}
ENGINES = {"auto": N.ENGINE_AUTO, "graph": N.ENGINE_GRAPH, "persistent": N.ENGINE_PERSISTENT}


@dataclasses.dataclass
class MonitorReport:
    """One periodic report of the driver loop (src/main.cpp:249-281)."""
    step: int
    t: float
    dt: float
    probe: tuple        # rho, v_z, v_phi, e, H_phi at the global cell (l 20, m 40)
    integrals: tuple    # Verification::ComputeIntegrals
    max_wave_speed: float
    dt_cfl: float
    cfl_warning: bool   # Diagnostics::CheckCfl's warning condition

    @classmethod
    def from_record(cls, r) -> "MonitorReport":
        return cls(r.step, r.t, r.dt, tuple(r.probe), tuple(r.integrals), r.max_wave_speed,
                   r.dt_cfl, bool(r.cfl_warning))


def reference_report(rep: MonitorReport, cfl_number: float, out=None) -> None:
    """Print a report the way the reference's driver does: the CheckCfl warning
    (src/diagnostics.cpp:112-125, only at multiples of 1000 steps), the
    checkpoint line (src/main.cpp:268-270) and the integral table row
    (Verification::PrintIntegrals, src/verification.cpp:59-66)."""
    import sys
    out = out or sys.stdout
    if rep.cfl_warning and rep.step % 1000 == 0:
        out.write(f"WARNING [step {rep.step}]: dt={rep.dt:.6e} exceeds CFL limit "
                  f"dt_max={rep.dt_cfl:.6e} (max_speed={rep.max_wave_speed:.3f}, "
                  f"CFL={rep.dt / rep.dt_cfl * cfl_number:.2f})\n")
    p = rep.probe
    out.write(f"{rep.t:<14.6f} {rep.dt:<14.6e} {p[0]:<14.6f} {p[1]:<14.6f} {p[2]:<14.6f} "
              f"{p[3]:<14.6f} {p[4]:<14.6f}\n")
    q = rep.integrals
    out.write(f"  {rep.step:<8d}  {rep.t:<12.5f}  " + "  ".join(f"{v:<14.6e}" for v in q) + "\n")


@dataclasses.dataclass
class RunResult:
    steps: int
    t: float
    dt: float
    residual: float
    change: float
    max_wave_speed: float
    converged: bool
    status: int
    device_ms: float


def _dp(a: np.ndarray):
    return a.ctypes.data_as(N.DP)


class GpuSolver:
    """One solve on the GPU.

    ``GpuSolver(cfg, grid, ic)`` does what the reference's main does between
    the Grid and the time loop: InitPhysical (``ic``), InitConservative,
    SavePrev when convergence checking is on, and the Solver ctor (boundary
    configuration validated and compiled).
    """

    def __init__(self, cfg: SimConfig, grid: Grid, ic: IInitialCondition | np.ndarray,
                 precision: str = "fast", with_prev: bool | None = None):
        self.lib = N.load()
        self.cfg = cfg
        self.grid = grid
        # an expression IC is evaluated on the device after creation
        on_device = isinstance(ic, ExpressionIC)
        if isinstance(ic, np.ndarray):
            phys = ArrayIC(ic).Apply(grid, cfg)
        else:
            phys = None if on_device else ic.Apply(grid, cfg)
        self.shape = (cfg.L_max + 2, cfg.M_max + 3)
        if with_prev is None:
            with_prev = cfg.convergence_threshold > 0.0
        self.with_prev = with_prev
        self._cc = CConfig(cfg, grid.r_0, PRECISIONS[precision], with_prev)
        self._prof = [np.ascontiguousarray(a, dtype=np.float64) for a in grid.profiles()]
        geo = N.Geometry(*(_dp(a) for a in self._prof))
        if phys is not None:
            phys = np.ascontiguousarray(phys, dtype=np.float64)
        h = C.c_void_p()
        N.check(self.lib.mpd_create(self._cc.ptr, C.byref(geo),
                                    _dp(phys) if phys is not None else None, C.byref(h)), self.lib)
        self.h = h
        self.precision = precision
        if on_device:
            rc = ic.ApplyDevice(self.lib, self.h)
            if rc == N.MPD_ERR_UNSUPPORTED_IC:
                # order-dependent expressions: the reference's sequential sweep
                self.set_physical(ic.Apply(grid, cfg))
            elif rc != N.MPD_OK:
                self.close()
                N.check(rc, self.lib)

    # -- lifetime -------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.lib.mpd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _call(self, name, *args):
        N.check(getattr(self.lib, name)(self.h, *args), self.lib)

    # -- hot path ---------------------------------------------------------------
    def Advance(self, dt: float) -> None:
        """Solver::Advance (src/solver.cpp:22-37); asynchronous."""
        self._call("mpd_advance", float(dt))

    def run(self, T: float = float("inf"), dt: float | None = None, adaptive: bool | None = None,
            max_steps: int = 1 << 40, residual_tol: float = 0.0, residual_every: int | None = None,
            convergence_threshold: float | None = None, check_frequency: int | None = None,
            steps_per_graph: int = 0, engine: str = "auto", monitor=None,
            monitor_every: int = 1000) -> RunResult:
        """Graph-resident driver loop (src/main.cpp:191-282).

        The L-inf residual (a separate pass over both state buffers) is
        evaluated every ``residual_every`` steps: by default every 50 steps
        when ``residual_tol`` is set, otherwise only for the final state.
        ``engine``: "graph" (two kernels per step from captured CUDA graphs),
        "persistent" (one cooperative launch for many steps; fast precision
        without convergence_threshold) or "auto" (graph); both give the same bits.
        ``monitor``: a callable given a ``MonitorReport`` after every
        ``monitor_every`` steps (the reference driver's 1000-step checkpoint,
        integrals and CheckCfl; ``reference_report`` prints it the reference's
        way); graph engine only.
        """
        cfg = self.cfg
        if residual_every is None:
            residual_every = 50 if residual_tol > 0.0 else 0
        p = N.RunParams()
        p.T = T
        p.dt = cfg.dt if dt is None else dt
        p.adaptive = int(cfg.adaptive_dt if adaptive is None else adaptive)
        p.cfl_number, p.dt_growth_factor = cfg.cfl_number, cfg.dt_growth_factor
        p.dt_min, p.dt_max = cfg.dt_min, cfg.dt_max
        p.convergence_threshold = (cfg.convergence_threshold if convergence_threshold is None
                                   else convergence_threshold)
        p.check_frequency = cfg.check_frequency if check_frequency is None else check_frequency
        p.residual_tol = residual_tol
        p.residual_every = residual_every
        p.max_steps = int(max_steps)
        p.steps_per_graph = steps_per_graph
        p.engine = ENGINES[engine]
        errors = []
        if monitor is not None:
            def _cb(rec, _user):
                try:
                    monitor(MonitorReport.from_record(rec.contents))
                except Exception as exc:  # noqa: BLE001 - re-raised after the run
                    errors.append(exc)
            cb = N.MonitorFn(_cb)
            p.monitor = cb
            p.monitor_every = int(monitor_every)
        st = N.RunStats()
        rc = self.lib.mpd_run(self.h, C.byref(p), C.byref(st))
        if errors:
            raise errors[0]
        if rc not in (N.MPD_OK, N.MPD_ERR_NONFINITE):
            N.check(rc, self.lib)
        return RunResult(st.steps, st.t, st.dt, st.residual, st.change, st.max_wave_speed,
                         bool(st.converged), st.status, st.device_ms)

    # -- diagnostics -------------------------------------------------------------
    def _scalar(self, name) -> float:
        out = C.c_double()
        self._call(name, C.byref(out))
        return out.value

    def MaxWaveSpeed(self) -> float:
        return self._scalar("mpd_max_wave_speed")

    def ComputeDt(self, dt_current: float) -> float:
        cfg = self.cfg
        out = C.c_double()
        self._call("mpd_compute_dt", cfg.cfl_number, cfg.dt_growth_factor, cfg.dt_min,
                   cfg.dt_max, float(dt_current), C.byref(out))
        return out.value

    def SolutionChange(self) -> float:
        return self._scalar("mpd_solution_change")

    def SavePrev(self) -> None:
        self._call("mpd_save_prev")

    def CheckRadialSymmetry(self) -> float:
        return self._scalar("mpd_radial_symmetry")

    def residual(self) -> float:
        return self._scalar("mpd_residual")

    def ComputeIntegrals(self) -> np.ndarray:
        out = np.zeros(7)
        self._call("mpd_integrals", _dp(out))
        return out

    def outlet(self):
        a, b = C.c_double(), C.c_double()
        self._call("mpd_outlet", C.byref(a), C.byref(b))
        return a.value, b.value

    def GetMassFlux(self) -> float:
        return self.outlet()[0]

    def GetThrust(self) -> float:
        return self.outlet()[1]

    def probe(self, l_global: int, m_global: int) -> np.ndarray:
        out = np.zeros(10)
        self._call("mpd_probe", int(l_global), int(m_global), _dp(out))
        return out

    def time(self):
        t = C.c_double()
        s = C.c_longlong()
        self._call("mpd_time", C.byref(t), C.byref(s))
        return t.value, s.value

    # -- state -------------------------------------------------------------------
    def download(self, which: int) -> np.ndarray:
        out = np.empty(self.shape)
        self._call("mpd_download", int(which), _dp(out))
        return out

    def conserved(self) -> np.ndarray:
        return np.stack([self.download(k) for k in range(8)])

    def physical(self) -> np.ndarray:
        return np.stack([self.download(8 + k) for k in range(10)])

    def snapshot_async(self, pinned_phys10) -> None:
        """IOManager's output planes (src/io_manager.cpp:68-77): the 10 physical
        planes of the current state, copied on a side stream into caller-owned
        pinned host memory of shape (10, L+2, M+3) (a pinned torch tensor, or
        any object with ``data_ptr()``); stepping may continue meanwhile.  The
        buffer is complete after ``snapshot_wait``."""
        ptr = pinned_phys10.data_ptr() if hasattr(pinned_phys10, "data_ptr") else \
            pinned_phys10.ctypes.data
        self._call("mpd_snapshot_async", C.cast(C.c_void_p(ptr), N.DP))

    def snapshot_wait(self) -> None:
        self._call("mpd_snapshot_wait")

    def set_physical(self, phys10: np.ndarray) -> None:
        a = np.ascontiguousarray(phys10, dtype=np.float64)
        self._call("mpd_set_physical", _dp(a))

    def stream_handle(self) -> int:
        s = C.c_void_p()
        self._call("mpd_get_stream", C.byref(s))
        return s.value or 0

    @property
    def ring_overlap(self) -> bool:
        """Whether fast steps run the boundary ring beside the interior kernel
        (bc_overlap_kernel) instead of after it (bc_kernel, the default); both
        give the same bits.  Setting it takes effect from the next step."""
        a = C.c_int()
        self._call("mpd_ring_overlap_active", C.byref(a))
        return bool(a.value)

    @ring_overlap.setter
    def ring_overlap(self, on: bool) -> None:
        self._call("mpd_set_ring_overlap", 1 if on else 0)

    def profile_kernels(self, steps: int, dt: float):
        """Mean device ms per launch of (interior kernel, boundary kernel)."""
        out = np.zeros(2)
        self._call("mpd_profile_kernels", int(steps), float(dt), _dp(out))
        return float(out[0]), float(out[1])

    def profile_kernel(self, which: str, launches: int, dt: float) -> float:
        """Mean device ms of one launch of the interior kernel ("interior"),
        its two-column form ("interior_pair") or the residual pass
        ("residual"), from back-to-back launches."""
        out = np.zeros(1)
        k = {"interior": N.KERNEL_INTERIOR, "residual": N.KERNEL_RESIDUAL,
             "interior_pair": N.KERNEL_INTERIOR_PAIR}[which]
        self._call("mpd_profile_kernel", k, int(launches), float(dt), _dp(out))
        return float(out[0])

    def device_bytes(self) -> int:
        b = C.c_size_t()
        self._call("mpd_device_bytes", C.byref(b))
        return b.value


def build_case(cfg: SimConfig, precision: str = "fast", with_prev: bool | None = None,
               ic: IInitialCondition | None = None) -> GpuSolver:
    """Everything src/main.cpp does before the time loop, from a SimConfig."""
    geom = GeometryRegistry.Instance().Create(cfg.geometry.type, cfg.geometry.params)
    grid = Grid(cfg, geom)
    if ic is None:
        if cfg.initial_conditions.vtk_file:
            from .io import VtkIC
            ic = VtkIC(cfg.initial_conditions.vtk_file)
        else:
            ic = ExpressionIC(cfg.initial_conditions.params)
    return GpuSolver(cfg, grid, ic, precision=precision, with_prev=with_prev)
