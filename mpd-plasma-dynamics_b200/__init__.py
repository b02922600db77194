"""mpd_b200 — B200-native Lax-Friedrichs hot path of the axisymmetric MHD
plasma-thruster solver (seajoyer/mpd-plasma-dynamics).

The compute path is the CUDA library ``libmpd_b200.so`` behind the C ABI of
``include/mpd_b200.h``; this package is its Python host side: configuration
(``config``), geometry plugins and grid profiles (``geometry``), initial
conditions (``ic``), the solver handle (``solver``), batched solves and their
autotuner (``batch``), batched solves sharded over the GPUs of a node
(``sharding``).
"""
from . import _native, io, nn, serve, sharding, surrogate, warmstart, workloads
from .config import BCSegmentConfig, ConfigError, FieldCond, SimConfig, segment
from .geometry import GeometryRegistry, Grid, IGeometry, register_all_geometries
from .ic import ArrayIC, ExpressionIC, IInitialCondition
from .solver import GpuSolver, RunResult, build_case
from .batch import Autotuner, BatchPlan, BatchResult, BatchSolver

__all__ = [
    "SimConfig", "FieldCond", "BCSegmentConfig", "segment", "ConfigError",
    "IGeometry", "GeometryRegistry", "Grid", "register_all_geometries",
    "IInitialCondition", "ExpressionIC", "ArrayIC",
    "GpuSolver", "RunResult", "build_case",
    "BatchSolver", "BatchPlan", "BatchResult", "Autotuner",
]
