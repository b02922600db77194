"""The reference's own driver pattern with its Solver replaced by GpuSolver
(mpd-plasma-dynamics_b200/host/gpu_solver.hpp), compiled against the
reference's headers (oracle/Makefile `dropin`), must leave every Fields array
bit-identical to the reference's CPU Solver."""
import pathlib
import subprocess

import pytest

pytestmark = pytest.mark.gpu

BIN = pathlib.Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "dropin_check"


@pytest.mark.skipif(not BIN.exists(), reason="drop-in check not built (needs the reference sources)")
@pytest.mark.parametrize("L,M,steps", [(80, 40, 300), (160, 64, 150)])
def test_gpu_solver_is_a_drop_in_for_solver(L, M, steps):
    out = subprocess.run([str(BIN), str(L), str(M), str(steps)], capture_output=True, text=True,
                         timeout=600, env={"OMP_NUM_THREADS": "1", "PATH": "/usr/bin:/bin"})
    assert out.returncode == 0, out.stdout + out.stderr
    assert "DROPIN OK" in out.stdout
