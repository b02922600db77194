"""Build the native libraries in-tree with nvcc for sm_100a.

* ``libmpd_b200.so`` — the product: CUDA kernels + C ABI (include/mpd_b200.h).
* ``libmpd_emu.so``  — the same per-cell code compiled for the host, used only
  by the CPU test suite to check the kernels' boundary logic without a GPU.

Both are compiled with ``--fmad=false`` / ``-ffp-contract=off`` so that no
multiply-add is fused unless the source asks for it (the exact path must
round exactly like the reference's CPU build).
"""
from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
CSRC = PKG / "csrc"
ROOT = PKG.parent
LIB = PKG / "libmpd_b200.so"
EMU = PKG / "libmpd_emu.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_FLAGS = "-fPIC,-ffp-contract=off,-fno-fast-math,-O3"
COMMON = ["-std=c++17", "-O3", "--fmad=false", "-lineinfo", "-Xcompiler", HOST_FLAGS,
          f"-I{ROOT / 'include'}", f"-I{CSRC}"]


def _nvcc() -> str:
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not pathlib.Path(nvcc).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libmpd_b200.so")
    return nvcc


def _sources(*names):
    return [str(CSRC / n) for n in names]


def _stale(target: pathlib.Path) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    deps = list(CSRC.glob("*")) + [ROOT / "include" / "mpd_b200.h", pathlib.Path(__file__)]
    return any(d.stat().st_mtime > t for d in deps if d.is_file())


def build_lib(force: bool = False, verbose: bool = False) -> pathlib.Path:
    if not force and not _stale(LIB):
        return LIB
    cmd = [_nvcc(), *ARCH, *COMMON, "-shared", "-o", str(LIB),
           *_sources("mpd_abi.cu", "noalloc.cu", "nn_gemm.cu", "nn_ops.cu", "remap.cu", "bc_compile.cpp", "expr.cpp",
                    "ic_host.cpp")]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    env = dict(os.environ)
    env.pop("CC", None)   # nvcc picks the host compiler from PATH
    env.pop("CXX", None)
    res = subprocess.run(cmd, capture_output=True, text=True, env=env)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libmpd_b200.so")
    if verbose:
        sys.stderr.write(res.stderr)
    return LIB


def build_emu(force: bool = False) -> pathlib.Path:
    if not force and not _stale(EMU):
        return EMU
    gxx = shutil.which("g++-13") or "/usr/bin/g++"
    cmd = [gxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
           f"-I{ROOT / 'include'}", f"-I{CSRC}", "-o", str(EMU),
           *_sources("emu.cpp", "bc_compile.cpp", "expr.cpp", "ic_host.cpp")]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("g++ failed building libmpd_emu.so")
    return EMU


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_lib(force=force, verbose=verbose)
    build_emu(force=force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB, EMU)
