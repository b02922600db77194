"""Snapshot I/O: the legacy-VTK structured grid of IOManager::WriteVtk
(src/io_manager.cpp:218-315), written and read without the VTK library, and
the restart initial condition VtkIC (src/ics/vtk_ic.cpp:137-239) whose
bilinear remap onto the new grid runs on the GPU (mpd_remap_snapshot).

File layout (binary legacy VTK, big-endian doubles): a structured grid of
(L+1) x (M+1) points, point (i, j) at (z = i dz, r = r[min(i, L-1)][j], 0)
with i fastest; point arrays Rho, Energy, MPI_Rank (one rank: zeros),
Hphi_times_r, and the vectors Velocity (v_z, v_r, v_phi) and MagneticField
(H_z, H_r, H_phi), each point taking row min(i, L-1) like the reference.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

from . import _native as N
from .ic import IInitialCondition

_SCALARS = ("Rho", "Energy", "MPI_Rank", "Hphi_times_r")
_VECTORS = ("Velocity", "MagneticField")


def snapshot_arrays(phys10: np.ndarray, r: np.ndarray, L: int, M: int) -> dict:
    """The point arrays of one snapshot from the 10 dense physical planes
    ((L+2) x (M+3), Fields member order) and the dense r plane."""
    li = np.minimum(np.arange(L + 1), L - 1) + 1          # plane row of point i
    mj = np.arange(M + 1) + 1                              # plane column of point j

    def pts(plane):                                        # (nj, ni) -> i fastest
        return plane[li][:, mj].T.copy()

    rho, vz, vr, vphi, e = (pts(phys10[k]) for k in (0, 1, 2, 3, 4))
    Hz, Hr, Hphi = (pts(phys10[k]) for k in (7, 8, 9))
    return {
        "Rho": rho, "Energy": e, "MPI_Rank": np.zeros_like(rho),
        "Hphi_times_r": Hphi * pts(r),
        "Velocity": np.stack([vz, vr, vphi], axis=-1),
        "MagneticField": np.stack([Hz, Hr, Hphi], axis=-1),
    }


def write_vtk(path, phys10: np.ndarray, r: np.ndarray, dz: float, L: int, M: int) -> pathlib.Path:
    """One snapshot as IOManager::WriteVtk writes it (file name of the
    reference's run loop: run_dir/step_NNNN.vtk, chosen by the caller)."""
    path = pathlib.Path(path)
    ni, nj = L + 1, M + 1
    n = ni * nj
    li = np.minimum(np.arange(ni), L - 1) + 1
    zz = np.broadcast_to((np.arange(ni) * dz)[None, :], (nj, ni))
    rr = r[li][:, 1:M + 2].T
    pts = np.stack([zz, rr, np.zeros((nj, ni))], axis=-1).reshape(n, 3)
    arrays = snapshot_arrays(phys10, r, L, M)
    be = ">f8"
    with open(path, "wb") as f:
        f.write(b"# vtk DataFile Version 5.1\nvtk output\nBINARY\nDATASET STRUCTURED_GRID\n")
        f.write(f"DIMENSIONS {ni} {nj} 1\nPOINTS {n} double\n".encode())
        f.write(pts.astype(be).tobytes())
        f.write(f"\nPOINT_DATA {n}\nFIELD FieldData {len(arrays)}\n".encode())
        for name in _SCALARS + _VECTORS:
            a = arrays[name]
            comps = 1 if a.ndim == 2 else a.shape[-1]
            f.write(f"{name} {comps} {n} double\n".encode())
            f.write(np.ascontiguousarray(a.reshape(n, comps)).astype(be).tobytes())
            f.write(b"\n")
    return path


def read_vtk(path) -> dict:
    """Point arrays (and 'dims') of a file written by write_vtk or by VTK's
    legacy structured-grid writer with a FIELD block of double arrays."""
    data = pathlib.Path(path).read_bytes()
    pos = 0

    def line():
        nonlocal pos
        end = data.index(b"\n", pos)
        s = data[pos:end].decode().strip()
        pos = end + 1
        return s

    out = {}
    ni = nj = n = None
    while pos < len(data):
        s = line()
        if not s:
            continue
        tok = s.split()
        if tok[0] == "DIMENSIONS":
            ni, nj = int(tok[1]), int(tok[2])
        elif tok[0] == "POINTS":
            n = int(tok[1])
            out["points"] = np.frombuffer(data, ">f8", n * 3, pos).reshape(n, 3)
            pos += n * 3 * 8
        elif tok[0] == "FIELD":
            for _ in range(int(tok[2])):
                s = line()
                while not s:
                    s = line()
                name, comps, count, _typ = s.split()
                comps, count = int(comps), int(count)
                a = np.frombuffer(data, ">f8", count * comps, pos).astype(np.float64)
                pos += count * comps * 8
                out[name] = a.reshape(count, comps) if comps > 1 else a
    out["dims"] = (ni, nj)
    return out


class VtkIC(IInitialCondition):
    """VtkIC (src/ics/vtk_ic.cpp): a snapshot remapped bilinearly onto the
    new grid by mpd_remap_snapshot on the device, p and P derived."""

    def __init__(self, path):
        self.path = str(path)
        self.snap = read_vtk(path)

    @staticmethod
    def source_fields(snap: dict) -> np.ndarray:
        v, h = snap["Velocity"], snap["MagneticField"]
        return np.stack([snap["Rho"], v[:, 0], v[:, 1], v[:, 2], h[:, 0], h[:, 1], h[:, 2],
                         snap["Energy"]])

    def Apply(self, grid, cfg):
        import torch
        lib = N.load()
        ni, nj = self.snap["dims"]
        src = torch.from_numpy(np.ascontiguousarray(self.source_fields(self.snap))).cuda()
        out = torch.zeros((10, cfg.L_max + 2, cfg.M_max + 3), dtype=torch.float64, device="cuda")
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        N.check(lib.mpd_remap_snapshot(C.c_void_p(src.data_ptr()), ni, nj, cfg.L_max, cfg.M_max,
                                       float(cfg.gamma), C.c_void_p(out.data_ptr()), stream), lib)
        return out.cpu().numpy()

    def Name(self):
        return "vtk"
