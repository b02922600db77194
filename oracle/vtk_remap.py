"""CPU restatement of VtkIC::Apply and Impl::Interp (src/ics/vtk_ic.cpp:137-239),
test infrastructure only: the checker of the device remap.  numpy evaluates
each expression left to right in float64, the reference's order."""
import numpy as np


def interp(d, ni, nj, fi, fj):
    fi = np.clip(fi, 0.0, float(ni - 1))                       # vtk_ic.cpp:141-142
    fj = np.clip(fj, 0.0, float(nj - 1))
    i0 = np.minimum(fi.astype(np.int64), ni - 2)               # :145-146
    j0 = np.minimum(fj.astype(np.int64), nj - 2)
    ti = fi - i0.astype(np.float64)                            # :149-150
    tj = fj - j0.astype(np.float64)
    v00 = d[i0 + j0 * ni]
    v10 = d[(i0 + 1) + j0 * ni]
    v01 = d[i0 + (j0 + 1) * ni]
    v11 = d[(i0 + 1) + (j0 + 1) * ni]
    return (1.0 - ti) * (1.0 - tj) * v00 + ti * (1.0 - tj) * v10 + (1.0 - ti) * tj * v01 + ti * tj * v11


def remap(src8, ni, nj, L, M, gamma):
    """10 dense planes (L+2) x (M+3) from 8 point fields (rho, v_z, v_r,
    v_phi, H_z, H_r, H_phi, e) of ni x nj points."""
    i_scale = (ni - 1) / (float(L) - 1.0) if L > 1 else 0.0    # :203-205
    j_scale = (nj - 1) / float(M) if M > 0 else 0.0            # :206-208
    lg = np.arange(L, dtype=np.float64)[:, None] * i_scale
    mg = np.arange(M + 1, dtype=np.float64)[None, :] * j_scale
    fi = np.broadcast_to(lg, (L, M + 1))
    fj = np.broadcast_to(mg, (L, M + 1))
    v = [interp(src8[k], ni, nj, fi, fj) for k in range(8)]
    rho, vz, vr, vphi, Hz, Hr, Hphi, e = v
    p = (gamma - 1.0) * rho * e                                # :229
    P = p + 0.5 * (Hz * Hz + Hr * Hr + Hphi * Hphi)            # :230-233
    out = np.zeros((10, L + 2, M + 3))
    for k, a in enumerate((rho, vz, vr, vphi, e, p, P, Hz, Hr, Hphi)):
        out[k, 1:L + 1, 1:M + 2] = a
    return out
