// Bilinear remap of a snapshot onto a new grid: VtkIC::Apply and Impl::Interp
// (src/ics/vtk_ic.cpp:137-239) as one device kernel, one thread per cell of
// the new grid.  Fractional source indices
//   i = l_global * (ni - 1) / (L_max - 1),   j = m_global * (nj - 1) / M_max
// (the reference's mapping, its axial scale included), clamped to the point
// range; the lower-left corner clamped so its +1 neighbours exist; weights
// (1-ti)(1-tj), ti(1-tj), (1-ti)tj, ti tj in that order; then p and P
// derived as ExpressionIC derives them.
#include <cuda_runtime.h>

#include <string>

#include "../../include/mpd_b200.h"

namespace mpd {
void SetLastError(const std::string &msg);
}

namespace {

__device__ __forceinline__ double interp(const double *d, int ni, int nj, double fi, double fj) {
    fi = fi < 0.0 ? 0.0 : (fi > (double)(ni - 1) ? (double)(ni - 1) : fi);
    fj = fj < 0.0 ? 0.0 : (fj > (double)(nj - 1) ? (double)(nj - 1) : fj);
    int i0 = (int)fi, j0 = (int)fj;
    if (i0 > ni - 2) i0 = ni - 2;
    if (j0 > nj - 2) j0 = nj - 2;
    const double ti = fi - (double)i0, tj = fj - (double)j0;
    const double v00 = d[(size_t)i0 + (size_t)j0 * ni];
    const double v10 = d[(size_t)(i0 + 1) + (size_t)j0 * ni];
    const double v01 = d[(size_t)i0 + (size_t)(j0 + 1) * ni];
    const double v11 = d[(size_t)(i0 + 1) + (size_t)(j0 + 1) * ni];
    return (1.0 - ti) * (1.0 - tj) * v00 + ti * (1.0 - tj) * v10 + (1.0 - ti) * tj * v01 +
           ti * tj * v11;
}

// src: 8 fields (rho, v_z, v_r, v_phi, H_z, H_r, H_phi, e) of ni x nj points,
// point (i, j) at i + j ni.  out: 10 dense planes (L+2) x (M+3) in the
// Fields member order, interior cells written, the rest untouched.
__global__ void remap_kernel(const double *src, int ni, int nj, int L, int M, double gamma,
                             double *out) {
    const int cols = M + 3, rows = L + 2;
    const size_t plane = (size_t)rows * cols, sp = (size_t)ni * nj;
    const double i_scale = L > 1 ? (double)(ni - 1) / ((double)L - 1.0) : 0.0;
    const double j_scale = M > 0 ? (double)(nj - 1) / (double)M : 0.0;
    const int n = L * (M + 1);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int lg = c / (M + 1), mg = c % (M + 1);
        const double fi = (double)lg * i_scale, fj = (double)mg * j_scale;
        double v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = interp(src + k * sp, ni, nj, fi, fj);
        const double rho = v[0], vz = v[1], vr = v[2], vphi = v[3];
        const double Hz = v[4], Hr = v[5], Hphi = v[6], e = v[7];
        const double p = (gamma - 1.0) * rho * e;
        const double P = p + 0.5 * (Hz * Hz + Hr * Hr + Hphi * Hphi);
        const size_t o = (size_t)(lg + 1) * cols + (mg + 1);
        const double planes[10] = {rho, vz, vr, vphi, e, p, P, Hz, Hr, Hphi};
#pragma unroll
        for (int k = 0; k < 10; ++k) out[k * plane + o] = planes[k];
    }
}

}  // namespace

extern "C" int mpd_remap_snapshot(const double *d_src, int ni, int nj, int L_max, int M_max,
                                  double gamma, double *d_out10, void *stream) {
    if (!d_src || !d_out10 || ni < 2 || nj < 2 || L_max < 1 || M_max < 1) {
        mpd::SetLastError("mpd_remap_snapshot: bad arguments (need ni, nj >= 2)");
        return MPD_ERR_INVALID;
    }
    const int n = L_max * (M_max + 1);
    int blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    remap_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_src, ni, nj, L_max,
                                                                         M_max, gamma, d_out10);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        mpd::SetLastError(std::string("mpd_remap_snapshot: ") + cudaGetErrorString(e));
        return MPD_ERR_CUDA;
    }
    return MPD_OK;
}
