// Conserved integrals over caller-owned device planes with no device
// allocation (C ABI entry point mpd_integrals_noalloc).
//
// Some callers cannot let a library call cudaMalloc: a host code whose
// framework owns every byte of device memory through its own pool (a stray
// cudaMalloc bypasses the pool's accounting, and fails outright once the
// pool has reserved the device), or a caller that has already handed its
// memory budget out and must not see new allocations appear.  For them this
// variant of Verification::ComputeIntegrals keeps its only scratch — one
// partial sum per grid row — in a fixed file-scope device array instead of
// the handle's cudaMalloc'd buffer.  The array belongs to this file's module:
// under CUDA's lazy module loading (the default) a device gets its copy when
// the first call on it loads the module, and keeps it until the process
// exits; with eager loading, when the library is loaded.
#include <cuda_runtime.h>

#include <string>

#include "../../include/mpd_b200.h"

namespace mpd {
void SetLastError(const std::string &msg);
}

namespace {

constexpr int kNoAllocMaxRows = 8192;   // grid rows L_max the scratch can hold

// One partial sum per row and integral (7 doubles per row, 458,752 bytes).
static __device__ __align__(256) double g_row_partials[kNoAllocMaxRows * 7];


// Row l = 1 + blockIdx.x: the 7 sums of Verification::ComputeIntegrals
// (src/verification.cpp:16-45) over m = 1..M+1, in order mass, mom_z, mom_r,
// mom_phi, energy, mag_flux_z (u_7), mag_flux_phi (u_6).
__global__ void noalloc_row_kernel(const double *__restrict__ u, size_t ps, int pitch, int M,
                                   const double *__restrict__ dr, double dz, double *partials) {
    const int l = 1 + blockIdx.x;
    const double cell_area = dr[l] * dz;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int m = 1 + threadIdx.x; m <= M + 1; m += blockDim.x) {
        const size_t i = static_cast<size_t>(l) * pitch + m;
        acc[0] += u[0 * ps + i] * cell_area;
        acc[1] += u[1 * ps + i] * cell_area;
        acc[2] += u[2 * ps + i] * cell_area;
        acc[3] += u[3 * ps + i] * cell_area;
        acc[4] += u[4 * ps + i] * cell_area;
        acc[5] += u[6 * ps + i] * cell_area;
        acc[6] += u[5 * ps + i] * cell_area;
    }
    __shared__ double red[32][7];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        double x = acc[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) red[warp][k] = x;
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w][threadIdx.x];
        partials[static_cast<size_t>(blockIdx.x) * 7 + threadIdx.x] = s;
    }
}

// Adds the row partials in row order into out7 (device memory).
__global__ void noalloc_sum_kernel(const double *partials, int rows, double *out7) {
    if (threadIdx.x >= 7) return;
    double s = 0.0;
    for (int r = 0; r < rows; ++r) s += partials[static_cast<size_t>(r) * 7 + threadIdx.x];
    out7[threadIdx.x] = s;
}

// The device address of g_row_partials in the current context.  In host code
// the symbol names a host-side stand-in, not device memory, so kernels are
// given this address instead.  It is looked up on every call rather than
// cached: a cached address would outlive a device reset or belong to another
// context (a framework may make a non-primary context current), and the
// lookup itself allocates nothing once the module is loaded.
int ScratchForCurrentContext(double **out) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_row_partials);
    if (e != cudaSuccess || !p) {
        mpd::SetLastError(std::string("mpd_integrals_noalloc: cudaGetSymbolAddress: ") +
                          cudaGetErrorString(e));
        return MPD_ERR_CUDA;
    }
    *out = static_cast<double *>(p);
    return MPD_OK;
}

}  // namespace

extern "C" int mpd_integrals_noalloc(const double *d_u, size_t plane_stride, int pitch, int L_max,
                                     int M_max, const double *d_dr, double dz, double *d_out7,
                                     void *stream) {
    if (!d_u || !d_dr || !d_out7 || L_max < 1 || M_max < 1 || pitch < M_max + 3 ||
        plane_stride < static_cast<size_t>(L_max + 2) * static_cast<size_t>(pitch)) {
        mpd::SetLastError("mpd_integrals_noalloc: bad arguments");
        return MPD_ERR_INVALID;
    }
    if (L_max > kNoAllocMaxRows) {
        mpd::SetLastError("mpd_integrals_noalloc: L_max = " + std::to_string(L_max) +
                          " exceeds the " + std::to_string(kNoAllocMaxRows) +
                          " rows its fixed scratch holds");
        return MPD_ERR_INVALID;
    }
    double *partials = nullptr;
    const int rc = ScratchForCurrentContext(&partials);
    if (rc != MPD_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // every row's partials are rewritten before they are summed: nothing in
    // the scratch has to start at zero
    noalloc_row_kernel<<<L_max, 128, 0, s>>>(d_u, plane_stride, pitch, M_max, d_dr, dz, partials);
    noalloc_sum_kernel<<<1, 32, 0, s>>>(partials, L_max, d_out7);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        mpd::SetLastError(std::string("mpd_integrals_noalloc: launch: ") + cudaGetErrorString(e));
        return MPD_ERR_CUDA;
    }
    return MPD_OK;
}
