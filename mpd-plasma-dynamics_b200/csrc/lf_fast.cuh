// Fast interior kernel of the plain FP64 path (MPD_PRECISION_FAST).
//
// Same update as Solver::ComputeCentralUpdate (src/solver.cpp:59-153), with
// the per-point quantities each cell's 5-point stencil needs computed once per
// point instead of once per use:
//   * one warp owns a strip of 32 consecutive m columns (30 output cells,
//     lanes 0 and 31 are the strip's halo) and marches down TL rows, keeping
//     rows l-1, l and the prefetched row l+1 in registers;
//   * z neighbours come from the register window, r neighbours from the
//     adjacent lanes through warp shuffles;
//   * divides become one reciprocal of u_1 and one of r per point and the
//     constant factors dt/(2 dz), dt/(2 dr_l) per row; sums use FMA.
// The result differs from the exact kernel by rounding only (checked against
// the oracle at <= 1e-12 relative L-inf after 1000 steps).
#pragma once

#include <cuda_runtime.h>

#include "kernels.cuh"

namespace mpd {

constexpr int kFastWarps = 4;   // warps per block, stacked along l
constexpr int kFastRows = 16;   // rows per warp
constexpr int kFastCells = 30;  // output columns per warp

__global__ void __launch_bounds__(32 * kFastWarps) lf_fast_kernel(Geo g, double *buf0, double *buf1,
                                                                   DevState *st, double dt_arg,
                                                                   int use_state_dt) {
    if (st->done) return;
    const long long step = st->step;
    const double *__restrict__ u0 = (step & 1) ? buf1 : buf0;
    double *__restrict__ u = (step & 1) ? buf0 : buf1;
    const double dt = use_state_dt ? st->dt : dt_arg;
    const int flags = step_flags(st);
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int p = 1 + kFastCells * (int)blockIdx.x + lane;  // this lane's point column
    const int l_begin = 1 + ((int)blockIdx.y * kFastWarps + wib) * kFastRows;
    const int l_end = min(l_begin + kFastRows, g.L + 1);     // exclusive
    const bool pvalid = p <= g.M + 1;
    const bool out_lane = lane >= 1 && lane <= kFastCells && p >= 2 && p <= g.M;
    const double frac = (double)(p - 1) * g.dy;
    const double gm1 = g.gamma - 1.0;
    const double kz = dt * (0.5 / g.dz);

    CellStats cs;
    cs.init();

    if (l_begin <= g.L) {
        auto load_row = [&](int l, double U[8]) {
            if (pvalid && l >= 0 && l <= g.L + 1) {
                const size_t i = g.ix(l, p);
#pragma unroll
                for (int k = 0; k < 8; ++k) U[k] = __ldg(u0 + (size_t)k * g.ps + i);
            } else {
#pragma unroll
                for (int k = 0; k < 8; ++k) U[k] = 0.0;
            }
        };
        auto point = [&](int l, const double U[8], ZPoint &z, RPoint &q) {
            if (!pvalid || l <= 0 || l >= g.L + 1) {
                zero_point(z, q);  // ghost rows hold zero state, zero fluxes
                return;
            }
            const double r = (1.0 - frac) * g.rin[l] + frac * g.rout[l];
            fast_point(U, r, gm1, z, q);
        };

        ZPoint zS, zC, zN;
        RPoint qS, qC, qN;
        double Ua[8], Ub[8];
        load_row(l_begin - 1, Ua);
        load_row(l_begin, Ub);
        point(l_begin - 1, Ua, zS, qS);
        point(l_begin, Ub, zC, qC);
        double Upre[8];
        load_row(l_begin + 1, Upre);

        for (int l = l_begin; l < l_end; ++l) {
            double Un[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) Un[k] = Upre[k];
            if (l + 2 <= l_end) load_row(l + 2, Upre);  // prefetch one row ahead
            point(l + 1, Un, zN, qN);

            const double kr = dt * (0.5 / g.dr[l]);
            double Ue[8], Uw[8], Ge[8], Gw[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                Uw[k] = __shfl_up_sync(0xffffffffu, zC.U[k], 1);
                Ue[k] = __shfl_down_sync(0xffffffffu, zC.U[k], 1);
                Gw[k] = __shfl_up_sync(0xffffffffu, qC.Gr[k], 1);
                Ge[k] = __shfl_down_sync(0xffffffffu, qC.Gr[k], 1);
            }
            double out[8];
            fast_cell(zS, zN, qC, Ue, Uw, Ge, Gw, kz, kr, dt, out);
            if (out_lane) {
                const size_t i = g.ix(l, p);
#pragma unroll
                for (int k = 0; k < 8; ++k) u[(size_t)k * g.ps + i] = out[k];
                if (p == g.M && (l == 1 || l == g.L)) {
#pragma unroll
                    for (int k = 0; k < 8; ++k) st->snap[(l == 1 ? 0 : 8) + k] = out[k];
                }
                if (l >= 2 && l <= g.L - 1 && flags) {
                    if (flags & kFlagWs) {
                        const double r = (1.0 - frac) * g.rin[l] + frac * g.rout[l];
                        cs.add_ws(fast_wave_speed(out, r, g.gamma));
                    }
                    if (flags & kFlagRes) cs.add_res(out, zC.U);
                }
            }
            // slide the window
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                zS.U[k] = zC.U[k];
                zS.Gz[k] = zC.Gz[k];
                zC.U[k] = zN.U[k];
                zC.Gz[k] = zN.Gz[k];
                qC.Gr[k] = qN.Gr[k];
            }
            qC.S3 = qN.S3;
            qC.S4 = qN.S4;
            qC.p = qN.p;
        }
    }
    if (flags) cs.flush(st, flags);
}

inline void launch_lf_fast(const Geo &g, double *buf0, double *buf1, DevState *st, double dt,
                           int use_state_dt, cudaStream_t stream) {
    const int gx = (g.M - 1 + kFastCells - 1) / kFastCells;
    const int rows_per_block = kFastWarps * kFastRows;
    const int gy = (g.L + rows_per_block - 1) / rows_per_block;
    lf_fast_kernel<<<dim3(gx, gy), 32 * kFastWarps, 0, stream>>>(g, buf0, buf1, st, dt,
                                                                 use_state_dt);
}

}  // namespace mpd
