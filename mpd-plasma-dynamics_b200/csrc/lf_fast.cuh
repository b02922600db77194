// Per-warp arithmetic of the fast interior kernel (MPD_PRECISION_FAST;
// the kernel itself, with its TMA row staging, is lf_tma.cuh).
//
// Same update as Solver::ComputeCentralUpdate (src/solver.cpp:59-153),
// organised for registers and bandwidth:
//   * one warp owns a strip of 32 consecutive m columns (30 output cells;
//     lanes 0 and 31 are the strip's halo points) and marches down the rows
//     of its band, receiving each row of the 8 conserved planes once;
//   * every point is evaluated once (fast_prim / fast_gz / fast_gr) and folded
//     into two running sums: A for the cell row below it and, with the r
//     neighbours taken from the adjacent lanes by warp shuffles, B for its own
//     cell row, which is added to that row's A at once (S = A + B); a cell row
//     is closed when the point row after it arrives (fast_finish), so only 19
//     doubles of state (A of the next row, S of the current one) cross rows;
//   * divides are reciprocals from the hardware's approximate seed with one
//     polynomial correction (rcp_nr);
//   * a row's geometry (r profiles, dr) is loaded before its conserved values
//     are waited for, so those loads overlap the wait.
// The result differs from the exact kernel by rounding only (checked against
// the oracle at <= 1e-12 relative L-inf after 1000 steps).  Fused: the new
// state's maximum wave speed (adaptive dt) and the NaN/Inf sentinel.
#pragma once

#include <cuda_runtime.h>

#include "kernels.cuh"

namespace mpd {

constexpr int kFastCells = 30;  // output columns per warp

// Geometry of one point row: the wall radii and 0.5 / dr of the row (an
// IEEE division done once on the host instead of once per point and step).
struct RowGeo {
    double rin, rout, hdr;
};

struct FastStrip {
    Geo g;
    double *__restrict__ u;
    DevState *st;
    double *cphys;   // central lines (boundary inputs)
    int len;         // line length
    int p;           // this lane's point column
    bool pvalid;     // column inside [1, M+1]
    bool out_lane;   // lane writes a cell
    double frac, gm1, kz, dt;

    __device__ __forceinline__ RowGeo row_geo(int n) const {
        return RowGeo{__ldg(g.rin + n), __ldg(g.rout + n), __ldg(g.hdr + n)};
    }
    __device__ __forceinline__ double radius(const RowGeo &rg) const {
        return (1.0 - frac) * rg.rin + frac * rg.rout;
    }
    __device__ __forceinline__ bool ghost(int l) const { return !pvalid || l <= 0 || l >= g.L + 1; }

    // Point row n, a cell row of this strip: its B (the r neighbours' shares
    // by warp shuffles, its own sources) folded with the row's A into S, then
    // A replaced by the A this point row gives the cell row below it.  On a
    // ghost point U and q are zero, so its r fluxes are zero without a branch.
    // The shuffles have all 32 lanes taking part.
    __device__ __forceinline__ void point(const RowGeo &rg, const double U[8], const FastPrim &q,
                                          double r, const double Gz[8], double A[9],
                                          double S[10]) const {
        double Gr[8];
        fast_gr(U, q, r, Gr);
        // fast_rc + fast_b, each equation's two shuffles folded in as they arrive
        const double kr = dt * rg.hdr;
        double B[9];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const double q4 = 0.25 * U[k];
            const double ce = (k == 7) ? q4 : fma(kr, Gr[k], q4);
            const double cw = (k == 7) ? q4 : fma(-kr, Gr[k], q4);
            B[k] = __shfl_down_sync(0xffffffffu, ce, 1) + __shfl_up_sync(0xffffffffu, cw, 1);
        }
        const double d7 = __shfl_down_sync(0xffffffffu, Gr[7], 1) -
                          __shfl_up_sync(0xffffffffu, Gr[7], 1);
        B[2] = fma(dt, fma(q.rho * q.vphi, q.vphi, q.P) - q.Hphi * q.Hphi, B[2]);
        B[3] = fma(dt, fma(-q.rho * q.vr, q.vphi, q.Hphi * q.Hr), B[3]);
        B[4] = fma(-q.p * kr, d7, B[4]);
        B[8] = q.p;
        fast_sum(A, B, S);
        fast_a(U, Gz, kz, A);
    }

    // Primitives and z fluxes of point row n.  Ghost points (U = 0 by the
    // row staging) take 1/u_1 = 0 instead of a reciprocal of zero, which makes
    // every primitive and flux exactly zero, as the reference's zero ghost
    // values give, without a branch.
    __device__ __forceinline__ void eval(int n, const RowGeo &rg, const double U[8], FastPrim &q,
                                         double &r, double Gz[8]) const {
        const bool gh = ghost(n);
        r = gh ? 1.0 : radius(rg);  // a ghost column past the wall may have no positive radius
        q = fast_prim(U, r, gm1, gh);
        fast_gz(U, q, r, Gz);
    }
};

}  // namespace mpd
