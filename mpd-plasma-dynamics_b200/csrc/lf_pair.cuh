// Interior kernel of the plain FP64 path with two point columns per lane
// (MPD_PRECISION_FAST, steps >= 1 of the graph engine).
//
// Same per-point arithmetic as lf_tma_kernel (fast_prim, fast_gz, fast_gr,
// fast_a, fast_sum, fast_finish, fast_wave_speed, in the same operand order),
// so the results are bit-identical to it; what changes is the work per lane:
//   * a warp owns a strip of 64 point columns starting at x0 = 62 s (62
//     output cells x0+1 .. x0+62); lane i holds the adjacent points
//     a = x0 + 2i and b = x0 + 2i + 1, so of each point's two r neighbours
//     one is in the lane itself and only one crosses lanes: one warp shuffle
//     per equation and point instead of two, and the strip's halo is 2 of 64
//     points instead of 2 of 32;
//   * each staged row is one TMA tile {64 columns} x {1 row} x {8 planes}
//     (4 KB) read back as one 16-byte shared-memory load per plane, and the
//     two new cells of a lane leave as one 16-byte store per plane;
//   * the per-row work that does not depend on the point (geometry loads,
//     the wait for the staged row, loop control) is shared by two points.
// Two chains per lane also give the scheduler independent work at the
// register budget of two resident blocks per SM.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "lf_tma.cuh"

namespace mpd {

#ifndef MPD_PAIR_MINB
#define MPD_PAIR_MINB 2
#endif
#ifndef MPD_PAIR_STAGES
#define MPD_PAIR_STAGES 4
#endif
#ifndef MPD_PAIR_WARPS
#define MPD_PAIR_WARPS 4
#endif

constexpr int kPairCells = 62;                  // output columns per warp
constexpr int kPairWarps = MPD_PAIR_WARPS;      // warps per block
constexpr int kPairStages = MPD_PAIR_STAGES;    // rows in flight per warp
constexpr int kPairRow = 8 * 64;                // doubles per staged row
constexpr int kPairRowBytes = kPairRow * 8;     // 4096
constexpr int kPairSmem = kPairWarps * kPairStages * (kPairRowBytes + 8) + 128;

// A 16-byte store of two doubles carrying an L2 eviction-priority policy.
__device__ __forceinline__ void st_global_v2_hint(double *p, double a, double b, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(p), "d"(a), "d"(b),
                 "l"(pol)
                 : "memory");
}

// One point of a lane: its column and what it takes part in.
struct PairPt {
    int p;          // point column
    bool pvalid;    // column inside [0, M+1] (past M+1: ghost or tile fill)
    bool out;       // writes a cell: an output point of the strip with 2 <= p <= M
    double frac;    // (p - 1) dy
};

struct PairWarp {
    Geo g;
    double *__restrict__ u;
    DevState *st;
    double *cphys;
    int len;
    PairPt a, b;
    double gm1, kz, dt;
    uint64_t pol_read, pol_write;
    const CUtensorMap *map;
    double *stage;   // kPairStages rows of [8][64]
    uint32_t bar0;   // shared address of this warp's first barrier
    uint32_t jbase;  // running row count at the band's first staged row
    int x0;          // first column of the strip
    int row0;        // plane row of the band's first staged row
    int nrows;       // rows the band stages
    int lane;

    __device__ __forceinline__ uint32_t bar(uint32_t s) const { return bar0 + 8u * s; }

    __device__ __forceinline__ RowGeo row_geo(int n) const {
        return RowGeo{__ldg(g.rin + n), __ldg(g.rout + n), __ldg(g.hdr + n)};
    }

    __device__ __forceinline__ void issue(uint32_t j) const {
        if (lane == 0 && j - jbase < (uint32_t)nrows) {
            const uint32_t s = j % kPairStages;
            mbar_expect_tx(bar(s), kPairRowBytes);
#if MPD_L2_HINTS
            tma_load_3d_hint(smem_addr(stage + s * kPairRow), map, bar(s), x0,
                             row0 + (int)(j - jbase), 0, pol_read);
#else
            tma_load_3d(smem_addr(stage + s * kPairRow), map, bar(s), x0, row0 + (int)(j - jbase),
                        0);
#endif
        }
    }

    // Staged row j: the lane's two points of every plane; false if the wait gave up.
    __device__ __forceinline__ bool take(uint32_t j, double Ua[8], double Ub[8]) const {
        const uint32_t s = j % kPairStages;
        const bool ok =
            __all_sync(0xffffffffu, mbar_wait_bounded(bar(s), (j / kPairStages) & 1));
        const double2 *src = reinterpret_cast<const double2 *>(stage + s * kPairRow) + lane;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const double2 v = src[32 * k];
            Ua[k] = v.x;
            Ub[k] = v.y;
        }
        return ok;
    }

    __device__ __forceinline__ void release(uint32_t j) const {
        __syncwarp();
        issue(j + kPairStages);
    }

    // Primitives and z fluxes of one point of row n (FastStrip::eval).
    __device__ __forceinline__ void eval(const PairPt &pt, int n, const RowGeo &rg,
                                         const double U[8], FastPrim &q, double &r,
                                         double Gz[8]) const {
        const bool gh = !pt.pvalid || n <= 0 || n >= g.L + 1;
        r = gh ? 1.0 : (1.0 - pt.frac) * rg.rin + pt.frac * rg.rout;
        q = fast_prim(U, r, gm1, gh);
        fast_gz(U, q, r, Gz);
    }

    __device__ __forceinline__ void sources(const FastPrim &q, double kr, double d7,
                                            double B[9]) const {
        B[2] = fma(dt, fma(q.rho * q.vphi, q.vphi, q.P) - q.Hphi * q.Hphi, B[2]);
        B[3] = fma(dt, fma(-q.rho * q.vr, q.vphi, q.Hphi * q.Hr), B[3]);
        B[4] = fma(-q.p * kr, d7, B[4]);
        B[8] = q.p;
    }

    // Point row n of both points (FastStrip::point): B from the r neighbours
    // (one in the lane, one across lanes) and the point's sources, folded with
    // A into S; A replaced by the A this point row gives the row below.
    __device__ __forceinline__ void point(const RowGeo &rg, const double Ua[8],
                                          const FastPrim &qa, double ra, const double Gza[8],
                                          const double Ub[8], const FastPrim &qb, double rb,
                                          const double Gzb[8], double Aa[9], double Sa[10],
                                          double Ab[9], double Sb[10]) const {
        double Gra[8], Grb[8];
        fast_gr(Ua, qa, ra, Gra);
        fast_gr(Ub, qb, rb, Grb);
        const double kr = dt * rg.hdr;
        double Ba[9], Bb[9];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const double q4a = 0.25 * Ua[k], q4b = 0.25 * Ub[k];
            const double cea = (k == 7) ? q4a : fma(kr, Gra[k], q4a);
            const double cwa = (k == 7) ? q4a : fma(-kr, Gra[k], q4a);
            const double ceb = (k == 7) ? q4b : fma(kr, Grb[k], q4b);
            const double cwb = (k == 7) ? q4b : fma(-kr, Grb[k], q4b);
            // east neighbour + west neighbour, as in the one-column kernel
            Ba[k] = ceb + __shfl_up_sync(0xffffffffu, cwb, 1);
            Bb[k] = __shfl_down_sync(0xffffffffu, cea, 1) + cwa;
        }
        const double d7a = Grb[7] - __shfl_up_sync(0xffffffffu, Grb[7], 1);
        const double d7b = __shfl_down_sync(0xffffffffu, Gra[7], 1) - Gra[7];
        sources(qa, kr, d7a, Ba);
        sources(qb, kr, d7b, Bb);
        fast_sum(Aa, Ba, Sa);
        fast_a(Ua, Gza, kz, Aa);
        fast_sum(Ab, Bb, Sb);
        fast_a(Ub, Gzb, kz, Ab);
    }

    // Store the new cells of row l: one 16-byte store per plane when both
    // points write (the pair starts at an even column of a 256-byte row).
    __device__ __forceinline__ void store(int l, const double oa[8], const double ob[8]) const {
        const size_t i = g.ix(l, a.p);
#if MPD_L2_HINTS
        if (a.out && b.out) {
#pragma unroll
            for (int k = 0; k < 8; ++k)
                st_global_v2_hint(u + (size_t)k * g.ps + i, oa[k], ob[k], pol_write);
        } else if (a.out) {
#pragma unroll
            for (int k = 0; k < 8; ++k) st_global_hint(u + (size_t)k * g.ps + i, oa[k], pol_write);
        } else if (b.out) {
#pragma unroll
            for (int k = 0; k < 8; ++k)
                st_global_hint(u + (size_t)k * g.ps + i + 1, ob[k], pol_write);
        }
#else
        if (a.out && b.out) {
#pragma unroll
            for (int k = 0; k < 8; ++k)
                *reinterpret_cast<double2 *>(u + (size_t)k * g.ps + i) = make_double2(oa[k], ob[k]);
        } else if (a.out) {
#pragma unroll
            for (int k = 0; k < 8; ++k) u[(size_t)k * g.ps + i] = oa[k];
        } else if (b.out) {
#pragma unroll
            for (int k = 0; k < 8; ++k) u[(size_t)k * g.ps + i + 1] = ob[k];
        }
#endif
        if (a.out && wants_central(g.L, g.M, l, a.p)) store_central(cphys, len, g.L, g.M, l, a.p, oa);
        if (b.out && wants_central(g.L, g.M, l, b.p)) store_central(cphys, len, g.L, g.M, l, b.p, ob);
    }
};

// Close cell row l of both points with point row n = l + 1 and, unless it is
// the band's last row, fold that point row in (tma_row for two points).
template <bool WANT_WS, bool WITH_POINT>
__device__ __forceinline__ bool pair_row(const PairWarp &w, int l, uint32_t &j, double Aa[9],
                                         double Sa[10], double Ab[9], double Sb[10],
                                         double &rla, double &irla, double &rlb, double &irlb,
                                         unsigned long long &ws_key) {
    const int n = l + 1;
    const RowGeo rg = w.row_geo(n);  // issued before the wait, so the loads overlap it
    double Ua[8], Ub[8];
    if (!w.take(j, Ua, Ub)) return false;
    FastPrim qa, qb;
    double ra, rb, Gza[8], Gzb[8], oa[8], ob[8];
    w.eval(w.a, n, rg, Ua, qa, ra, Gza);
    w.eval(w.b, n, rg, Ub, qb, rb, Gzb);
    w.release(j);
    ++j;
    fast_finish(Sa, Ua, Gza, w.kz, oa);
    fast_finish(Sb, Ub, Gzb, w.kz, ob);
    w.store(l, oa, ob);
    if (WANT_WS) {
        // bits of a positive or NaN / inf speed order like its value: a
        // non-finite cell wins the maximum and the controller flags the step
        const bool row_ok = l >= 2 && l <= w.g.L - 1;
        const double wsa = fast_wave_speed(oa, rla, irla, w.g.gamma);
        const double wsb = fast_wave_speed(ob, rlb, irlb, w.g.gamma);
        const unsigned long long ka =
            (w.a.out && row_ok) ? (unsigned long long)__double_as_longlong(wsa) : 0ull;
        const unsigned long long kb =
            (w.b.out && row_ok) ? (unsigned long long)__double_as_longlong(wsb) : 0ull;
        const unsigned long long kk = ka > kb ? ka : kb;
        ws_key = kk > ws_key ? kk : ws_key;
    }
    if (WITH_POINT) w.point(rg, Ua, qa, ra, Gza, Ub, qb, rb, Gzb, Aa, Sa, Ab, Sb);
    rla = ra;
    irla = qa.ir;
    rlb = rb;
    irlb = qb.ir;
    return true;
}

// Cell rows [l_begin, l_end) of the warp's strip (tma_band_run for two points).
template <bool WANT_WS>
__device__ __forceinline__ bool pair_band_run(PairWarp &w, int l_begin, int l_end, uint32_t &j,
                                              unsigned long long &ws_key) {
    w.row0 = l_begin - 1;
    w.nrows = l_end - l_begin + 2;
    w.jbase = j;
    for (int k = 0; k < kPairStages; ++k) w.issue(j + k);
    bool ok;
    double Aa[9], Sa[10], Ab[9], Sb[10], Ua[8], Ub[8], Gza[8], Gzb[8], ra, rb;
    double rla = 1.0, irla = 1.0, rlb = 1.0, irlb = 1.0;
    FastPrim qa, qb;
    RowGeo rg = w.row_geo(l_begin - 1);
    ok = w.take(j, Ua, Ub);
    if (ok) {
        w.eval(w.a, l_begin - 1, rg, Ua, qa, ra, Gza);
        w.eval(w.b, l_begin - 1, rg, Ub, qb, rb, Gzb);
        w.release(j);
        ++j;
        fast_a(Ua, Gza, w.kz, Aa);  // A of the first cell row
        fast_a(Ub, Gzb, w.kz, Ab);
        rg = w.row_geo(l_begin);
        ok = w.take(j, Ua, Ub);
        if (ok) {
            w.eval(w.a, l_begin, rg, Ua, qa, ra, Gza);
            w.eval(w.b, l_begin, rg, Ub, qb, rb, Gzb);
            w.release(j);
            ++j;
            w.point(rg, Ua, qa, ra, Gza, Ub, qb, rb, Gzb, Aa, Sa, Ab, Sb);
            rla = ra;
            irla = qa.ir;
            rlb = rb;
            irlb = qb.ir;
        }
    }
    int l = l_begin;
    for (; ok && l < l_end - 1; ++l)
        ok = pair_row<WANT_WS, true>(w, l, j, Aa, Sa, Ab, Sb, rla, irla, rlb, irlb, ws_key);
    if (ok) ok = pair_row<WANT_WS, false>(w, l, j, Aa, Sa, Ab, Sb, rla, irla, rlb, irlb, ws_key);
    if (!ok) {
        if (w.lane == 0) {
            const uint32_t end = w.jbase + (uint32_t)w.nrows;
            for (uint32_t jj = j; jj < end && jj < j + kPairStages; ++jj)
                mbar_wait_bounded(w.bar(jj % kPairStages), (jj / kPairStages) & 1);
        }
        __syncwarp();
    }
    return ok;
}

template <bool WANT_WS>
__global__ void __launch_bounds__(32 * kPairWarps, MPD_PAIR_MINB)
    lf_pair_kernel(Geo g, const __grid_constant__ CUtensorMap map0,
                   const __grid_constant__ CUtensorMap map1, double *buf0, double *buf1,
                   DevState *st, double dt_arg, int use_state_dt, double *cphys, int len,
                   int nstrips, int nbands, int nbands_edge) {
    extern __shared__ __align__(128) unsigned char pair_smem_raw[];
    unsigned char *smem = tma_smem_base(pair_smem_raw);
    const int wib = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int task = (int)blockIdx.x * kPairWarps + wib;
    int strip, band, nb;
    tma_task(task, nstrips, nbands, nbands_edge, strip, band, nb);
    int l_begin = 1, l_end = 1;
    if (band < nb) tma_band(1, g.L, nb, band, l_begin, l_end);
    const uint32_t bar0 =
        smem_addr(smem + kPairWarps * kPairStages * kPairRowBytes) + 8u * wib * kPairStages;
    // While the previous kernel of the stream may still run: only this
    // block's shared memory and the tensor maps, which no kernel writes.
    if (l_begin < l_end && lane == 0) {
        tmap_prefetch(&map0);
        tmap_prefetch(&map1);
        for (int k = 0; k < kPairStages; ++k) mbar_init(bar0 + 8u * k, 1);
        mbar_init_fence();
    }
    pdl_wait();
    if (MPD_PDL_TRIG_INT == 1) pdl_trigger();
    if (st->done) return;
    const long long step = st->step;

    PairWarp w;
    w.g = g;
    w.u = (step & 1) ? buf0 : buf1;
    w.st = st;
    w.cphys = cphys;
    w.len = len;
    w.dt = use_state_dt ? st->dt : dt_arg;
    w.gm1 = g.gamma - 1.0;
    w.kz = w.dt * (0.5 / g.dz);
    w.x0 = kPairCells * strip;
    w.a.p = w.x0 + 2 * lane;
    w.b.p = w.a.p + 1;
    w.a.pvalid = w.a.p <= g.M + 1;
    w.b.pvalid = w.b.p <= g.M + 1;
    w.a.out = lane >= 1 && w.a.p >= 2 && w.a.p <= g.M;
    w.b.out = lane <= 30 && w.b.p >= 2 && w.b.p <= g.M;
    w.a.frac = (double)(w.a.p - 1) * g.dy;
    w.b.frac = (double)(w.b.p - 1) * g.dy;
    w.map = (step & 1) ? &map1 : &map0;
    w.lane = lane;
#if MPD_L2_HINTS
    w.pol_read = l2_policy_evict_first();
    w.pol_write = l2_policy_evict_last();
#else
    w.pol_read = w.pol_write = 0;
#endif
    w.stage = reinterpret_cast<double *>(smem) + wib * kPairStages * kPairRow;
    w.bar0 = bar0;

    unsigned long long ws_key = 0ull;
    if (l_begin < l_end) {
        __syncwarp();
        uint32_t j = 0;
        if (!pair_band_run<WANT_WS>(w, l_begin, l_end, j, ws_key) && lane == 0) {
            // a row never arrived: record the failure and stop the run
            atomicExch(&st->wait_fail, 1);
            atomicExch(&st->done, 1);
            if (st->mirror) {
                st->mirror->wait_fail = 1;
                __threadfence_system();
            }
        }
    }
    if (MPD_PDL_TRIG_INT == 2) pdl_trigger();
    if (WANT_WS) {
        unsigned long long key[1] = {ws_key};
        unsigned long long *dst[1] = {&st->ws_acc};
        block_max_atomic<1>(key, 0u, dst, &st->nf_acc);
    }
}

// Strips and bands for one wave of lf_pair_kernel on this device.
inline cudaError_t plan_lf_pair(const Geo &g, int device, TmaPlan &plan) {
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(lf_pair_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kPairSmem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(lf_pair_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kPairSmem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lf_pair_kernel<true>,
                                                      32 * kPairWarps, kPairSmem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    const int warps = sms * per_sm * kPairWarps;
    const int S = (g.M + kPairCells - 1) / kPairCells;
    plan.nstrips = S;
    const int max_nb = g.L / MPD_TMA_MIN_BAND > 1 ? g.L / MPD_TMA_MIN_BAND : 1;
    int nb, nbe;
    if (S >= 3) {
        nb = (int)((long long)warps * 100 / ((long long)(S - 2) * 100 + 2 * MPD_EDGE_WEIGHT));
        if (nb > max_nb) nb = max_nb;
        if (nb < 1) nb = 1;
        nbe = (int)((long long)nb * MPD_EDGE_WEIGHT / 100);
        if (nbe > max_nb) nbe = max_nb;
        if (nbe < nb) nbe = nb;
    } else {
        nb = warps / S;
        if (nb > max_nb) nb = max_nb;
        if (nb < 1) nb = 1;
        nbe = nb;
    }
    plan.nbands = nb;
    plan.nbands_edge = nbe;
    const int tasks = S >= 3 ? (S - 2) * nb + 2 * nbe : S * nb;
    plan.blocks = (tasks + kPairWarps - 1) / kPairWarps;
    return cudaSuccess;
}

inline cudaError_t launch_lf_pair(const Geo &g, const TmaPlan &plan, const CUtensorMap &map0,
                                  const CUtensorMap &map1, double *buf0, double *buf1,
                                  DevState *st, double dt, int use_state_dt, bool want_ws,
                                  double *cphys, int len, cudaStream_t stream) {
    if (want_ws)
        return launch_pdl(lf_pair_kernel<true>, dim3(plan.blocks), dim3(32 * kPairWarps),
                          kPairSmem, stream, g, map0, map1, buf0, buf1, st, dt, use_state_dt,
                          cphys, len, plan.nstrips, plan.nbands, plan.nbands_edge);
    return launch_pdl(lf_pair_kernel<false>, dim3(plan.blocks), dim3(32 * kPairWarps), kPairSmem,
                      stream, g, map0, map1, buf0, buf1, st, dt, use_state_dt, cphys, len,
                      plan.nstrips, plan.nbands, plan.nbands_edge);
}

}  // namespace mpd
