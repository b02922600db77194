// TMA-staged interior kernel of the plain FP64 path (MPD_PRECISION_FAST).
//
// The arithmetic is lf_fast.cuh's (FastStrip::eval / point, fast_finish), so
// the result is bit-identical to it; what changes is how the rows arrive and
// how the work is spread:
//   * a warp owns a strip of 32 point columns starting at an even column
//     x0 = 30 s (30 output cells, lanes 0 and 31 are halo points) and a band
//     of rows; the rows it needs are fetched by one TMA tile load each
//     ({32 columns} x {1 row} x {8 conserved planes} = 2 KB) into a ring of
//     kTmaStages shared-memory stages, kTmaStages - 1 rows ahead of use, so a
//     warp keeps several rows in flight without holding them in registers;
//   * the launch is one wave: bands are sized so that strips x bands equals
//     the number of warps the GPU holds at once, instead of a fixed band
//     height that leaves a partial second wave.
// Rows outside the planes (l = -1, l = L+2) and columns past M+2 arrive as
// zeros (TMA out-of-bounds fill); ghost rows and columns are zero in memory.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "lf_fast.cuh"
#include "tma.cuh"

namespace mpd {

// Build-time tuning: resident blocks per SM the register budget is cut for,
// staged rows per warp, warps per block and the fewest rows a band gets.
// A small grid has more warps than (strip, row) pairs: one-row bands then
// give the shortest chain per warp (measured on a B200: 100 x 40 step
// 18.2 -> 15.4 us, 400 x 160 18.1 -> 16.7 us; large grids unaffected).
#ifndef MPD_TMA_MINB
#define MPD_TMA_MINB 3
#endif
#ifndef MPD_TMA_STAGES
#define MPD_TMA_STAGES 4
#endif
#ifndef MPD_TMA_WARPS
#define MPD_TMA_WARPS 4
#endif
#ifndef MPD_TMA_MIN_BAND
#define MPD_TMA_MIN_BAND 1
#endif
// L2 eviction priorities on the interior's traffic: the rows a step reads are
// never read again (the buffer is next overwritten), the cells it writes are
// the next step's input.
#ifndef MPD_L2_HINTS
#define MPD_L2_HINTS 1
#endif

constexpr int kTmaWarps = MPD_TMA_WARPS;      // warps per block
constexpr int kTmaStages = MPD_TMA_STAGES;    // rows in flight per warp
constexpr int kTmaRow = 8 * 32;               // doubles per staged row
constexpr int kTmaRowBytes = kTmaRow * 8;     // 2048
// + 128 bytes to align the stages: TMA destinations need 128-byte alignment
constexpr int kTmaSmem = kTmaWarps * kTmaStages * (kTmaRowBytes + 8) + 128;

// Rows [l_begin, l_end) of band b out of nbands over the rows first ..
// first + count - 1 (1..L, or 2..L-1 when the boundary ring runs beside the
// interior and computes rows 1 and L itself).
__host__ __device__ inline void tma_band(int first, int count, int nbands, int b, int &l_begin,
                                         int &l_end) {
    l_begin = first + (int)((long long)b * count / nbands);
    l_end = first + (int)((long long)(b + 1) * count / nbands);
}

// The first and last strips cost more per row than the others (a per-warp
// timestamp probe on a B200 at 1600 x 640: 24.1 us per 20-row band against
// 21.5 us; they store a central column every row).  Their tasks come first,
// four consecutive bands of one edge strip per block, then the middle
// strips band by band: that order measured 37.7 us per step against 39.2 us
// for every strip band by band.  MPD_EDGE_WEIGHT gives the edge strips that
// percentage of a middle strip's band count; more, shorter edge bands (112,
// 120) measured no better, so it stays 100.
#ifndef MPD_EDGE_WEIGHT
#define MPD_EDGE_WEIGHT 100
#endif

// Task -> (strip, band, bands of that strip): with three or more strips the
// first nbands_edge tasks are the first strip's bands, the next nbands_edge
// the last strip's, the rest the middle strips' (nbands each); otherwise
// every strip has nbands bands.
__host__ __device__ inline void tma_task(int task, int nstrips, int nbands, int nbands_edge,
                                         int &strip, int &band, int &nb) {
    if (nstrips >= 3) {
        if (task < 2 * nbands_edge) {
            strip = task < nbands_edge ? 0 : nstrips - 1;
            band = task < nbands_edge ? task : task - nbands_edge;
            nb = nbands_edge;
            return;
        }
        const int u = task - 2 * nbands_edge;
        strip = 1 + u % (nstrips - 2);
        band = u / (nstrips - 2);
        nb = nbands;
        return;
    }
    strip = task % nstrips;
    band = task / nstrips;
    nb = nbands;
}

struct TmaWarp {
    FastStrip f;
    uint64_t pol_read, pol_write;  // L2 policies of the loads and stores
    const CUtensorMap *map;
    double *stage;   // kTmaStages rows of [8][32]
    uint32_t bar0;   // shared address of this warp's first barrier
    uint32_t jbase;  // running row count at the band's first staged row
    int row0;        // plane row of the band's first staged row
    int nrows;       // rows the band stages
    int lane;

    __device__ __forceinline__ uint32_t bar(uint32_t s) const { return bar0 + 8u * s; }

    // Barriers of this warp's stages; once per launch, before the first issue.
    __device__ __forceinline__ void init() const {
        if (lane == 0) {
            tmap_prefetch(map);
            for (int k = 0; k < kTmaStages; ++k) mbar_init(bar(k), 1);
            mbar_init_fence();
        }
        __syncwarp();
    }

    // Staged row j (running count) of the band: one TMA tile load into stage j % kTmaStages.
    __device__ __forceinline__ void issue(uint32_t j) const {
        if (lane == 0 && j - jbase < (uint32_t)nrows) {
            const uint32_t s = j % kTmaStages;
            mbar_expect_tx(bar(s), kTmaRowBytes);
#if MPD_L2_HINTS
            tma_load_3d_hint(smem_addr(stage + s * kTmaRow), map, bar(s), f.p - lane,
                             row0 + (int)(j - jbase), 0, pol_read);
#else
            tma_load_3d(smem_addr(stage + s * kTmaRow), map, bar(s), f.p - lane,
                        row0 + (int)(j - jbase), 0);
#endif
        }
    }

    // Staged row j into U; false if the wait gave up.  Columns past M+1 hold
    // the zero ghost column M+2 or the tile's zero fill; their lanes write no
    // cell and feed no output lane's sums either way.
    __device__ __forceinline__ bool take(uint32_t j, double U[8]) const {
        const uint32_t s = j % kTmaStages;
        const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(bar(s), (j / kTmaStages) & 1));
        const double *src = stage + s * kTmaRow + lane;
#pragma unroll
        for (int k = 0; k < 8; ++k) U[k] = src[32 * k];
        return ok;
    }

    // Row j's values are in registers and used: refill its stage with row j + kTmaStages.
    __device__ __forceinline__ void release(uint32_t j) const {
        __syncwarp();
        issue(j + kTmaStages);
    }
};

// Close cell row l (sums S) with point row n = l + 1 and, unless it is the
// band's last row (WITH_POINT false), fold that point row in: S and A move on
// to row n.  r_l / ir_l: radius of row l and its reciprocal (from the
// evaluation of point row l), replaced by row n's.
//
// After the stores the new cells' wave speed and point row n's shares are two
// independent dependency chains in one branch-free stretch of code, so the
// compiler interleaves them: every lane evaluates the wave speed (halo and
// ghost lanes too, on whatever their values give) and only output lanes of
// rows 2..L-1 feed it to the maximum.
template <bool WANT_WS, bool WITH_POINT, bool CENTRAL>
__device__ __forceinline__ bool tma_row(const TmaWarp &w, int l, uint32_t &j, double A[9],
                                        double S[10], double &r_l, double &ir_l,
                                        unsigned long long &ws_key, unsigned int &nf) {
    const FastStrip &s = w.f;
    const Geo &g = s.g;
    const int n = l + 1;
    const RowGeo rg = s.row_geo(n);  // issued before the wait, so the loads overlap it
    double Un[8];
    if (!w.take(j, Un)) return false;
    FastPrim q;
    double r, Gz[8], out[8];
    s.eval(n, rg, Un, q, r, Gz);
    w.release(j);
    ++j;
    fast_finish(S, Un, Gz, s.kz, out);
    if (s.out_lane) {
        const size_t i = g.ix(l, s.p);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
#if MPD_L2_HINTS
            st_global_hint(s.u + (size_t)k * g.ps + i, out[k], w.pol_write);
#else
            s.u[(size_t)k * g.ps + i] = out[k];
#endif
        }
        if (CENTRAL && wants_central(g.L, g.M, l, s.p))
            store_central(s.cphys, s.len, g.L, g.M, l, s.p, out);
    }
    if (WANT_WS) {
        // The wave speed is positive or NaN / inf, so its bits order like its
        // value with NaN and inf above every finite speed: a non-finite cell
        // wins the maximum and the controller flags the step.
        const double wsp = fast_wave_speed(out, r_l, ir_l, g.gamma);
        const bool ws_lane = s.out_lane && l >= 2 && l <= g.L - 1;
        const unsigned long long kk = ws_lane ? (unsigned long long)__double_as_longlong(wsp) : 0ull;
        ws_key = kk > ws_key ? kk : ws_key;
    }
    if (WITH_POINT) s.point(rg, Un, q, r, Gz, A, S);
    r_l = r;
    ir_l = q.ir;
    return true;
}

// Cell rows [l_begin, l_end) of the warp's strip.  j is the running staged-row
// count (advanced by the l_end - l_begin + 2 rows the band consumes).  Returns
// false if a row never arrived; the copies still in flight have then been
// waited for (bounded).
template <bool WANT_WS, bool CENTRAL>
__device__ __forceinline__ bool tma_band_run(TmaWarp &w, int l_begin, int l_end, uint32_t &j,
                                             unsigned long long &ws_key, unsigned int &nf) {
    const FastStrip &s = w.f;
    w.row0 = l_begin - 1;
    w.nrows = l_end - l_begin + 2;
    w.jbase = j;
    for (int k = 0; k < kTmaStages; ++k) w.issue(j + k);
    bool ok;
    double A[9], S[10], U[8], Gz[8], r, r_l = 1.0, ir_l = 1.0;
    FastPrim q;
    RowGeo rg = s.row_geo(l_begin - 1);
    ok = w.take(j, U);
    if (ok) {
        s.eval(l_begin - 1, rg, U, q, r, Gz);
        w.release(j);
        ++j;
        fast_a(U, Gz, s.kz, A);  // A of the first cell row
        rg = s.row_geo(l_begin);
        ok = w.take(j, U);
        if (ok) {
            s.eval(l_begin, rg, U, q, r, Gz);
            w.release(j);
            ++j;
            s.point(rg, U, q, r, Gz, A, S);  // S of the first cell row, A of the next
            r_l = r;
            ir_l = q.ir;
        }
    }
    int l = l_begin;
    for (; ok && l < l_end - 1; ++l)
        ok = tma_row<WANT_WS, true, CENTRAL>(w, l, j, A, S, r_l, ir_l, ws_key, nf);
    if (ok) ok = tma_row<WANT_WS, false, CENTRAL>(w, l, j, A, S, r_l, ir_l, ws_key, nf);
    if (!ok) {
        if (w.lane == 0) {
            const uint32_t end = w.jbase + (uint32_t)w.nrows;
            for (uint32_t jj = j; jj < end && jj < j + kTmaStages; ++jj)
                mbar_wait_bounded(w.bar(jj % kTmaStages), (jj / kTmaStages) & 1);
        }
        __syncwarp();
    }
    return ok;
}

// Strip, lanes and per-step constants of warp `task`'s FastStrip.
__device__ __forceinline__ void tma_warp_setup(TmaWarp &w, const Geo &g, int strip, double *u,
                                               DevState *st, double *cphys, int len, double dt,
                                               const CUtensorMap *map) {
    FastStrip &s = w.f;
    const int lane = threadIdx.x & 31;
    s.g = g;
    s.u = u;
    s.st = st;
    s.cphys = cphys;
    s.len = len;
    s.dt = dt;
    s.p = kFastCells * strip + lane;
    s.pvalid = s.p <= g.M + 1;
    s.out_lane = lane >= 1 && lane <= kFastCells && s.p >= 2 && s.p <= g.M;
    s.frac = (double)(s.p - 1) * g.dy;
    s.gm1 = g.gamma - 1.0;
    s.kz = dt * (0.5 / g.dz);
    w.map = map;
    w.lane = lane;
#if MPD_L2_HINTS
    w.pol_read = l2_policy_evict_first();
    w.pol_write = l2_policy_evict_last();
#else
    w.pol_read = w.pol_write = 0;
#endif
}

__device__ __forceinline__ unsigned char *tma_smem_base(unsigned char *raw) {
    return raw + ((128u - (smem_addr(raw) & 127u)) & 127u);
}

// RING_BESIDE: the boundary ring of this step runs in bc_overlap_kernel,
// launched right after this kernel and running beside it: cell rows 2..L-1
// only (the ring kernel computes rows 1 and L) and no central lines.
// early_trigger: the next kernel of the stream is let in as soon as this one
// has read the step's state (the ring kernel, which must start at once);
// otherwise once a block's rows are done.  Back-to-back launches of this
// kernel alone take the latter: a next interior placed block by block as
// this one's blocks retire would crowd its edge-strip blocks onto the SMs
// that free first.
template <bool WANT_WS, bool RING_BESIDE>
__global__ void __launch_bounds__(32 * kTmaWarps, MPD_TMA_MINB)
    lf_tma_kernel(Geo g, const __grid_constant__ CUtensorMap map0,
                  const __grid_constant__ CUtensorMap map1, double *buf0, double *buf1,
                  DevState *st, double dt_arg, int use_state_dt, double *cphys, int len,
                  int nstrips, int nbands, int nbands_edge, int early_trigger) {
    extern __shared__ __align__(128) unsigned char tma_smem_raw[];
    unsigned char *tma_smem = tma_smem_base(tma_smem_raw);
    const int wib = threadIdx.x >> 5;
    const int task = (int)blockIdx.x * kTmaWarps + wib;
    int strip, band, nb;
    tma_task(task, nstrips, nbands, nbands_edge, strip, band, nb);
    int l_begin = 1, l_end = 1;
    if (band < nb) {
        if (RING_BESIDE)
            tma_band(2, g.L - 2, nb, band, l_begin, l_end);
        else
            tma_band(1, g.L, nb, band, l_begin, l_end);
    }
    const uint32_t bar0 =
        smem_addr(tma_smem + kTmaWarps * kTmaStages * kTmaRowBytes) + 8u * wib * kTmaStages;
    // While the previous kernel of the stream may still run: only this
    // block's shared memory and the tensor maps, which no kernel writes.
    if (l_begin < l_end && (threadIdx.x & 31) == 0) {
        tmap_prefetch(&map0);
        tmap_prefetch(&map1);
        for (int k = 0; k < kTmaStages; ++k) mbar_init(bar0 + 8u * k, 1);
        mbar_init_fence();
    }
    pdl_wait();
    if (early_trigger) pdl_trigger();
    // the step's state in one memory round trip: all three loads issue
    // before the branch
    const int done = st->done;
    const long long step = st->step;
    const double st_dt = st->dt;
    if (done) return;

    TmaWarp w;
    tma_warp_setup(w, g, strip, (step & 1) ? buf0 : buf1, st, cphys, len,
                   use_state_dt ? st_dt : dt_arg, (step & 1) ? &map1 : &map0);
    w.stage = reinterpret_cast<double *>(tma_smem) + wib * kTmaStages * kTmaRow;
    w.bar0 = bar0;

    unsigned long long ws_key = 0ull;
    unsigned int nf = 0u;
    if (l_begin < l_end) {
        __syncwarp();
        uint32_t j = 0;
        if (!tma_band_run<WANT_WS, !RING_BESIDE>(w, l_begin, l_end, j, ws_key, nf) &&
            w.lane == 0) {
            // a row never arrived: record the failure and stop the run
            atomicExch(&st->wait_fail, 1);
            atomicExch(&st->done, 1);
            if (st->mirror) {
                st->mirror->wait_fail = 1;
                __threadfence_system();
            }
        }
    }
    if (!early_trigger) pdl_trigger();
    if (WANT_WS) {
        unsigned long long key[1] = {ws_key};
        unsigned long long *dst[1] = {&st->ws_acc};
        block_max_atomic<1>(key, nf, dst, &st->nf_acc);
    }
}

// Strips and bands for one wave of lf_tma_kernel on this device.
struct TmaPlan {
    int nstrips = 0, nbands = 0, nbands_edge = 0, blocks = 0;
};

inline cudaError_t plan_lf_tma(const Geo &g, int device, TmaPlan &plan) {
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    void (*const kernels[4])(Geo, const CUtensorMap, const CUtensorMap, double *, double *,
                             DevState *, double, int, double *, int, int, int, int, int) = {
        lf_tma_kernel<true, false>, lf_tma_kernel<false, false>, lf_tma_kernel<true, true>,
        lf_tma_kernel<false, true>};
    for (auto k : kernels) {
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kTmaSmem);
        if (e != cudaSuccess) return e;
    }
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lf_tma_kernel<true, false>,
                                                      32 * kTmaWarps, kTmaSmem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    const int warps = sms * per_sm * kTmaWarps;
    const int S = (g.M + kFastCells - 1) / kFastCells;
    plan.nstrips = S;
    const int max_nb = g.L / MPD_TMA_MIN_BAND > 1 ? g.L / MPD_TMA_MIN_BAND : 1;
    int nb, nbe;
    if (S >= 3) {
        // (S - 2) nb + 2 nbe <= warps with nbe = nb * weight
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
    plan.blocks = (tasks + kTmaWarps - 1) / kTmaWarps;
    return cudaSuccess;
}

inline cudaError_t launch_lf_tma(const Geo &g, const TmaPlan &plan, const CUtensorMap &map0,
                                 const CUtensorMap &map1, double *buf0, double *buf1,
                                 DevState *st, double dt, int use_state_dt, bool want_ws,
                                 bool ring_beside, bool early_trigger, double *cphys, int len,
                                 cudaStream_t stream) {
    auto kernel = want_ws ? (ring_beside ? lf_tma_kernel<true, true> : lf_tma_kernel<true, false>)
                          : (ring_beside ? lf_tma_kernel<false, true> : lf_tma_kernel<false, false>);
    return launch_pdl(kernel, dim3(plan.blocks), dim3(32 * kTmaWarps), kTmaSmem, stream, g, map0,
                      map1, buf0, buf1, st, dt, use_state_dt, cphys, len, plan.nstrips,
                      plan.nbands, plan.nbands_edge, early_trigger ? 1 : 0);
}

}  // namespace mpd
