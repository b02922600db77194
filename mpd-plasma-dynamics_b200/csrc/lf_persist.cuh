// Persistent time loop of the plain FP64 path (MPD_PRECISION_FAST): one
// cooperative launch runs many whole time steps.
//
// The graph path launches an interior kernel and a boundary kernel per step;
// every launch starts with cold instruction and data caches, stages the
// boundary table again and waits for the previous launch to drain.  Here every
// block stays resident for the whole run and a step is
//   interior   each warp runs its (strip, band) task exactly as lf_tma_kernel,
//              folding its cells' wave speeds into a per-step maximum;
//   barrier    all interior cells and central lines of the step are written;
//   boundary   the boundary-ring cells (Solver::Advance's four faces, src/
//              solver.cpp:29-32) spread over all threads, folding their wave
//              speeds into the same maximum;
//   barrier    the step is complete;
//   controller every block computes t, dt and the stop condition from the same
//              maximum (src/main.cpp:191-282, adaptive dt after the step), so
//              all blocks agree without another exchange; block 0 records them.
// Every residual_every steps a residual pass over both buffers (one more
// barrier) evaluates the L-inf residual the graph path's residual_kernel
// computes.  Results are identical to the graph path: the same per-cell
// functions, the same maxima.
//
// The grid is one block per resident slot (cooperative launch, so every block
// is co-resident) and each barrier is a counter plus a generation word with a
// bounded wait: a barrier that does not complete within kWaitLimitNs records
// wait_fail and ends the run.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "lf_tma.cuh"

namespace mpd {

// Device-side words of the grid barrier and the per-step reductions.
struct GridSync {
    unsigned int count;              // arrivals at the current barrier
    unsigned int gen;                // barrier generation
    unsigned long long ws[2];        // max wave-speed key, by step parity
    unsigned int nf[2];              // non-finite flag, by step parity
    unsigned int rnf[2];             // residual non-finite flag, by residual parity
    unsigned long long rkey[2][16];  // residual maxima |du_k|, |u_k|, by residual parity
};

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u32(unsigned int *p, unsigned int v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// All blocks of the launch meet here.  Returns false (in every thread of the
// block) if the barrier did not complete within kWaitLimitNs.
__device__ __forceinline__ bool grid_barrier(GridSync *gs, unsigned int nblocks) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned int g0 = ld_acquire_u32(&gs->gen);
        __threadfence();
        if (atomicAdd(&gs->count, 1u) == nblocks - 1) {
            atomicExch(&gs->count, 0u);
            __threadfence();
            st_release_u32(&gs->gen, g0 + 1u);
        } else if (ld_acquire_u32(&gs->gen) == g0) {
            const unsigned long long t0 = global_ns();
            while (ld_acquire_u32(&gs->gen) == g0) {
                if (global_ns() - t0 > kWaitLimitNs) {
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Order the generic-proxy stores other blocks made before a barrier ahead of
// this thread's following TMA (async-proxy) reads of the same memory.
__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

struct PersistArgs {
    Geo g;
    double *buf0, *buf1;
    double *cphys;
    double *wall0, *wall1;
    int len;
    BcTable bc;
    DevState *st;
    GridSync *gs;
    int nstrips, nbands;
    long long nsteps;      // steps this launch may take at most
    long long resid_base;  // the residual is evaluated after steps with
                           // (step - resid_base) % resid_every == 0
};

constexpr int kPersistThreads = 32 * kTmaWarps;
constexpr int kPersistSmem = kTmaSmem + kMaxSegments * (int)sizeof(SegDesc);

// Run parameters every block reads in its controller (staged in shared memory).
struct PersistRun {
    double T, cfl, growth, dt_min, dt_max, resid_tol;
    long long max_steps;
    int adaptive, resid_every;
};

// This thread's boundary-ring cells of one step, their wave speeds folded
// into key / nf.  Out of line: the face
// logic is long and its registers must not stay live across the interior.
__device__ __noinline__ void persist_ring_phase(const PersistArgs &a, const SegDesc *s_seg,
                                                int par, double dt, unsigned long long &key,
                                                unsigned int &nf) {
    BcView v;
    v.g = a.g;
    v.u0 = par ? a.buf1 : a.buf0;
    v.u = par ? a.buf0 : a.buf1;
    v.ic = nullptr;
    v.cphys = a.cphys;
    v.wphys = par ? a.wall1 : a.wall0;
    v.len = a.len;
    v.first = 0;
    v.fast = 1;
    v.dt = dt;
    v.bc = a.bc;
    v.bc.seg = s_seg;
    double *wnext = par ? a.wall0 : a.wall1;
    CellStats cs;
    cs.init();
    // chunks of 32 consecutive ring cells (one face, mostly) per warp, chunk c
    // on block c % nblocks, so the lanes of a warp take the same face code
    const int nring = ring_count(a.g);
    const int nwarps = (int)(blockDim.x >> 5);
    const int lane = threadIdx.x & 31;
    const int chunk0 = (int)((threadIdx.x >> 5) * gridDim.x + blockIdx.x);
    for (int c = chunk0; c * 32 < nring; c += (int)gridDim.x * nwarps) {
        const int i = c * 32 + lane;
        if (i < nring) ring_cell_update(v, i, wnext, true, cs);
    }
    key = cs.key[0];
    nf = cs.nf;
}

// This thread's share of the residual maxima max |u_new - u_old|, max |u_old|
// per conserved field over the interior cells (residual_kernel's pass).
__device__ __noinline__ void persist_resid_phase(const PersistArgs &a, int par,
                                                 unsigned long long key[16], unsigned int &nf) {
    const Geo &g = a.g;
    const double *un = par ? a.buf0 : a.buf1;  // written by the step that just ended
    const double *uo = par ? a.buf1 : a.buf0;
#pragma unroll
    for (int k = 0; k < 16; ++k) key[k] = 0ull;
    nf = 0u;
    const int W = g.M + 1;
    const int total = g.L * W;
    for (int c = (int)(blockIdx.x * blockDim.x + threadIdx.x); c < total;
         c += (int)(gridDim.x * blockDim.x)) {
        const size_t i = g.ix(1 + c / W, 1 + c % W);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const double an = __ldcg(un + (size_t)k * g.ps + i);
            const double ao = __ldcg(uo + (size_t)k * g.ps + i);
            const unsigned long long d = max_key(fabs(an - ao), nf);
            const unsigned long long o = max_key(fabs(ao), nf);
            key[k] = d > key[k] ? d : key[k];
            key[8 + k] = o > key[8 + k] ? o : key[8 + k];
        }
    }
}

__global__ void __launch_bounds__(kPersistThreads, MPD_TMA_MINB)
    lf_persist_kernel(const __grid_constant__ CUtensorMap map0,
                      const __grid_constant__ CUtensorMap map1,
                      const __grid_constant__ PersistArgs a) {
    extern __shared__ __align__(128) unsigned char tma_smem_raw[];
    unsigned char *tma_smem = tma_smem_base(tma_smem_raw);
    SegDesc *s_seg = reinterpret_cast<SegDesc *>(tma_smem + kTmaSmem - 128);
    __shared__ PersistRun run;
    DevState *st = a.st;
    GridSync *gs = a.gs;
    const unsigned int nblocks = gridDim.x;
    const int wib = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;

    // the step state and run parameters, read once: every block sees the same
    long long step = st->step;
    double t = st->t, dt = st->dt;
    int done = st->done;
    if (threadIdx.x == 0) {
        run.T = st->T;
        run.cfl = st->cfl;
        run.growth = st->growth;
        run.dt_min = st->dt_min;
        run.dt_max = st->dt_max;
        run.resid_tol = st->resid_tol;
        run.max_steps = st->max_steps;
        run.adaptive = st->adaptive;
        run.resid_every = st->resid_every;
    }
    // boundary table, staged once for the whole launch
    {
        const int nwords = a.bc.nseg_total * (int)(sizeof(SegDesc) / sizeof(int));
        const int *src = reinterpret_cast<const int *>(a.bc.seg);
        int *dst = reinterpret_cast<int *>(s_seg);
        for (int w = threadIdx.x; w < nwords; w += blockDim.x) dst[w] = src[w];
    }

    // interior task of this warp
    const int task = (int)blockIdx.x * kTmaWarps + wib;
    const int strip = task % a.nstrips;
    const int band = task / a.nstrips;
    int l_begin = 1, l_end = 1;
    if (band < a.nbands) tma_band(a.g.L, a.nbands, band, l_begin, l_end);
    TmaWarp w;
    w.stage = reinterpret_cast<double *>(tma_smem) + wib * kTmaStages * kTmaRow;
    w.bar0 = smem_addr(tma_smem + kTmaWarps * kTmaStages * kTmaRowBytes) + 8u * wib * kTmaStages;
    tma_warp_setup(w, a.g, strip, a.buf1, st, a.cphys, a.len, dt, &map0);
    if (l_begin < l_end) w.init();
    uint32_t jrow = 0;  // running staged-row count of this warp
    long long nresid = 0;
    bool ok = __syncthreads_and(1);

    for (long long it = 0; ok && !done && it < a.nsteps; ++it) {
        const int par = (int)(step & 1);

        // ---- interior -----------------------------------------------------
        unsigned long long ws_key = 0ull;
        unsigned int nf = 0u;
        if (l_begin < l_end) {
            tma_warp_setup(w, a.g, strip, par ? a.buf0 : a.buf1, st, a.cphys, a.len, dt,
                           par ? &map1 : &map0);
            if (lane == 0) fence_proxy_async_global();
            __syncwarp();
            if (!tma_band_run<true>(w, l_begin, l_end, jrow, ws_key, nf)) ok = false;
        }
        {
            unsigned long long key[1] = {ws_key};
            unsigned long long *dst[1] = {&gs->ws[par]};
            block_max_atomic<1>(key, nf, dst, &gs->nf[par]);
        }
        ok = __syncthreads_and(ok) && grid_barrier(gs, nblocks);
        if (!ok) break;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            gs->ws[par ^ 1] = 0ull;  // next step's slot: last read before this barrier
            gs->nf[par ^ 1] = 0u;
        }

        // ---- boundary ring ---------------------------------------------------
        {
            unsigned long long key[1];
            unsigned int rnf;
            persist_ring_phase(a, s_seg, par, dt, key[0], rnf);
            unsigned long long *dst[1] = {&gs->ws[par]};
            block_max_atomic<1>(key, rnf, dst, &gs->nf[par]);
        }
        ok = grid_barrier(gs, nblocks);
        if (!ok) break;

        // ---- controller (identical in every block) --------------------------
        const double ws = __longlong_as_double((long long)__ldcg(&gs->ws[par]));
        int nonfinite = (__ldcg(&gs->nf[par]) || !isfinite(ws)) ? 1 : 0;
        const double dt_used = dt;
        t = t + dt;
        step = step + 1;
        double dtn = dt;
        if (run.adaptive)
            dtn = compute_dt_from_speed(ws, a.g.dz, a.g.dy, run.cfl, run.growth, run.dt_min,
                                        run.dt_max, dt);
        done = (nonfinite || !(t < run.T) || step >= run.max_steps) ? 1 : 0;
        if (t + dtn > run.T) dtn = run.T - t;
        dt = dtn;

        // ---- residual every resid_every steps (after the step, both buffers) --
        int converged = 0, resid_now = 0;
        double R = 0.0;
        if (run.resid_every > 0 && (step - a.resid_base) % run.resid_every == 0) {
            resid_now = 1;
            const int rp = (int)(nresid & 1);
            unsigned long long key[16];
            unsigned int rnf;
            persist_resid_phase(a, par, key, rnf);
            unsigned long long *dst[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) dst[k] = &gs->rkey[rp][k];
            block_max_atomic<16>(key, rnf, dst, &gs->rnf[rp]);
            ok = grid_barrier(gs, nblocks);
            if (!ok) break;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const double num = __longlong_as_double((long long)__ldcg(&gs->rkey[rp][k]));
                const double den = __longlong_as_double((long long)__ldcg(&gs->rkey[rp][8 + k]));
                const double rk = num / (den > 1e-300 ? den : 1e-300);
                R = rk > R ? rk : R;
            }
            if (__ldcg(&gs->rnf[rp]) || !isfinite(R)) {
                nonfinite = 1;
                done = 1;
            }
            if (run.resid_tol > 0.0 && R <= run.resid_tol) {
                converged = 1;
                done = 1;
            }
            if (blockIdx.x == 0 && threadIdx.x == 0) {
#pragma unroll
                for (int k = 0; k < 16; ++k) gs->rkey[rp ^ 1][k] = 0ull;
                gs->rnf[rp ^ 1] = 0u;
            }
            ++nresid;
        }

        if (blockIdx.x == 0 && threadIdx.x == 0) {
            st->t = t;
            st->step = step;
            st->dt = dt;
            st->dt_used = dt_used;
            st->last_ws = ws;
            st->ws_valid = 1;
            st->nonfinite = nonfinite;
            st->done = done;
            if (resid_now) {
                st->last_resid = R;
                st->resid_valid = 1;
                st->resid_step = step;
                if (converged) st->converged = 1;
            } else {
                st->resid_valid = 0;
            }
        }
    }
    if (!ok && threadIdx.x == 0) {
        atomicExch(&st->wait_fail, 1);
        atomicExch(&st->done, 1);
    }
}

// Blocks of one cooperative wave of lf_persist_kernel and its interior plan.
inline cudaError_t plan_lf_persist(const Geo &g, int device, TmaPlan &plan) {
    int sms = 0, per_sm = 0, coop = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
    if (e != cudaSuccess) return e;
    if (!coop) return cudaErrorNotSupported;
    e = cudaFuncSetAttribute(lf_persist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kPersistSmem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lf_persist_kernel, kPersistThreads,
                                                      kPersistSmem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorNotSupported;
    plan.blocks = sms * per_sm;
    const int warps = plan.blocks * kTmaWarps;
    plan.nstrips = (g.M + kFastCells - 1) / kFastCells;
    int nb = warps / plan.nstrips;
    const int min_band = 4;
    if (nb > g.L / min_band) nb = g.L / min_band;
    if (nb < 1) nb = 1;
    if (plan.nstrips * nb > warps) return cudaErrorNotSupported;  // more strips than warps
    plan.nbands = nb;
    return cudaSuccess;
}

inline cudaError_t launch_lf_persist(const TmaPlan &plan, const CUtensorMap &map0,
                                     const CUtensorMap &map1, const PersistArgs &a,
                                     cudaStream_t stream) {
    void *args[] = {const_cast<CUtensorMap *>(&map0), const_cast<CUtensorMap *>(&map1),
                    const_cast<PersistArgs *>(&a)};
    return cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(lf_persist_kernel),
                                       dim3(plan.blocks), dim3(kPersistThreads), args,
                                       kPersistSmem, stream);
}

}  // namespace mpd
