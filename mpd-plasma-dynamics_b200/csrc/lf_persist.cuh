// Persistent time loops of the plain FP64 path (MPD_PRECISION_FAST): one
// cooperative launch runs many whole time steps, of one solve or of a batch.
//
// The graph path launches an interior kernel and a boundary kernel per step.
// Here blocks stay resident and are grouped into teams; a team runs one
// solve at a time and a step is
//   interior   each warp of the team runs (strip, band) tasks exactly as
//              lf_tma_kernel, folding its cells' wave speeds into a per-step
//              maximum;
//   barrier    all interior cells and central lines of the step are written;
//   boundary   the boundary-ring cells (Solver::Advance's four faces, src/
//              solver.cpp:29-32), 32 consecutive cells per warp, folding their
//              wave speeds into the same maximum;
//   barrier    the step is complete;
//   controller every block of the team computes t, dt and the stop condition
//              from the same maximum (src/main.cpp:191-282, adaptive dt after
//              the step), so the team agrees without another exchange; the
//              team's first block records them in the solve's DevState.
// Every residual_every steps a residual pass over both buffers (one more
// barrier) evaluates the L-inf residual of residual_kernel.  Results are the
// graph path's bits: the same per-cell functions, the same maxima.
//
// lf_persist_kernel: one team = the whole grid, one solve (mpd_run with
// MPD_ENGINE_PERSISTENT).  lf_batch_kernel: many teams, each with its own
// queue of solves (mpd_batch_run).  A team barrier is a counter plus a
// generation word with a bounded wait (a one-block team uses __syncthreads):
// a barrier that does not complete within kWaitLimitNs records wait_fail in
// the solve's DevState and ends the team's work.  The launch is cooperative,
// so every block of every team is resident.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "lf_tma.cuh"

namespace mpd {

// Device-side words of a team barrier and the per-step reductions.
struct GridSync {
    unsigned int count;              // arrivals at the current barrier
    unsigned int gen;                // barrier generation
    unsigned long long ws[2];        // max wave-speed key, by step parity
    unsigned int nf[2];              // non-finite flag, by step parity
    unsigned int rnf[2];             // residual non-finite flag, by residual parity
    unsigned long long rkey[2][16];  // residual maxima |du_k|, |u_k|, by residual parity
    unsigned int pad[28];            // keeps teams' words on separate 128-byte lines
};

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u32(unsigned int *p, unsigned int v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Blocks of one team and their barrier words.
struct TeamCtx {
    int rank;      // this block within the team
    int size;      // blocks in the team
    GridSync *gs;
};

// All blocks of the team meet here.  Returns false (in every thread of the
// block) if the barrier did not complete within kWaitLimitNs.
__device__ __forceinline__ bool team_barrier(const TeamCtx &tm) {
    if (tm.size == 1) {
        __syncthreads();
        return true;
    }
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        GridSync *gs = tm.gs;
        int ok = 1;
        const unsigned int g0 = ld_acquire_u32(&gs->gen);
        // release of the block's writes (cumulative over the barrier above);
        // the last arrival acquires every earlier one through the chain of
        // read-modify-writes, and its release of gen passes them all on
        if (atom_add_acq_rel_u32(&gs->count, 1u) == (unsigned int)tm.size - 1) {
            atomicExch(&gs->count, 0u);
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

// One solve as the persistent loops see it.
struct PersistArgs {
    Geo g;
    double *buf0, *buf1;
    double *cphys;
    double *wall0, *wall1;
    int len;
    BcTable bc;
    DevState *st;
    int nstrips, nbands;   // interior tasks: strips x bands
    long long nsteps;      // steps this launch may take at most
    long long resid_base;  // the residual is evaluated after steps with
                           // (step - resid_base) % resid_every == 0
};

// Run parameters every block reads in its controller (staged in shared memory).
struct PersistRun {
    double T, cfl, growth, dt_min, dt_max, resid_tol;
    long long max_steps;
    int adaptive, resid_every;
};

// Resident blocks per SM the persistent kernels' register budget is cut for.
// Two (255 registers, the ring code nearly spill-free) shortens a team's step
// by a quarter (B200: 100 x 40 on one block 85 -> 66 us, 400 x 160 on four
// 239 -> 178 us) but a wave then holds 296 blocks instead of 444, and the
// batched sweep measured 7.47 against 8.09 solves/s; three stays.
#ifndef MPD_PERSIST_MINB
#define MPD_PERSIST_MINB MPD_TMA_MINB
#endif
constexpr int kPersistThreads = 32 * kTmaWarps;
constexpr int kPersistSmem = kTmaSmem + kMaxSegments * (int)sizeof(SegDesc);

// This thread's boundary-ring cells of one step, their wave speeds folded
// into key / nf.  Out of line: the face logic is long and its registers must
// not stay live across the interior.
__device__ __noinline__ void persist_ring_phase(const PersistArgs &a, const SegDesc *s_seg,
                                                int par, double dt, int rank, int size,
                                                unsigned long long &key, unsigned int &nf) {
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
    // on block c % size, so the lanes of a warp take the same face code
    const int nring = ring_count(a.g);
    const int nwarps = (int)(blockDim.x >> 5);
    const int lane = threadIdx.x & 31;
    for (int c = (int)(threadIdx.x >> 5) * size + rank; c * 32 < nring; c += size * nwarps) {
        const int i = c * 32 + lane;
        if (i < nring) ring_cell_update(v, i, wnext, true, cs);
    }
    key = cs.key[0];
    nf = cs.nf;
}

// This thread's share of the residual maxima max |u_new - u_old|, max |u_old|
// per conserved field over the interior cells (residual_kernel's pass).
__device__ __noinline__ void persist_resid_phase(const PersistArgs &a, int par, int rank,
                                                 int size, unsigned long long key[16],
                                                 unsigned int &nf) {
    const Geo &g = a.g;
    const double *un = par ? a.buf0 : a.buf1;  // written by the step that just ended
    const double *uo = par ? a.buf1 : a.buf0;
    ResidAcc acc;
    acc.init();
    const int W = g.M + 1;
    const int total = g.L * W;
    for (int c = rank * (int)blockDim.x + (int)threadIdx.x; c < total;
         c += size * (int)blockDim.x) {
        const size_t i = g.ix(1 + c / W, 1 + c % W);
        double an[8], ao[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            an[k] = __ldcg(un + (size_t)k * g.ps + i);
            ao[k] = __ldcg(uo + (size_t)k * g.ps + i);
        }
        acc.fold(an, ao);
    }
    unsigned long long k16[16];
    acc.keys(k16, nf);
#pragma unroll
    for (int k = 0; k < 16; ++k) key[k] = k16[k];
}

// Per-block working memory of the persistent loops.
struct PersistBlock {
    unsigned char *tma;   // 128-byte aligned TMA stages and barriers
    SegDesc *seg;         // staged boundary table
    PersistRun *run;
};

// Run solve `a` with team `tm` until it is done or a.nsteps steps have been
// taken.  w / jrow: this warp's TMA ring and running staged-row count (they
// carry over between solves).  Returns false after a barrier or TMA wait gave
// up (wait_fail recorded).
__device__ __forceinline__ bool persist_solve(const PersistArgs &a, const CUtensorMap *map0,
                                              const CUtensorMap *map1, const TeamCtx &tm,
                                              const PersistBlock &pb, TmaWarp &w,
                                              uint32_t &jrow) {
    DevState *st = a.st;
    GridSync *gs = tm.gs;
    PersistRun &run = *pb.run;
    const int wib = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;

    // the step state and run parameters of the solve: every block sees the same
    __syncthreads();
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
    {
        const int nwords = a.bc.nseg_total * (int)(sizeof(SegDesc) / sizeof(int));
        const int *src = reinterpret_cast<const int *>(a.bc.seg);
        int *dst = reinterpret_cast<int *>(pb.seg);
        for (int k = threadIdx.x; k < nwords; k += blockDim.x) dst[k] = src[k];
    }
    // the team's reduction slots start clean for this solve
    if (tm.rank == 0 && threadIdx.x == 0) {
        if (st->t0_ns == 0ull) st->t0_ns = global_ns();
        gs->ws[0] = gs->ws[1] = 0ull;
        gs->nf[0] = gs->nf[1] = 0u;
        gs->rnf[0] = gs->rnf[1] = 0u;
        for (int k = 0; k < 16; ++k) gs->rkey[0][k] = gs->rkey[1][k] = 0ull;
    }
    bool ok = team_barrier(tm);

    const int team_warps = tm.size * kTmaWarps;
    const int my_warp = tm.rank * kTmaWarps + wib;
    const int ntasks = a.nstrips * a.nbands;
    long long nresid = 0;
    for (long long it = 0; ok && !done && it < a.nsteps; ++it) {
        const int par = (int)(step & 1);

        // ---- interior -----------------------------------------------------
        unsigned long long ws_key = 0ull;
        unsigned int nf = 0u;
        for (int task = my_warp; ok && task < ntasks; task += team_warps) {
            const int strip = task % a.nstrips;
            int l_begin, l_end;
            tma_band(1, a.g.L, a.nbands, task / a.nstrips, l_begin, l_end);
            if (l_begin >= l_end) continue;
            tma_warp_setup(w, a.g, strip, par ? a.buf0 : a.buf1, st, a.cphys, a.len, dt,
                           par ? map1 : map0);
            if (lane == 0) fence_proxy_async_global();
            __syncwarp();
            if (!tma_band_run<true, true>(w, l_begin, l_end, jrow, ws_key, nf)) ok = false;
        }
        {
            unsigned long long key[1] = {ws_key};
            unsigned long long *dst[1] = {&gs->ws[par]};
            block_max_atomic<1>(key, nf, dst, &gs->nf[par]);
        }
        ok = __syncthreads_and(ok) && team_barrier(tm);
        if (!ok) break;
        if (tm.rank == 0 && threadIdx.x == 0) {
            gs->ws[par ^ 1] = 0ull;  // next step's slot: last read before this barrier
            gs->nf[par ^ 1] = 0u;
        }

        // ---- boundary ring ---------------------------------------------------
        {
            unsigned long long key[1];
            unsigned int rnf;
            persist_ring_phase(a, pb.seg, par, dt, tm.rank, tm.size, key[0], rnf);
            unsigned long long *dst[1] = {&gs->ws[par]};
            block_max_atomic<1>(key, rnf, dst, &gs->nf[par]);
        }
        ok = team_barrier(tm);
        if (!ok) break;

        // ---- controller (identical in every block of the team) --------------
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
            persist_resid_phase(a, par, tm.rank, tm.size, key, rnf);
            unsigned long long *dst[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) dst[k] = &gs->rkey[rp][k];
            block_max_atomic<16>(key, rnf, dst, &gs->rnf[rp]);
            ok = team_barrier(tm);
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
            if (tm.rank == 0 && threadIdx.x == 0) {
#pragma unroll
                for (int k = 0; k < 16; ++k) gs->rkey[rp ^ 1][k] = 0ull;
                gs->rnf[rp ^ 1] = 0u;
            }
            ++nresid;
        }

        if (tm.rank == 0 && threadIdx.x == 0) {
            st->t = t;
            st->step = step;
            st->dt = dt;
            st->dt_used = dt_used;
            st->last_ws = ws;
            st->ws_valid = 1;
            st->nonfinite = nonfinite;
            st->done = done;
            if (done) st->done_ns = global_ns();
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
    return ok;
}

__device__ __forceinline__ PersistBlock persist_block(unsigned char *raw, PersistRun *run) {
    PersistBlock pb;
    pb.tma = tma_smem_base(raw);
    pb.seg = reinterpret_cast<SegDesc *>(pb.tma + kTmaSmem - 128);
    pb.run = run;
    return pb;
}

__device__ __forceinline__ void persist_warp_init(TmaWarp &w, const PersistBlock &pb,
                                                  const CUtensorMap *map) {
    const int wib = threadIdx.x >> 5;
    w.stage = reinterpret_cast<double *>(pb.tma) + wib * kTmaStages * kTmaRow;
    w.bar0 = smem_addr(pb.tma + kTmaWarps * kTmaStages * kTmaRowBytes) + 8u * wib * kTmaStages;
    w.map = map;
    w.lane = threadIdx.x & 31;
    w.init();
}

// One solve, the whole grid as one team.
__global__ void __launch_bounds__(kPersistThreads, MPD_PERSIST_MINB)
    lf_persist_kernel(const __grid_constant__ CUtensorMap map0,
                      const __grid_constant__ CUtensorMap map1,
                      const __grid_constant__ PersistArgs a, GridSync *gs) {
    extern __shared__ __align__(128) unsigned char persist_smem[];
    __shared__ PersistRun run;
    const PersistBlock pb = persist_block(persist_smem, &run);
    TmaWarp w;
    persist_warp_init(w, pb, &map0);
    uint32_t jrow = 0;
    TeamCtx tm;
    tm.rank = (int)blockIdx.x;
    tm.size = (int)gridDim.x;
    tm.gs = gs;
    persist_solve(a, &map0, &map1, tm, pb, w, jrow);
}

// A batch: team k is blocks [team_first[k], team_first[k+1]) and runs solves
// order[solve_first[k] .. solve_first[k+1]) one after the other.
struct BatchArgs {
    const PersistArgs *solves;   // per solve
    const CUtensorMap *maps;     // per solve: map of buf0, map of buf1 (64-byte aligned)
    const int *team_first;       // nteams + 1 block offsets
    const int *solve_first;      // nteams + 1 offsets into order
    const int *order;            // solve indices, grouped by team
    GridSync *gs;                // per team
    int nteams;
};

__global__ void __launch_bounds__(kPersistThreads, MPD_PERSIST_MINB)
    lf_batch_kernel(const __grid_constant__ BatchArgs b) {
    extern __shared__ __align__(128) unsigned char persist_smem[];
    __shared__ PersistRun run;
    __shared__ int s_team;
    if (threadIdx.x == 0) {
        int lo = 0, hi = b.nteams - 1;  // last team whose first block <= blockIdx.x
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (b.team_first[mid] <= (int)blockIdx.x) lo = mid;
            else hi = mid - 1;
        }
        s_team = lo;
    }
    __syncthreads();
    const int team = s_team;
    const int first = b.team_first[team];
    if ((int)blockIdx.x >= b.team_first[team + 1]) return;  // past the last team
    const PersistBlock pb = persist_block(persist_smem, &run);
    TmaWarp w;
    persist_warp_init(w, pb, b.maps);
    uint32_t jrow = 0;
    TeamCtx tm;
    tm.rank = (int)blockIdx.x - first;
    tm.size = b.team_first[team + 1] - first;
    tm.gs = b.gs + team;
    for (int k = b.solve_first[team]; k < b.solve_first[team + 1]; ++k) {
        const int s = b.order[k];
        if (!persist_solve(b.solves[s], b.maps + 2 * s, b.maps + 2 * s + 1, tm, pb, w, jrow))
            break;
    }
}

// Resident blocks per SM of the persistent kernels (0 if they cannot run).
inline cudaError_t persist_blocks_per_sm(int &per_sm) {
    per_sm = 0;
    cudaError_t e = cudaFuncSetAttribute(lf_persist_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kPersistSmem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(lf_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kPersistSmem);
    if (e != cudaSuccess) return e;
    int a = 0, b = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, lf_persist_kernel, kPersistThreads,
                                                      kPersistSmem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, lf_batch_kernel, kPersistThreads,
                                                      kPersistSmem);
    if (e != cudaSuccess) return e;
    per_sm = a < b ? a : b;
    return cudaSuccess;
}

// Interior tasks of a solve run by a team of `blocks` blocks: strips of 30
// columns x bands of at least MPD_TMA_MIN_BAND rows, about one task per warp.
inline void persist_tasks(const Geo &g, int blocks, int &nstrips, int &nbands) {
    const int warps = blocks * kTmaWarps;
    nstrips = (g.M + kFastCells - 1) / kFastCells;
    int nb = warps / nstrips;
    if (nb > g.L / MPD_TMA_MIN_BAND) nb = g.L / MPD_TMA_MIN_BAND;
    if (nb < 1) nb = 1;
    nbands = nb;
}

// Blocks of one cooperative wave of lf_persist_kernel and its interior plan.
inline cudaError_t plan_lf_persist(const Geo &g, int device, TmaPlan &plan) {
    int sms = 0, per_sm = 0, coop = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
    if (e != cudaSuccess) return e;
    if (!coop) return cudaErrorNotSupported;
    e = persist_blocks_per_sm(per_sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorNotSupported;
    plan.blocks = sms * per_sm;
    persist_tasks(g, plan.blocks, plan.nstrips, plan.nbands);
    return cudaSuccess;
}

inline cudaError_t launch_lf_persist(const TmaPlan &plan, const CUtensorMap &map0,
                                     const CUtensorMap &map1, const PersistArgs &a,
                                     GridSync *gs, cudaStream_t stream) {
    void *args[] = {const_cast<CUtensorMap *>(&map0), const_cast<CUtensorMap *>(&map1),
                    const_cast<PersistArgs *>(&a), &gs};
    return cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(lf_persist_kernel),
                                       dim3(plan.blocks), dim3(kPersistThreads), args,
                                       kPersistSmem, stream);
}

inline cudaError_t launch_lf_batch(int blocks, const BatchArgs &b, cudaStream_t stream) {
    void *args[] = {const_cast<BatchArgs *>(&b)};
    return cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(lf_batch_kernel),
                                       dim3(blocks), dim3(kPersistThreads), args, kPersistSmem,
                                       stream);
}

}  // namespace mpd
