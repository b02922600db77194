// CUDA kernels of the plain FP64 path (everything except the fast interior
// kernel, which lives in lf_fast.cuh).
#pragma once

#include <cuda_runtime.h>
#include <float.h>

#include <utility>

#include "lf_core.cuh"

// Programmatic dependent launch of the step kernels (1: on) and where each
// step kernel lets the next one be scheduled (0: at its end, 1: right after
// its own wait, 2: after its main work).  Measured on a B200 (1600 x 640 and
// 100 x 40 channels): 2 / 2 is the fastest; an early trigger lets the next
// kernel's blocks take SM space the running one still needs and costs up to
// 4 us a step on the large grid.
#ifndef MPD_PDL
#define MPD_PDL 1
#endif
#ifndef MPD_PDL_TRIG_INT
#define MPD_PDL_TRIG_INT 2
#endif
#ifndef MPD_PDL_TRIG_BC
#define MPD_PDL_TRIG_BC 2
#endif

namespace mpd {

// Programmatic dependent launch.  A kernel launched with launch_pdl may be
// scheduled while the previous kernel of its stream is still running; before
// it reads anything that kernel writes it calls pdl_wait (which returns once
// the previous kernel has completed and its writes are visible; a no-op
// without the launch attribute), and pdl_trigger lets the next kernel of the
// stream be scheduled in turn.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t stream, Args &&...args) {
#if MPD_PDL
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
#else
    kernel<<<grid, block, smem, stream>>>(std::forward<Args>(args)...);
    return cudaGetLastError();
#endif
}

// What the per-call host path (mpd_compute_dt after mpd_advance) needs of
// the controller, written by it into mapped pinned host memory each step, so
// the host reads it after an event instead of copying the whole state back.
struct HostMirror {
    long long step;
    double last_ws;
    int ws_valid, wait_fail;
};

// Device-resident controller and reduction accumulators of one solve.  The
// boundary kernel's last block finalises each step here, so a captured CUDA
// graph can run many steps without the host (dt, t, step, stop flags stay on
// the device).
struct DevState {
    double t, dt, dt_used, T;
    long long step, max_steps;
    int done, converged, run_mode, adaptive;
    double cfl, growth, dt_min, dt_max;
    double resid_tol;
    int resid_every, want_ws;
    double conv_thr;
    int check_freq, check_due;
    double last_ws, last_resid, last_change;
    int ws_valid, nonfinite, resid_valid, wait_fail;
    unsigned long long ws_acc;
    unsigned long long num_acc[8], den_acc[8];
    unsigned int nf_acc, arrive;
    unsigned int res_nf, res_arrive;
    long long resid_step;
    unsigned long long t0_ns, done_ns;  // persistent loops: first step taken, run done
    HostMirror *mirror;                 // mapped host memory, or null
};

constexpr int kFlagWs = 1;

__device__ __forceinline__ int step_flags(const DevState *st) { return st->want_ws ? kFlagWs : 0; }

// Non-negative double as an order-preserving 64-bit key; NaN reported as 0
// and flagged.
__device__ __forceinline__ unsigned long long max_key(double x, unsigned int &nf) {
    if (!(x == x)) {
        nf = 1u;
        return 0ull;
    }
    return (unsigned long long)__double_as_longlong(x > 0.0 ? x : 0.0);
}

// Block-wide max of NV keys (any block size <= 1024, multiple of 32) followed
// by one atomicMax per key; also ORs the non-finite flag.
template <int NV>
__device__ __forceinline__ void block_max_atomic(unsigned long long (&key)[NV], unsigned int nf,
                                                 unsigned long long *dst[NV], unsigned int *nf_dst) {
    __shared__ unsigned long long red[32][NV];
    __shared__ unsigned int nf_red[32];
    const int lane = threadIdx.x & 31;
    const int warp = (threadIdx.x + threadIdx.y * blockDim.x) >> 5;
    const int nwarps = (blockDim.x * blockDim.y + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        unsigned long long v = key[k];
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
            v = w > v ? w : v;
        }
        key[k] = v;
    }
    nf = __any_sync(0xffffffffu, nf != 0u) ? 1u : 0u;
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) red[warp][k] = key[k];
        nf_red[warp] = nf;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            unsigned long long v = lane < nwarps ? red[lane][k] : 0ull;
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
                v = w > v ? w : v;
            }
            if (lane == 0 && dst[k] && v) atomicMax(dst[k], v);
        }
        unsigned int f = lane < nwarps ? nf_red[lane] : 0u;
        f = __any_sync(0xffffffffu, f != 0u) ? 1u : 0u;
        if (lane == 0 && f) atomicOr(nf_dst, 1u);
    }
}

// Running maximum wave speed of the cells a thread finished.
struct CellStats {
    unsigned long long key[1];
    unsigned int nf;
    __device__ __forceinline__ void init() {
        key[0] = 0ull;
        nf = 0u;
    }
    __device__ __forceinline__ void add_ws(double s) {
        if (!isfinite(s)) nf = 1u;
        const unsigned long long k = max_key(s, nf);
        key[0] = k > key[0] ? k : key[0];
    }
    __device__ __forceinline__ void flush(DevState *st) {
        unsigned long long *dst[1] = {&st->ws_acc};
        block_max_atomic<1>(key, nf, dst, &st->nf_acc);
    }
};

// Boundary-ring cell (l, m) of one step: its final conserved values into v.u,
// and the full reconstruction of the cell: its wave speed (want_ws) and, for
// the wall columns, the "old" value the next step's faces read (wall lines
// wnext).  No L1 prefetches ahead of the chain: 20-40 of them per cell queued
// in front of the chain's own first loads (measured on a B200: 35.87 us a
// 1600 x 640 step with them, 35.50 without).
__device__ __forceinline__ void ring_cell_at(const BcView &v, int l, int m, double *wnext,
                                             bool want_ws, CellStats &cs) {
    const Geo &g = v.g;
    double uf[8];
    bc_ring_final(v, l, m, uf);
    const size_t ix = g.ix(l, m);
#pragma unroll
    for (int k = 0; k < 8; ++k) v.u[(size_t)k * g.ps + ix] = uf[k];
    const bool wall = m == 1 || m == g.M + 1;
    if (want_ws || wall) {
        const double r = g.r(l, m);
        const Phys q = recon_bc(v, uf, r);
        if (want_ws)
            cs.add_ws(v.fast ? fast_wave_speed(uf, r, rcp_nr(r), g.gamma) : wave_speed(q, g.gamma));
        if (wall) store_line_phys(wnext, v.len, m == 1 ? 0 : 1, l, q);
    }
}

// Boundary-ring slot i of one step (nothing for an idle slot).
__device__ __forceinline__ void ring_cell_update(const BcView &v, int i, double *wnext,
                                                 bool want_ws, CellStats &cs) {
    int l, m;
    if (ring_cell(v.g, i, l, m)) ring_cell_at(v, l, m, wnext, want_ws, cs);
}

// The boundary inputs of one step: views of the state, the central and wall
// lines and the face table.
__device__ __forceinline__ BcView make_bc_view(const Geo &g, const double *u0, double *u,
                                               const double *ic, const double *cphys,
                                               const double *wphys, int len, bool first, int fast,
                                               double dt, const BcTable &bc) {
    BcView v;
    v.g = g;
    v.u0 = u0;
    v.u = u;
    v.ic = ic;
    v.cphys = cphys;
    v.wphys = wphys;
    v.len = len;
    v.first = first ? 1 : 0;
    v.fast = fast;
    v.dt = dt;
    v.bc = bc;
    return v;
}

__device__ __forceinline__ unsigned int atom_add_acq_rel_u32(unsigned int *p, unsigned int v) {
    unsigned int old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;"
                 : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// True in thread 0 of the last block of the grid to get here, after every
// block's writes (state, lines, reduction atomics) are visible to it.  Every
// thread of every block calls it.  The barrier orders the block's writes
// before thread 0's release (release is cumulative over what the barrier
// made visible to it); the arrivals form one read-modify-write chain, so
// the last one's acquire sees every block's writes.
// (Measured on a B200 against a fence in every thread before the barrier
// and one after the atomic: 0.5 us less per step at 1600 x 640.)
__device__ __forceinline__ bool last_block_of_grid(unsigned int *counter) {
    __syncthreads();
    if (threadIdx.x != 0) return false;
    return atom_add_acq_rel_u32(counter, 1u) == gridDim.x - 1;
}

__device__ __forceinline__ bool last_block_arrived(DevState *st) {
    return last_block_of_grid(&st->arrive);
}

// End of step `step` (dt the step used), run by one thread once every cell's
// reductions are in: wave speed and non-finite flag, t and step, and in run
// mode the next dt and the stop flags; then the accumulators are cleared.
__device__ __forceinline__ void step_controller(const Geo &g, DevState *st, long long step,
                                                double dt, int flags) {
    // All reads first, through L2 and independent of each other, so the
    // controller costs one memory round trip instead of one per field.
    const unsigned long long ws_bits = __ldcg(&st->ws_acc);
    const unsigned int nf_acc = __ldcg(&st->nf_acc);
    const double t0 = __ldcg(&st->t);
    const int nonfinite0 = __ldcg(&st->nonfinite);
    const int run_mode = __ldcg(&st->run_mode);
    const int adaptive = __ldcg(&st->adaptive);
    const double cfl = __ldcg(&st->cfl), growth = __ldcg(&st->growth);
    const double dt_min = __ldcg(&st->dt_min), dt_max = __ldcg(&st->dt_max);
    const double T = __ldcg(&st->T);
    const long long max_steps = __ldcg(&st->max_steps);
    const double conv_thr = __ldcg(&st->conv_thr);
    const int check_freq = __ldcg(&st->check_freq);

    const double ws = (flags & kFlagWs) ? __longlong_as_double((long long)ws_bits) : 0.0;
    if (flags & kFlagWs) st->last_ws = ws;
    st->ws_valid = (flags & kFlagWs) ? 1 : 0;
    const int nonfinite = (nonfinite0 || nf_acc || !isfinite(ws)) ? 1 : 0;
    st->nonfinite = nonfinite;
    const double t = t0 + dt;
    const long long nstep = step + 1;
    st->t = t;
    st->dt_used = dt;
    st->step = nstep;
    st->resid_valid = 0;  // the residual of this step is evaluated on request
    if (run_mode) {
        double dtn = dt;
        if (adaptive) dtn = compute_dt_from_speed(ws, g.dz, g.dy, cfl, growth, dt_min, dt_max, dt);
        const int done = (nonfinite || !(t < T) || nstep >= max_steps) ? 1 : 0;
        if (t + dtn > T) dtn = T - t;
        st->dt = dtn;
        st->check_due = (conv_thr > 0.0 && check_freq > 0 && nstep % check_freq == 0) ? 1 : 0;
        st->done = done;
    }
    st->ws_acc = 0ull;
    st->nf_acc = 0u;
    // per-call mode only: a run's loop is never watched from the host (the
    // host state, mirror included, is refreshed when the run ends), and a
    // system-scope fence costs each step ~1.7 us on its critical path
    // (measured on a B200: a run's step 39.7 -> 36.1 us without the two it had)
    HostMirror *hm = run_mode ? nullptr : st->mirror;
    if (hm) {
        if (flags & kFlagWs) hm->last_ws = ws;
        hm->ws_valid = (flags & kFlagWs) ? 1 : 0;
        hm->wait_fail = __ldcg(&st->wait_fail);
        // the fields above before the step number (a release at system
        // scope): a host that sees the new step sees them too
        asm volatile("st.release.sys.b64 [%0], %1;" ::"l"(&hm->step), "l"(nstep) : "memory");
    }
    // the next arrivals come from a later launch, which the launch order
    // places after every store of this one
    st->arrive = 0u;
}

// Exact interior update (Solver::ComputeCentralUpdate + the implicit
// UpdatePhysicalFromU of the neighbours), one thread per cell
// l in [1, L], m in [2, M].  FIRST: the stencil reads the initial physical
// planes instead of reconstructing them (step 0 of src/main.cpp:147-148).
template <bool FIRST>
__global__ void __launch_bounds__(256) lf_exact_kernel(Geo g, double *buf0, double *buf1,
                                                       const double *__restrict__ ic, DevState *st,
                                                       double dt_arg, int use_state_dt,
                                                       double *cphys, int len) {
    if (st->done) return;
    const long long step = st->step;
    const double *__restrict__ u0 = (step & 1) ? buf1 : buf0;
    double *__restrict__ u = (step & 1) ? buf0 : buf1;
    const double dt = use_state_dt ? st->dt : dt_arg;
    const int flags = step_flags(st);
    const int m = 2 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int l = 1 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
    CellStats cs;
    cs.init();
    if (m <= g.M && l <= g.L) {
        double U[5][8];
        Phys Q[5];
        double R[5];
        const int ls[5] = {l, l + 1, l - 1, l, l};
        const int ms[5] = {m, m, m, m + 1, m - 1};
#pragma unroll
        for (int p = 0; p < 5; ++p) {
            const size_t i = g.ix(ls[p], ms[p]);
            R[p] = g.r(ls[p], ms[p]);
            load_cons(u0, g.ps, i, U[p]);
            if (ls[p] == 0 || ls[p] == g.L + 1) Q[p] = phys_zero();
            else if (FIRST) Q[p] = load_phys(ic, g.ps, i);
            else Q[p] = recon_exact(U[p], R[p], g.gamma);
        }
        double out[8];
        lf_cell_exact(U, Q, R, dt, g.dz, g.dr[l], out);
        const size_t ic0 = g.ix(l, m);
#pragma unroll
        for (int k = 0; k < 8; ++k) u[(size_t)k * g.ps + ic0] = out[k];
        // cells no boundary face can overwrite feed the wave speed; cells the
        // faces read go to the central lines
        if ((flags & kFlagWs) && l >= 2 && l <= g.L - 1)
            cs.add_ws(wave_speed(recon_exact(out, R[0], g.gamma), g.gamma));
        if (wants_central(g.L, g.M, l, m)) store_central(cphys, len, g.L, g.M, l, m, out);
    }
    if (flags) cs.flush(st);
}

// Boundary faces, one thread per boundary-ring cell, plus the end-of-step
// controller in the last block to finish.  A few thousand threads on a
// dependent chain: registers are not what limits it, spills would lengthen
// the chain, so the register budget is lifted (MPD_BC_MAXNREG 0: the
// compiler's default for 64-thread blocks, 128 registers with spills; 255:
// ~214, no spills, 100 x 40 step 18.2 -> 17.4 us on a B200).
#ifndef MPD_BC_MAXNREG
#define MPD_BC_MAXNREG 255
#endif
#ifndef MPD_BC_SMEM_SEG
#define MPD_BC_SMEM_SEG 1
#endif
static_assert(sizeof(SegDesc) % 16 == 0, "segment descriptors are copied as 16-byte words");
#if MPD_BC_MAXNREG
#define MPD_BC_BOUNDS __maxnreg__(MPD_BC_MAXNREG)
#else
#define MPD_BC_BOUNDS __launch_bounds__(64)
#endif
__global__ void MPD_BC_BOUNDS bc_kernel(Geo g, double *buf0, double *buf1,
                                                 const double *__restrict__ ic, BcTable bc,
                                                 DevState *st, double dt_arg, int use_state_dt,
                                                 const double *cphys, double *wall0, double *wall1,
                                                 int len, int fast) {
#if MPD_BC_SMEM_SEG
    // The face segments into shared memory (dynamic, nseg_total of them):
    // every ring cell walks them in its dependent chain.  No kernel writes
    // them, so this runs before the previous kernel of the stream is waited for.
    extern __shared__ __align__(16) unsigned char bc_smem_raw[];
    {
        const int4 *src = reinterpret_cast<const int4 *>(bc.seg);
        int4 *dst = reinterpret_cast<int4 *>(bc_smem_raw);
        const int n = bc.nseg_total * (int)(sizeof(SegDesc) / sizeof(int4));
        for (int k = threadIdx.x; k < n; k += blockDim.x) dst[k] = src[k];
        __syncthreads();
        bc.seg = reinterpret_cast<const SegDesc *>(bc_smem_raw);
    }
#endif
    pdl_wait();
    if (MPD_PDL_TRIG_BC == 1) pdl_trigger();
    // the step's state in one memory round trip
    const int done = st->done;
    const long long step = st->step;
    const double st_dt = st->dt;
    const int flags = step_flags(st);
    if (done) return;
    const double *u0 = (step & 1) ? buf1 : buf0;
    double *u = (step & 1) ? buf0 : buf1;
    const double dt = use_state_dt ? st_dt : dt_arg;
    const BcView v = make_bc_view(g, u0, u, ic, cphys, (step & 1) ? wall1 : wall0, len,
                                  step == 0, fast, dt, bc);
    double *wnext = (step & 1) ? wall0 : wall1;
    CellStats cs;
    cs.init();
    const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (i < ring_count(g)) ring_cell_update(v, i, wnext, (flags & kFlagWs) != 0, cs);
    if (flags) cs.flush(st);
    if (MPD_PDL_TRIG_BC == 2) pdl_trigger();
    if (last_block_arrived(st)) step_controller(g, st, step, dt, flags);
}

// The boundary ring of a fast step run beside the interior kernel instead of
// after it (the interior launched just before, lf_tma_kernel<.., true>, which
// writes rows 2..L-1 only and lets this kernel start at once).  Every value
// the faces need from this step's central update is recomputed from the
// input state (BcView::recompute), so nothing here waits for the interior:
// the ring's dependent chains (several microseconds of loads, face
// evaluations and reconstructions per cell) overlap the interior instead of
// following it.  Blocks of one warp at most 128 registers fit beside three
// interior blocks of an SM; a grid of at most one block per SM strides over
// the ring slots.  Only the controller needs the interior's wave-speed
// maximum: the last ring block to finish waits for the interior to complete
// (pdl_wait), then runs it.  The state read before that wait was written by
// the previous step's controller, which completed before the interior
// launched; it is read through L2.  Exited blocks count as having let the
// next kernel in; the last one does so once the interior has completed.
#ifndef MPD_OVERLAP_MAXNREG
#define MPD_OVERLAP_MAXNREG 128
#endif
__global__ void __maxnreg__(MPD_OVERLAP_MAXNREG)
    bc_overlap_kernel(Geo g, double *buf0, double *buf1, const double *__restrict__ ic,
                      BcTable bc, DevState *st, double dt_arg, int use_state_dt, double *wall0,
                      double *wall1, int len) {
    extern __shared__ __align__(16) unsigned char bc_smem_raw[];
    {
        const int4 *src = reinterpret_cast<const int4 *>(bc.seg);
        int4 *dst = reinterpret_cast<int4 *>(bc_smem_raw);
        const int n = bc.nseg_total * (int)(sizeof(SegDesc) / sizeof(int4));
        for (int k = threadIdx.x; k < n; k += blockDim.x) dst[k] = src[k];
        __syncthreads();
        bc.seg = reinterpret_cast<const SegDesc *>(bc_smem_raw);
    }
    const int done = __ldcg(&st->done);
    const long long step = __ldcg(&st->step);
    const double st_dt = __ldcg(&st->dt);
    const int flags = __ldcg(&st->want_ws) ? kFlagWs : 0;
    if (done) return;
    const double *u0 = (step & 1) ? buf1 : buf0;
    double *u = (step & 1) ? buf0 : buf1;
    const double dt = use_state_dt ? st_dt : dt_arg;
    BcView v = make_bc_view(g, u0, u, ic, nullptr, (step & 1) ? wall1 : wall0, len, step == 0,
                            1, dt, bc);
    v.recompute = 1;
    double *wnext = (step & 1) ? wall0 : wall1;
    CellStats cs;
    cs.init();
    const int n = ring_count(g);
    const int stride = (int)(gridDim.x * blockDim.x);
    for (int i = (int)(blockIdx.x * blockDim.x + threadIdx.x); i < n; i += stride)
        ring_cell_update(v, i, wnext, (flags & kFlagWs) != 0, cs);
    if (flags) cs.flush(st);
    if (!last_block_arrived(st)) return;
    pdl_wait();
    // every interior block has retired: the next step's interior is placed
    // on a free GPU (all its blocks at once, spread over the SMs) while this
    // controller runs
    pdl_trigger();
    if (__ldcg(&st->done)) {
        // the interior gave up on a bounded wait and stopped the run: the
        // step is not taken
        st->arrive = 0u;
        return;
    }
    step_controller(g, st, step, dt, flags);
}

// L-inf residual of the step that just finished (new; the reference has only
// the relative-L2 change): R = max_k |u_k^{n+1} - u_k^n|_inf / max(|u_k^n|_inf,
// 1e-300) over the interior cells, reading both ping-pong buffers.  In run
// mode it also stops the loop once R <= residual_tol.  Skips a state it
// already evaluated (a run may have stopped before this graph node).
// Running maxima of |u_new - u_old| and |u_old| per conserved value.  A NaN
// is left out of the maxima (fmax drops it) and flagged through `poison`
// (d * 0 is NaN for a NaN or infinite difference, 0 otherwise): the same
// maxima and non-finite outcome as keys with a per-value NaN test, in four
// FP64 operations per value.
struct ResidAcc {
    double dmax[8], omax[8], poison;

    __device__ __forceinline__ void init() {
#pragma unroll
        for (int k = 0; k < 8; ++k) dmax[k] = omax[k] = 0.0;
        poison = 0.0;
    }
    __device__ __forceinline__ void fold(const double (&an)[8], const double (&ao)[8]) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const double d = an[k] - ao[k];
            dmax[k] = fmax(dmax[k], fabs(d));
            omax[k] = fmax(omax[k], fabs(ao[k]));
            poison = fma(d, 0.0, poison);
        }
    }
    // Order-preserving keys (non-negative doubles) and the non-finite flag.
    __device__ __forceinline__ void keys(unsigned long long (&key)[16], unsigned int &nf) const {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            key[k] = (unsigned long long)__double_as_longlong(dmax[k]);
            key[8 + k] = (unsigned long long)__double_as_longlong(omax[k]);
        }
        nf = (poison == poison) ? 0u : 1u;
    }
};

// force: evaluate even when this step's residual is already known (timing).
__global__ void __launch_bounds__(256) residual_kernel(Geo g, const double *buf0,
                                                       const double *buf1, DevState *st,
                                                       int force) {
    const long long step = st->step;
    if (step == 0 || (!force && st->resid_step == step)) return;
    const double *un = (step & 1) ? buf1 : buf0;
    const double *uo = (step & 1) ? buf0 : buf1;
    ResidAcc acc;
    acc.init();
    // Items of one row l in [1, L] x one pair of columns (2c, 2c + 1),
    // c < (M + 3) / 2: columns 0 .. M+1, plus the ghost column M+2 when M is
    // odd.  Ghost columns are zero in both buffers, so they leave every
    // maximum unchanged.  A thread issues all 16 of an item's 16-byte loads
    // (8 planes, new and old state) before using any; rows are 256-byte
    // aligned (pitch a multiple of 32 doubles), so every pair is a 16-byte
    // aligned load and a warp reads 512 contiguous bytes per plane.  The old
    // state is read with the streaming policy (the next step overwrites it);
    // the new one stays in L2 as that step's input.
    const int ncp = (g.M + 3) >> 1;
    const int items = g.L * ncp;
    const int stride = (int)(gridDim.x * blockDim.x);
    for (int it = (int)(blockIdx.x * blockDim.x + threadIdx.x); it < items; it += stride) {
        const int row = it / ncp;
        const int c = it - row * ncp;
        const size_t i = g.ix(1 + row, 2 * c);
        double2 a[8], b[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            a[k] = __ldg(reinterpret_cast<const double2 *>(un + (size_t)k * g.ps + i));
            b[k] = __ldcs(reinterpret_cast<const double2 *>(uo + (size_t)k * g.ps + i));
        }
        double an[8], ao[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            an[k] = a[k].x;
            ao[k] = b[k].x;
        }
        acc.fold(an, ao);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            an[k] = a[k].y;
            ao[k] = b[k].y;
        }
        acc.fold(an, ao);
    }
    unsigned long long key[16];
    unsigned int nf;
    acc.keys(key, nf);
    unsigned long long *dst[16];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        dst[k] = &st->num_acc[k];
        dst[8 + k] = &st->den_acc[k];
    }
    block_max_atomic<16>(key, nf, dst, &st->res_nf);
    if (!last_block_of_grid(&st->res_arrive)) return;
    unsigned long long num[8], den[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        num[k] = __ldcg(&st->num_acc[k]);
        den[k] = __ldcg(&st->den_acc[k]);
    }
    const unsigned int res_nf = __ldcg(&st->res_nf);
    const int run_mode = __ldcg(&st->run_mode);
    const double resid_tol = __ldcg(&st->resid_tol);
    const int nonfinite0 = __ldcg(&st->nonfinite);
    double R = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const double n = __longlong_as_double((long long)num[k]);
        const double d = __longlong_as_double((long long)den[k]);
        const double q = n / (d > 1e-300 ? d : 1e-300);
        R = q > R ? q : R;
        st->num_acc[k] = 0ull;
        st->den_acc[k] = 0ull;
    }
    const int nonfinite = (nonfinite0 || res_nf || !isfinite(R)) ? 1 : 0;
    st->nonfinite = nonfinite;
    st->res_nf = 0u;
    st->last_resid = R;
    st->resid_valid = 1;
    st->resid_step = step;
    if (run_mode && resid_tol > 0.0 && R <= resid_tol) {
        st->converged = 1;
        st->done = 1;
    }
    if (run_mode && nonfinite) st->done = 1;
    st->res_arrive = 0u;  // the next arrivals come from a later launch
}

// ---------------------------------------------------------------------------
// Reductions over the current state (Diagnostics / Verification).
// The current physical state is the initial condition before the first step,
// otherwise UpdatePhysicalFromU of the current conserved planes.
// ---------------------------------------------------------------------------
struct StateView {
    Geo g;
    const double *u0;
    const double *ic;
    int first;
    __device__ __forceinline__ Phys phys(int l, int m) const {
        const size_t i = g.ix(l, m);
        if (first) return load_phys(ic, g.ps, i);
        double u[8];
        load_cons(u0, g.ps, i, u);
        return recon_exact(u, g.r(l, m), g.gamma);
    }
};

// The current state's view, chosen on the device from the step counter so
// that the same launch works inside captured graphs.
struct StateBufs {
    Geo g;
    const double *buf0, *buf1, *ic;
    const DevState *st;
    __device__ __forceinline__ StateView view() const {
        StateView sv;
        sv.g = g;
        const long long step = st->step;
        sv.u0 = (step & 1) ? buf1 : buf0;
        sv.ic = ic;
        sv.first = step == 0;
        return sv;
    }
};

// Diagnostics::MaxWaveSpeed over [1,L] x [1,M+1] (max is order-free: exact).
__global__ void wave_speed_kernel(StateBufs sb, unsigned long long *out) {
    const StateView sv = sb.view();
    unsigned long long key[1] = {0ull};
    unsigned int nf = 0u;
    const int total = sv.g.L * (sv.g.M + 1);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int l = 1 + i / (sv.g.M + 1), m = 1 + i % (sv.g.M + 1);
        const double s = wave_speed(sv.phys(l, m), sv.g.gamma);
        // std::max(local_max, s): NaN never replaces the running max
        if (s == s) {
            const unsigned long long k = max_key(s, nf);
            key[0] = k > key[0] ? k : key[0];
        }
    }
    unsigned long long *dst[1] = {out};
    block_max_atomic<1>(key, nf, dst, reinterpret_cast<unsigned int *>(out + 1));
}

// Verification::CheckRadialSymmetry (src/verification.cpp:121-146).
__global__ void radial_kernel(StateBufs sb, unsigned long long *out) {
    const StateView sv = sb.view();
    unsigned long long key[1] = {0ull};
    unsigned int nf = 0u;
    const int W = sv.g.M;  // m = 1..M (pairs m, m+1)
    const int total = sv.g.L * W;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int l = 1 + i / W, m = 1 + i % W;
        const double a = sv.phys(l, m).rho;
        const double b = sv.phys(l, m + 1).rho;
        const double mean = 0.5 * (a + b);
        if (mean > 1.0e-15) {
            const double q = fabs(b - a) / mean;
            if (q == q) {
                const unsigned long long k = max_key(q, nf);
                key[0] = k > key[0] ? k : key[0];
            }
        }
    }
    unsigned long long *dst[1] = {out};
    block_max_atomic<1>(key, nf, dst, reinterpret_cast<unsigned int *>(out + 1));
}

// Deterministic block sums: each block writes NV partial sums for its rows,
// a single-block pass adds the partials in block order.
template <int NV>
__device__ __forceinline__ void block_sum_store(double (&v)[NV], double *partials) {
    __shared__ double red[32][NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) red[warp][k] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < NV; ++k) {
            double s = 0.0;
            for (int w = 0; w < nwarps; ++w) s += red[w][k];
            partials[(size_t)blockIdx.x * NV + k] = s;
        }
    }
}

// The partials (nblocks x NV) are first copied into shared memory by the
// whole block (dynamic shared memory of nblocks * NV doubles), then value k
// is summed by thread k in block order: the same additions as a serial loop
// over global memory, without a dependent global load per addition.
__device__ __forceinline__ void stage_partials(const double *partials, int n, double *sh) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) sh[i] = partials[i];
    __syncthreads();
}

template <int NV>
__global__ void sum_partials_kernel(const double *partials, int nblocks, double *out) {
    extern __shared__ double sh_partials[];
    stage_partials(partials, nblocks * NV, sh_partials);
    if (threadIdx.x >= NV) return;
    double s = 0.0;
#pragma unroll 8
    for (int b = 0; b < nblocks; ++b) s += sh_partials[b * NV + threadIdx.x];
    out[threadIdx.x] = s;
}

// Verification::ComputeIntegrals (src/verification.cpp:16-45): block b sums
// rows l = 1 + b, 1 + b + gridDim.x, ... in m order.  Output order:
// mass, mom_z, mom_r, mom_phi, energy, mag_flux_z (u_7), mag_flux_phi (u_6).
__global__ void integrals_kernel(StateBufs sb, double *partials) {
    const StateView sv = sb.view();
    const Geo &g = sv.g;
    const double *u0 = sv.u0;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int l = 1 + blockIdx.x; l <= g.L; l += gridDim.x) {
        const double cell_area = g.dr[l] * g.dz;
        for (int m = 1 + threadIdx.x; m <= g.M + 1; m += blockDim.x) {
            const size_t i = g.ix(l, m);
            acc[0] += u0[0 * g.ps + i] * cell_area;
            acc[1] += u0[1 * g.ps + i] * cell_area;
            acc[2] += u0[2 * g.ps + i] * cell_area;
            acc[3] += u0[3 * g.ps + i] * cell_area;
            acc[4] += u0[4 * g.ps + i] * cell_area;
            acc[5] += u0[6 * g.ps + i] * cell_area;
            acc[6] += u0[5 * g.ps + i] * cell_area;
        }
    }
    block_sum_store<7>(acc, partials);
}

// Diagnostics::SolutionChange + Fields::SavePrev (src/diagnostics.cpp:71-106,
// src/fields.cpp:59-74): sums of squared differences against the prev planes
// and of squared values, then prev <- current.
__global__ void change_kernel(StateBufs sb, double *prev, double *partials, int save,
                              int only_if_due) {
    if (only_if_due && !sb.st->check_due) return;
    const StateView sv = sb.view();
    double acc[2] = {0.0, 0.0};
    const Geo &g = sv.g;
    for (int l = 1 + blockIdx.x; l <= g.L; l += gridDim.x) {
        for (int m = 1 + threadIdx.x; m <= g.M + 1; m += blockDim.x) {
            const size_t i = g.ix(l, m);
            const Phys q = sv.phys(l, m);
            const double x[7] = {q.rho, q.vz, q.vr, q.vphi, q.Hz, q.Hr, q.Hphi};
            double d[7];
#pragma unroll
            for (int k = 0; k < 7; ++k) d[k] = x[k] - prev[(size_t)k * g.ps + i];
            acc[0] += d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + d[3] * d[3] + d[4] * d[4]
                    + d[5] * d[5] + d[6] * d[6];
            acc[1] += x[0] * x[0] + x[1] * x[1] + x[2] * x[2] + x[3] * x[3] + x[4] * x[4]
                    + x[5] * x[5] + x[6] * x[6];
            if (save) {
#pragma unroll
                for (int k = 0; k < 7; ++k) prev[(size_t)k * g.ps + i] = x[k];
            }
        }
    }
    block_sum_store<2>(acc, partials);
}

// Final relative change and the run loop's convergence decision
// (src/main.cpp:233-247).  Runs as one thread after change_kernel.
__global__ void change_finish_kernel(const double *partials, int nblocks, DevState *st,
                                     int from_run) {
    if (from_run && !st->check_due) return;
    extern __shared__ double sh_partials[];
    stage_partials(partials, 2 * nblocks, sh_partials);
    if (threadIdx.x != 0) return;
    double sd = 0.0, sc = 0.0;
#pragma unroll 8
    for (int b = 0; b < nblocks; ++b) {
        sd += sh_partials[2 * b];
        sc += sh_partials[2 * b + 1];
    }
    const double nd = sqrt(sd), nc = sqrt(sc);
    const double change = (nc > 1e-15) ? (nd / nc) : nd;
    st->last_change = change;
    if (from_run) {
        st->check_due = 0;
        if (change < st->conv_thr) {
            st->converged = 1;
            st->done = 1;
        }
    }
}

// Diagnostics::GetMassFlux / GetThrust (src/integrals.cpp:45-112): the outlet
// column is summed serially in m order, as the reference does.  The terms of
// kOutletChunk points are evaluated by the block's threads at once (each
// with the reference's expression), then thread 0 adds them in m order: the
// same additions of the same terms as one thread doing everything.
constexpr int kOutletThreads = 256;
constexpr int kOutletChunk = 1024;
__global__ void __launch_bounds__(kOutletThreads) outlet_kernel(StateBufs sb, double inv_8pi,
                                                                double *out) {
    __shared__ double tm[kOutletChunk], tt[kOutletChunk];
    const StateView sv = sb.view();
    const Geo &g = sv.g;
    const int l = g.L;
    const double dr_out = g.dr[l];
    double sm = 0.0, sth = 0.0;
    for (int m0 = 1; m0 <= g.M + 1; m0 += kOutletChunk) {
        const int n = min(kOutletChunk, g.M + 2 - m0);
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const int m_local = m0 + j;
            const int m_global = m_local - 1;
            const double w = (m_global == 0 || m_global == g.M) ? 0.5 : 1.0;
            const Phys q = sv.phys(l, m_local);
            const double r = g.r(l, m_local);
            const double fm = q.rho * q.vz;
            const double Fm = fm * 2.0 * M_PI * r;
            tm[j] = w * Fm * dr_out;
            const double v_z2 = q.vz * q.vz;
            const double H2 = q.Hz * q.Hz + q.Hr * q.Hr + q.Hphi * q.Hphi;
            const double ft = q.rho * v_z2 + q.p + H2 * inv_8pi;
            const double Ft = ft * 2.0 * M_PI * r;
            tt[j] = w * Ft * dr_out;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
#pragma unroll 8
            for (int j = 0; j < n; ++j) {
                sm += tm[j];
                sth += tt[j];
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sm;
        out[1] = sth;
    }
}

// Materialise the 10 physical planes of the current state (pitched); ghost
// cells are zero as in the reference's Fields arrays.
// The 10 physical planes of the current state, dense: plane k at
// out + k (L+2)(M+3), cell (l, m) at l (M+3) + m (the host's layout, so one
// contiguous copy moves them all).
__global__ void phys_planes_kernel(StateBufs sb, double *out) {
    const StateView sv = sb.view();
    const Geo &g = sv.g;
    const int cols = g.M + 3, rows = g.L + 2;
    const int total = rows * cols;
    const size_t ps = (size_t)total;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int l = i / cols, m = i % cols;
        Phys q = phys_zero();
        if (l >= 1 && l <= g.L && m >= 1 && m <= g.M + 1) q = sv.phys(l, m);
        out[0 * ps + i] = q.rho;
        out[1 * ps + i] = q.vz;
        out[2 * ps + i] = q.vr;
        out[3 * ps + i] = q.vphi;
        out[4 * ps + i] = q.e;
        out[5 * ps + i] = q.p;
        out[6 * ps + i] = q.P;
        out[7 * ps + i] = q.Hz;
        out[8 * ps + i] = q.Hr;
        out[9 * ps + i] = q.Hphi;
    }
}

// Interior cells (l in 1..L, m in 1..M+1) of 10 dense host-layout planes into
// the pitched initial planes (their ghost cells are left as they are).
__global__ void scatter_phys_kernel(Geo g, const double *dense, double *ic) {
    const int cols = g.M + 3;
    const int W = g.M + 1;
    const int total = g.L * W;
    const size_t dps = (size_t)(g.L + 2) * cols;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int l = 1 + i / W, m = 1 + i % W;
        const size_t src = (size_t)l * cols + m, dst = g.ix(l, m);
#pragma unroll
        for (int k = 0; k < 10; ++k) ic[(size_t)k * g.ps + dst] = dense[(size_t)k * dps + src];
    }
}

// Wall lines of step 0: the initial condition on columns 1 and M+1.
// ExpressionIC::Apply (src/ics/expression_ic.cpp:286-324) on the device:
// one thread per cell, the compiled programs of the 8 fields in evaluation
// order, then p and P, into the 10 pitched physical planes (ghost cells
// stay as they are).  The same arithmetic as the host sweep (mpd_expression_ic)
// for every program that reads only earlier fields of its cell; the caller
// refuses the others.
struct IcPrograms {
    const int32_t *code;
    const double *consts;
    int code_off[8], const_off[8];
};

__global__ void expression_ic_kernel(Geo g, double *ic, IcPrograms pr) {
    const int W = g.M + 1;
    const long long total = (long long)g.L * W;
    const int plane_of[8] = {P_RHO, P_VZ, P_VR, P_VPHI, P_HZ, P_HR, P_HPHI, P_E};
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < total;
         c += (long long)gridDim.x * blockDim.x) {
        const int l = 1 + (int)(c / W), m = 1 + (int)(c % W);
        const int l_global = l - 1, m_global = m - 1;
        double sym[IC_COUNT];
        sym[IC_GAMMA] = g.gamma;
        sym[IC_BETA] = g.beta;
        sym[IC_HZ0] = g.H_z0;
        sym[IC_R0] = g.r_0;
        const double frac = m_global * g.dy;
        sym[IC_Z] = l_global * g.dz;
        sym[IC_R] = (1.0 - frac) * g.rin[l] + frac * g.rout[l];
        sym[IC_RZ] = (1.0 - frac) * g.drin[l] + frac * g.drout[l];
        for (int j = 0; j < 8; ++j) sym[IC_F0 + j] = 0.0;
        for (int j = 0; j < 8; ++j)
            sym[IC_F0 + j] = eval_code(pr.code + pr.code_off[j], pr.consts + pr.const_off[j], sym);
        const size_t i = g.ix(l, m);
        for (int j = 0; j < 8; ++j) ic[(size_t)plane_of[j] * g.ps + i] = sym[IC_F0 + j];
        const double rho = sym[IC_F0 + 0], e = sym[IC_F0 + 7];
        const double Hz = sym[IC_F0 + 4], Hr = sym[IC_F0 + 5], Hphi = sym[IC_F0 + 6];
        const double p = (g.gamma - 1.0) * rho * e;
        ic[(size_t)P_PG * g.ps + i] = p;
        ic[(size_t)P_PT * g.ps + i] = p + 0.5 * (Hz * Hz + Hr * Hr + Hphi * Hphi);
    }
}

__global__ void init_wall_kernel(Geo g, const double *ic, double *wall0, int len) {
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < g.L + 2; l += gridDim.x * blockDim.x) {
        const bool in = l >= 1 && l <= g.L;
        store_line_phys(wall0, len, 0, l, in ? load_phys(ic, g.ps, g.ix(l, 1)) : phys_zero());
        store_line_phys(wall0, len, 1, l, in ? load_phys(ic, g.ps, g.ix(l, g.M + 1)) : phys_zero());
    }
}

// Fields::InitConservative (src/fields.cpp:40-57) on the device: interior
// cells from the physical planes, ghosts zero.
__global__ void init_conservative_kernel(Geo g, const double *ic, double *u0) {
    const int cols = g.M + 3, rows = g.L + 2;
    const int total = rows * cols;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int l = i / cols, m = i % cols;
        const size_t o = g.ix(l, m);
        double u[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (l >= 1 && l <= g.L && m >= 1 && m <= g.M + 1) rebuild_u(load_phys(ic, g.ps, o), g.r(l, m), u);
#pragma unroll
        for (int k = 0; k < 8; ++k) u0[(size_t)k * g.ps + o] = u[k];
    }
}

}  // namespace mpd
