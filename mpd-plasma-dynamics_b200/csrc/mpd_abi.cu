// C ABI of the B200 solver (include/mpd_b200.h): handle lifetime, the step
// launch sequence, the graph-resident run loop, diagnostics and transfers.
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mpd_b200.h"
#include "bc_compile.hpp"
#include "kernels.cuh"
#include "lf_fast.cuh"
#include "lf_pair.cuh"
#include "lf_persist.cuh"
#include "lf_tma.cuh"

namespace mpd {
namespace {
thread_local std::string g_last_error;
}
void SetLastError(const std::string &msg) { g_last_error = msg; }
}  // namespace mpd

using mpd::SetLastError;

namespace {

int Fail(int code, const std::string &msg) {
    SetLastError(msg);
    return code;
}

#define MPD_CK(call)                                                                         \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return Fail(e_ == cudaErrorMemoryAllocation ? MPD_ERR_NOMEM : MPD_ERR_CUDA,      \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                 \
    } while (0)

constexpr int kRedBlocks = 592;  // 4 x 148 SMs for the deterministic sums
// Boundary-ring threads per block: measured on a B200, 32 and 128 no better
// than 64 and 256 2 us a step slower (fewer, fuller SMs lengthen the chains).
#ifndef MPD_BC_BLOCK
#define MPD_BC_BLOCK 64
#endif
constexpr int kBcBlock = MPD_BC_BLOCK;  // boundary-ring threads per block

// cuTensorMapEncodeTiled, fetched from the driver at run time (no -lcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                   const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                   const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn GetEncodeTiled() {
    static EncodeTiledFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return static_cast<EncodeTiledFn>(nullptr);
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

// The 8 conserved planes of one state buffer as a 3-D tensor
// {columns M+3, rows L+2, planes 8} with the row pitch and plane stride of the
// allocation; tiles are {box_cols columns, 1 row, 8 planes}, zero-filled outside.
int EncodeStateMap(CUtensorMap *map, double *base, int cols, int rows, int pitch, size_t ps,
                   int box_cols) {
    EncodeTiledFn enc = GetEncodeTiled();
    if (!enc) return Fail(MPD_ERR_CUDA, "cuTensorMapEncodeTiled unavailable from the driver");
    const cuuint64_t dims[3] = {(cuuint64_t)cols, (cuuint64_t)rows, 8};
    const cuuint64_t strides[2] = {(cuuint64_t)pitch * sizeof(double), (cuuint64_t)ps * sizeof(double)};
    const cuuint32_t box[3] = {(cuuint32_t)box_cols, 1, 8};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return Fail(MPD_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return MPD_OK;
}

}  // namespace

struct mpd_solver {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;
    mpd::Geo g{};
    int L = 0, M = 0, rows = 0, cols = 0, pitch = 0;
    size_t ps = 0;
    double *buf[2] = {nullptr, nullptr};
    double *ic = nullptr, *prev = nullptr, *geo = nullptr, *stage = nullptr;
    double *partials = nullptr, *small = nullptr;
    double *cphys = nullptr;                 // central lines (boundary inputs)
    double *wall[2] = {nullptr, nullptr};    // wall lines, by step parity
    int len = 0;                             // line length
    int resid_blocks = 0;                    // residual_kernel: one resident wave
    CUtensorMap tmap[2];                     // conserved planes of buf[0] / buf[1]
    CUtensorMap tmap_pair[2];                // the same with 64-column tiles
    mpd::TmaPlan plan;                       // one-wave strips x bands
    mpd::TmaPlan pair_plan;                  // the same for lf_pair_kernel
    int ring_overlap = 0;                    // fast steps: ring beside the interior (if ok)
    bool overlap_ok = false;                 // bc_overlap_kernel fits beside the interior
    int overlap_blocks = 0;                  // its grid: at most one block per SM
    bool ring_beside = false;                // the interior just launched left the ring to it
    mpd::TmaPlan pplan;                      // persistent launch (cooperative wave)
    bool persist_ok = false;                 // the persistent engine can run here
    mpd::GridSync *gsync = nullptr;          // its barrier and reduction words
    unsigned long long *red = nullptr;
    mpd::DevState *st = nullptr;
    mpd::DevState *h_st = nullptr;  // pinned mirror
    mpd::DevState *h_ring = nullptr;  // pinned: the state after each in-flight graph launch
    cudaEvent_t ev_ring[2] = {nullptr, nullptr};
    cudaEvent_t ev_end[2] = {nullptr, nullptr};  // timing: end of each in-flight launch's work
    cudaEvent_t ev_stop = nullptr;               // ev_end of the launch the run stopped in
    mpd::HostMirror *hm = nullptr;   // mapped pinned: the controller's per-step outputs
    cudaEvent_t ev_sync = nullptr;   // completion of the enqueued work, for hm
    mpd::SegDesc *d_seg = nullptr;
    int32_t *d_code = nullptr;
    double *d_consts = nullptr;
    mpd::BcTable bc{};
    int precision = MPD_PRECISION_EXACT;
    int with_prev = 0;
    long long host_step = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0, graph_check = 0, graph_resid = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, snap_ev = nullptr, stage_ev = nullptr;
    bool snap_pending = false;
    size_t dev_bytes = 0;
};

namespace {

template <typename T>
int DevAlloc(mpd_solver *s, T **p, size_t count) {
    const size_t bytes = count * sizeof(T);
    MPD_CK(cudaMalloc(reinterpret_cast<void **>(p), bytes));
    s->dev_bytes += bytes;
    return MPD_OK;
}

// Device address of the mapped mirror (null when there is none).
mpd::HostMirror *DeviceMirror(mpd_solver *s) {
    void *d = nullptr;
    if (!s->hm || cudaHostGetDevicePointer(&d, s->hm, 0) != cudaSuccess) return nullptr;
    return static_cast<mpd::HostMirror *>(d);
}

// The mirror's fields from the host copy of the state.
void RefreshMirror(mpd_solver *s) {
    if (!s->hm) return;
    s->hm->step = s->h_st->step;
    s->hm->last_ws = s->h_st->last_ws;
    s->hm->ws_valid = s->h_st->ws_valid;
    s->hm->wait_fail = s->h_st->wait_fail;
}

void FreeAll(mpd_solver *s) {
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->side) cudaStreamSynchronize(s->side);
    if (s->graph) cudaGraphExecDestroy(s->graph);
    cudaFree(s->buf[0]);
    cudaFree(s->buf[1]);
    cudaFree(s->ic);
    cudaFree(s->prev);
    cudaFree(s->geo);
    cudaFree(s->stage);
    cudaFree(s->partials);
    cudaFree(s->cphys);
    cudaFree(s->gsync);
    cudaFree(s->wall[0]);
    cudaFree(s->wall[1]);
    cudaFree(s->small);
    cudaFree(s->red);
    cudaFree(s->st);
    cudaFree(s->d_seg);
    cudaFree(s->d_code);
    cudaFree(s->d_consts);
    if (s->h_st) cudaFreeHost(s->h_st);
    if (s->h_ring) cudaFreeHost(s->h_ring);
    for (cudaEvent_t e : s->ev_end)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : s->ev_ring)
        if (e) cudaEventDestroy(e);
    if (s->hm) cudaFreeHost(s->hm);
    if (s->ev_sync) cudaEventDestroy(s->ev_sync);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->snap_ev) cudaEventDestroy(s->snap_ev);
    if (s->stage_ev) cudaEventDestroy(s->stage_ev);
    if (s->stream) cudaStreamDestroy(s->stream);
    if (s->side) cudaStreamDestroy(s->side);
    delete s;
}

mpd::StateBufs Bufs(const mpd_solver *s) {
    mpd::StateBufs b;
    b.g = s->g;
    b.buf0 = s->buf[0];
    b.buf1 = s->buf[1];
    b.ic = s->ic;
    b.st = s->st;
    return b;
}

// Upload dense host planes (interior only) into pitched device planes and
// rebuild the conserved state (Fields::InitConservative).
int InitFromIc(mpd_solver *s);

// The initial physical planes from the host (NULL: all zero), then InitFromIc.
int UploadPhysical(mpd_solver *s, const double *phys10) {
    const size_t n = static_cast<size_t>(s->rows) * s->cols;
    MPD_CK(cudaMemsetAsync(s->ic, 0, 10 * s->ps * sizeof(double), s->stream));
    if (phys10 && s->stage) {
        // one contiguous copy into the dense staging planes, then the
        // interior cells into the pitched planes on the device
        MPD_CK(cudaMemcpyAsync(s->stage, phys10, 10 * n * sizeof(double), cudaMemcpyHostToDevice,
                               s->stream));
        mpd::scatter_phys_kernel<<<4 * 148, 256, 0, s->stream>>>(s->g, s->stage, s->ic);
        MPD_CK(cudaGetLastError());
        return InitFromIc(s);
    }
    for (int k = 0; phys10 && k < 10; ++k) {
        const double *src = phys10 + k * n + s->cols + 1;  // (l=1, m=1)
        double *dst = s->ic + k * s->ps + s->pitch + 1;
        MPD_CK(cudaMemcpy2DAsync(dst, s->pitch * sizeof(double), src, s->cols * sizeof(double),
                                 (s->M + 1) * sizeof(double), s->L, cudaMemcpyHostToDevice,
                                 s->stream));
    }
    return InitFromIc(s);
}

// Fields::InitConservative, the boundary lines, SavePrev and a fresh
// controller from the initial physical planes in s->ic.
int InitFromIc(mpd_solver *s) {
    MPD_CK(cudaMemsetAsync(s->buf[0], 0, 8 * s->ps * sizeof(double), s->stream));
    MPD_CK(cudaMemsetAsync(s->buf[1], 0, 8 * s->ps * sizeof(double), s->stream));
    mpd::init_conservative_kernel<<<4 * 148, 256, 0, s->stream>>>(s->g, s->ic, s->buf[0]);
    MPD_CK(cudaGetLastError());
    const size_t line_bytes = static_cast<size_t>(10) * s->len * sizeof(double);
    MPD_CK(cudaMemsetAsync(s->cphys, 0, mpd::kCentralLines * 8 * s->len * sizeof(double),
                           s->stream));
    MPD_CK(cudaMemsetAsync(s->wall[1], 0, mpd::kWallLines * line_bytes, s->stream));
    mpd::init_wall_kernel<<<(s->rows + 127) / 128, 128, 0, s->stream>>>(s->g, s->ic, s->wall[0],
                                                                          s->len);
    MPD_CK(cudaGetLastError());
    if (s->with_prev) {
        // Fields::SavePrev after initialisation (src/main.cpp:150-152)
        const int from[7] = {mpd::P_RHO, mpd::P_VZ, mpd::P_VR, mpd::P_VPHI,
                             mpd::P_HZ,  mpd::P_HR, mpd::P_HPHI};
        for (int k = 0; k < 7; ++k)
            MPD_CK(cudaMemcpyAsync(s->prev + k * s->ps, s->ic + from[k] * s->ps,
                                   s->ps * sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
    }
    mpd::DevState init{};
    init.mirror = DeviceMirror(s);
    init.T = INFINITY;
    init.max_steps = LLONG_MAX;
    init.want_ws = 1;
    init.resid_every = 1;
    *s->h_st = init;
    MPD_CK(cudaMemcpyAsync(s->st, s->h_st, sizeof(mpd::DevState), cudaMemcpyHostToDevice,
                           s->stream));
    MPD_CK(cudaStreamSynchronize(s->stream));
    RefreshMirror(s);
    s->host_step = 0;
    return MPD_OK;
}

// One time step: interior kernel, boundary kernel (+ controller), in run mode
// the guarded relative-L2 convergence check and, every residual_every steps,
// the L-inf residual.  want_ws: fuse the maximum
// wave speed (adaptive dt and the per-call ComputeDt need it).
// Interior kernel of fast steps >= 1 on the graph and per-call paths:
// lf_tma_kernel (one point column per lane), or lf_pair_kernel (two) with
// MPD_INTERIOR_PAIR 1; both give the same bits.  Measured on a B200 at
// 1600 x 640 (30 back-to-back launches): 26.3 us one column, 28.4 us pair
// (8 resident warps per SM at 244 registers against 12 at 160).
#ifndef MPD_INTERIOR_PAIR
#define MPD_INTERIOR_PAIR 0
#endif

// alone: launches of the interior kernel with no boundary kernel after them
// (per-kernel timing): the ring-beside form's rows and stores, with the
// next launch let in only once a block's rows are done.
int LaunchInterior(mpd_solver *s, bool first, bool use_state_dt, double dt, bool want_ws,
                   int variant = MPD_INTERIOR_PAIR, bool alone = false) {
    const mpd::Geo &g = s->g;
    const int usd = use_state_dt ? 1 : 0;
    s->ring_beside = false;
    if (first || s->precision == MPD_PRECISION_EXACT) {
        dim3 block(32, 8);
        dim3 grid((g.M - 1 + 31) / 32, (g.L + 7) / 8);
        if (first)
            mpd::lf_exact_kernel<true><<<grid, block, 0, s->stream>>>(
                g, s->buf[0], s->buf[1], s->ic, s->st, dt, usd, s->cphys, s->len);
        else
            mpd::lf_exact_kernel<false><<<grid, block, 0, s->stream>>>(
                g, s->buf[0], s->buf[1], s->ic, s->st, dt, usd, s->cphys, s->len);
    } else if (variant) {
        MPD_CK(mpd::launch_lf_pair(g, s->pair_plan, s->tmap_pair[0], s->tmap_pair[1], s->buf[0],
                                   s->buf[1], s->st, dt, usd, want_ws, s->cphys, s->len,
                                   s->stream));
    } else {
        const bool beside = s->ring_overlap && s->overlap_ok;
        MPD_CK(mpd::launch_lf_tma(g, s->plan, s->tmap[0], s->tmap[1], s->buf[0], s->buf[1],
                                  s->st, dt, usd, want_ws, beside, beside && !alone, s->cphys,
                                  s->len, s->stream));
        s->ring_beside = beside;
    }
    MPD_CK(cudaGetLastError());
    return MPD_OK;
}

int LaunchBoundary(mpd_solver *s, bool use_state_dt, double dt) {
    const int nring = mpd::ring_count(s->g);
    const size_t smem = MPD_BC_SMEM_SEG ? s->bc.nseg_total * sizeof(mpd::SegDesc) : 0;
    if (s->ring_beside) {
        s->ring_beside = false;
        MPD_CK(mpd::launch_pdl(mpd::bc_overlap_kernel, dim3(s->overlap_blocks), dim3(32),
                               s->bc.nseg_total * sizeof(mpd::SegDesc), s->stream, s->g,
                               s->buf[0], s->buf[1], (const double *)s->ic, s->bc, s->st, dt,
                               use_state_dt ? 1 : 0, s->wall[0], s->wall[1], s->len));
        return MPD_OK;
    }
    MPD_CK(mpd::launch_pdl(mpd::bc_kernel, dim3((nring + kBcBlock - 1) / kBcBlock),
                           dim3(kBcBlock), smem, s->stream, s->g, s->buf[0], s->buf[1],
                           (const double *)s->ic, s->bc, s->st, dt, use_state_dt ? 1 : 0,
                           (const double *)s->cphys, s->wall[0], s->wall[1], s->len,
                           s->precision == MPD_PRECISION_FAST ? 1 : 0));
    return MPD_OK;
}

int EnqueueStep(mpd_solver *s, bool first, bool use_state_dt, double dt, bool with_check,
                bool want_ws, bool with_residual) {
    const mpd::Geo &g = s->g;
    int rc = LaunchInterior(s, first, use_state_dt, dt, want_ws);
    if (rc != MPD_OK) return rc;
    rc = LaunchBoundary(s, use_state_dt, dt);
    if (rc != MPD_OK) return rc;
    if (with_check) {
        mpd::change_kernel<<<kRedBlocks, 256, 0, s->stream>>>(Bufs(s), s->prev, s->partials, 1, 1);
        mpd::change_finish_kernel<<<1, 256, 2 * kRedBlocks * sizeof(double), s->stream>>>(
            s->partials, kRedBlocks, s->st, 1);
        MPD_CK(cudaGetLastError());
    }
    if (with_residual) {
        mpd::residual_kernel<<<s->resid_blocks, 256, 0, s->stream>>>(g, s->buf[0], s->buf[1], s->st, 0);
        MPD_CK(cudaGetLastError());
    }
    return MPD_OK;
}

int SyncState(mpd_solver *s) {
    MPD_CK(cudaMemcpyAsync(s->h_st, s->st, sizeof(mpd::DevState), cudaMemcpyDeviceToHost,
                           s->stream));
    MPD_CK(cudaStreamSynchronize(s->stream));
    RefreshMirror(s);
    if (s->h_st->wait_fail)
        return Fail(MPD_ERR_TIMEOUT, "a bounded device wait gave up; the state is not valid");
    return MPD_OK;
}

int PushState(mpd_solver *s) {
    MPD_CK(cudaMemcpyAsync(s->st, s->h_st, sizeof(mpd::DevState), cudaMemcpyHostToDevice,
                           s->stream));
    MPD_CK(cudaStreamSynchronize(s->stream));
    RefreshMirror(s);
    return MPD_OK;
}

int CheckHandle(mpd_solver *s) {
    if (!s) return Fail(MPD_ERR_INVALID, "NULL solver handle");
    MPD_CK(cudaSetDevice(s->device));
    return MPD_OK;
}

int BuildGraph(mpd_solver *s, int steps, bool with_check, bool want_ws, int resid_every) {
    const int key = (with_check ? 1 : 0) | (want_ws ? 2 : 0) | (s->ring_overlap ? 4 : 0);
    if (s->graph && s->graph_steps == steps && s->graph_check == key &&
        s->graph_resid == resid_every)
        return MPD_OK;
    if (s->graph) {
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
    }
    cudaGraph_t graph = nullptr;
    MPD_CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int rc = MPD_OK;
    for (int i = 0; i < steps && rc == MPD_OK; ++i) {
        const bool res = resid_every > 0 && (i + 1) % resid_every == 0;
        rc = EnqueueStep(s, false, true, 0.0, with_check, want_ws, res);
    }
    const cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
    if (rc != MPD_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return Fail(MPD_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    const cudaError_t e2 = cudaGraphInstantiate(&s->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) return Fail(MPD_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e2));
    s->graph_steps = steps;
    s->graph_check = key;
    s->graph_resid = resid_every;
    return MPD_OK;
}

__global__ void fast_math_kernel(const double *x, long long n, double *rcp, double *sqr) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        rcp[i] = mpd::rcp_nr(x[i]);
        sqr[i] = mpd::sqrt_nr(x[i]);
    }
}

}  // namespace

extern "C" {

int mpd_fast_math(const double *d_x, long long n, double *d_rcp, double *d_sqrt, void *stream) {
    if (!d_x || !d_rcp || !d_sqrt || n < 0) return Fail(MPD_ERR_INVALID, "mpd_fast_math: bad arguments");
    if (n == 0) return MPD_OK;
    long long blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    fast_math_kernel<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_x, n, d_rcp,
                                                                                     d_sqrt);
    MPD_CK(cudaGetLastError());
    return MPD_OK;
}

const char *mpd_last_error(void) { return mpd::g_last_error.c_str(); }

int mpd_create(const mpd_config *cfg, const mpd_geometry *geom, const double *phys10,
               mpd_solver **out) {
    std::string err;
    if (!out) return Fail(MPD_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int rc = mpd::ValidateConfig(cfg, geom, err);
    if (rc != MPD_OK) return Fail(rc, err);
    if (!geom) return Fail(MPD_ERR_INVALID, "geometry is required");
    mpd::CompiledBc cbc;
    rc = mpd::CompileBc(*cfg, cbc, err);
    if (rc != MPD_OK) return Fail(rc, err);

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return Fail(MPD_ERR_NO_DEVICE, "no CUDA device available");

    auto *s = new mpd_solver();
    MPD_CK(cudaGetDevice(&s->device));
    s->L = cfg->L_max;
    s->M = cfg->M_max;
    s->rows = s->L + 2;
    s->cols = s->M + 3;
    s->pitch = (s->cols + 31) / 32 * 32;
    s->ps = static_cast<size_t>(s->rows) * s->pitch;
    s->precision = cfg->precision;
    s->with_prev = cfg->with_prev ? 1 : 0;

#define STEP(x)               \
    do {                      \
        const int rc_ = (x);  \
        if (rc_ != MPD_OK) {  \
            FreeAll(s);       \
            return rc_;       \
        }                     \
    } while (0)

    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&s->ev0) != cudaSuccess || cudaEventCreate(&s->ev1) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->snap_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->stage_ev, cudaEventDisableTiming) != cudaSuccess) {
        FreeAll(s);
        return Fail(MPD_ERR_CUDA, "stream/event creation failed");
    }
    STEP(DevAlloc(s, &s->buf[0], 8 * s->ps));
    STEP(DevAlloc(s, &s->buf[1], 8 * s->ps));
    STEP(DevAlloc(s, &s->ic, 10 * s->ps));
    if (s->with_prev) STEP(DevAlloc(s, &s->prev, 7 * s->ps));
    STEP(DevAlloc(s, &s->geo, 6 * static_cast<size_t>(s->rows)));
    STEP(DevAlloc(s, &s->partials, static_cast<size_t>(kRedBlocks) * 8));
    s->len = mpd::line_len(s->L, s->M);
    STEP(DevAlloc(s, &s->cphys, static_cast<size_t>(mpd::kCentralLines) * 8 * s->len));
    STEP(DevAlloc(s, &s->wall[0], static_cast<size_t>(mpd::kWallLines) * 10 * s->len));
    STEP(DevAlloc(s, &s->wall[1], static_cast<size_t>(mpd::kWallLines) * 10 * s->len));
    STEP(DevAlloc(s, &s->small, 16));
    STEP(DevAlloc(s, &s->red, 4));
    STEP(DevAlloc(s, &s->st, 1));
    if (cudaMallocHost(reinterpret_cast<void **>(&s->h_st), sizeof(mpd::DevState)) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void **>(&s->h_ring), 2 * sizeof(mpd::DevState)) !=
            cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_ring[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_ring[1], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&s->ev_end[0]) != cudaSuccess || cudaEventCreate(&s->ev_end[1]) != cudaSuccess ||
        cudaHostAlloc(reinterpret_cast<void **>(&s->hm), sizeof(mpd::HostMirror),
                      cudaHostAllocMapped) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_sync, cudaEventDisableTiming) != cudaSuccess) {
        FreeAll(s);
        return Fail(MPD_ERR_NOMEM, "pinned allocation failed");
    }
    std::memset(s->hm, 0, sizeof(mpd::HostMirror));
    // wall profiles + dr (Grid::Build: R = r_outer - r_inner, dr = R / M_max)
    {
        std::vector<double> h(6 * static_cast<size_t>(s->rows));
        for (int l = 0; l < s->rows; ++l) {
            h[0 * s->rows + l] = geom->r_inner[l];
            h[1 * s->rows + l] = geom->r_outer[l];
            h[2 * s->rows + l] = geom->dr_inner_dz[l];
            h[3 * s->rows + l] = geom->dr_outer_dz[l];
            const double R = geom->r_outer[l] - geom->r_inner[l];
            h[4 * s->rows + l] = R / cfg->M_max;
            h[5 * s->rows + l] = 0.5 / h[4 * s->rows + l];
        }
        if (cudaMemcpy(s->geo, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice) !=
            cudaSuccess) {
            FreeAll(s);
            return Fail(MPD_ERR_CUDA, "geometry upload failed");
        }
    }
    mpd::Geo &g = s->g;
    g.L = s->L;
    g.M = s->M;
    g.pitch = s->pitch;
    g.ps = s->ps;
    g.dz = cfg->dz;
    g.dy = cfg->dy;
    g.gamma = cfg->gamma;
    g.beta = cfg->beta;
    g.H_z0 = cfg->H_z0;
    g.r_0 = cfg->r_0;
    g.rin = s->geo;
    g.rout = s->geo + s->rows;
    g.drin = s->geo + 2 * s->rows;
    g.drout = s->geo + 3 * s->rows;
    g.dr = s->geo + 4 * s->rows;
    g.hdr = s->geo + 5 * s->rows;
    {
        int sms = 0, per_sm = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mpd::residual_kernel, 256, 0) !=
                cudaSuccess) {
            FreeAll(s);
            return Fail(MPD_ERR_CUDA, "occupancy query for the residual kernel failed");
        }
        s->resid_blocks = sms * (per_sm > 0 ? per_sm : 1);
    }
    if (s->precision == MPD_PRECISION_FAST) {
        for (int b = 0; b < 2; ++b)
            STEP(EncodeStateMap(&s->tmap[b], s->buf[b], s->cols, s->rows, s->pitch, s->ps, 32));
        for (int b = 0; b < 2; ++b)
            STEP(EncodeStateMap(&s->tmap_pair[b], s->buf[b], s->cols, s->rows, s->pitch, s->ps,
                                64));
        if (mpd::plan_lf_tma(g, s->device, s->plan) != cudaSuccess ||
            mpd::plan_lf_pair(g, s->device, s->pair_plan) != cudaSuccess) {
            FreeAll(s);
            return Fail(MPD_ERR_CUDA, "occupancy query for the interior kernel failed");
        }
        {
            // the ring beside the interior: rows 2..L-1 must exist; one block
            // of one warp per SM at most, striding over the ring slots
            int sms = 0;
            if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device) !=
                cudaSuccess) {
                FreeAll(s);
                return Fail(MPD_ERR_CUDA, "device query failed");
            }
            const int groups = (mpd::ring_count(g) + 31) / 32;
            s->overlap_blocks = groups < sms ? groups : sms;
            s->overlap_ok = g.L >= 4 && s->overlap_blocks > 0;
        }
        // the persistent engine needs cooperative launch and a strip per warp
        s->persist_ok = mpd::plan_lf_persist(g, s->device, s->pplan) == cudaSuccess;
        cudaGetLastError();
        if (s->persist_ok) STEP(DevAlloc(s, &s->gsync, 1));
    }
    // boundary table
    STEP(DevAlloc(s, &s->d_seg, cbc.seg.size() ? cbc.seg.size() : 1));
    STEP(DevAlloc(s, &s->d_code, cbc.code.size()));
    STEP(DevAlloc(s, &s->d_consts, cbc.consts.size()));
    if ((!cbc.seg.empty() &&
         cudaMemcpy(s->d_seg, cbc.seg.data(), cbc.seg.size() * sizeof(mpd::SegDesc),
                    cudaMemcpyHostToDevice) != cudaSuccess) ||
        cudaMemcpy(s->d_code, cbc.code.data(), cbc.code.size() * sizeof(int32_t),
                   cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->d_consts, cbc.consts.data(), cbc.consts.size() * sizeof(double),
                   cudaMemcpyHostToDevice) != cudaSuccess) {
        FreeAll(s);
        return Fail(MPD_ERR_CUDA, "boundary table upload failed");
    }
    for (int f = 0; f < 4; ++f) {
        s->bc.nseg[f] = cbc.nseg[f];
        s->bc.first[f] = cbc.first[f];
    }
    s->bc.seg = s->d_seg;
    s->bc.code = s->d_code;
    s->bc.consts = s->d_consts;
    s->bc.nseg_total = static_cast<int>(cbc.seg.size());
    s->bc.ncode = static_cast<int>(cbc.code.size());
    s->bc.nconst = static_cast<int>(cbc.consts.size());
    STEP(UploadPhysical(s, phys10));
#undef STEP
    *out = s;
    return MPD_OK;
}

void mpd_destroy(mpd_solver *s) {
    if (!s) return;
    cudaSetDevice(s->device);
    FreeAll(s);
}

int mpd_advance(mpd_solver *s, double dt) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    rc = EnqueueStep(s, s->host_step == 0, false, dt, false, true, false);
    if (rc != MPD_OK) return rc;
    s->host_step++;
    return MPD_OK;
}

// End of mpd_run: device time, the final residual, stats, and back to per-call mode.
static int FinishRun(mpd_solver *s, long long step0, mpd_run_stats *stats) {
    mpd::DevState &h = *s->h_st;
    int rc = MPD_OK;
    // device time: to the end of the graph launch the run stopped in (the
    // host learns of the stop only later, through the launch's state copy),
    // else to an event recorded now (the persistent engine)
    cudaEvent_t end = s->ev_stop;
    s->ev_stop = nullptr;
    if (!end) {
        MPD_CK(cudaEventRecord(s->ev1, s->stream));
        end = s->ev1;
    }
    MPD_CK(cudaEventSynchronize(end));
    float ms = 0.f;
    MPD_CK(cudaEventElapsedTime(&ms, s->ev0, end));
    rc = SyncState(s);  // the loop read the controller through its own slots
    if (rc != MPD_OK) return rc;
    // the residual of the final state, when the loop stopped between checks
    if (!h.resid_valid && h.step > 0) {
        mpd::residual_kernel<<<s->resid_blocks, 256, 0, s->stream>>>(s->g, s->buf[0], s->buf[1], s->st, 0);
        MPD_CK(cudaGetLastError());
    }
    rc = SyncState(s);
    if (rc != MPD_OK) return rc;
    if (stats) {
        stats->steps = h.step - step0;
        stats->t = h.t;
        stats->dt = h.dt;
        stats->residual = h.resid_valid ? h.last_resid : NAN;
        stats->change = h.last_change;
        stats->max_wave_speed = h.last_ws;
        stats->converged = h.converged;
        stats->status = h.nonfinite ? MPD_ERR_NONFINITE : MPD_OK;
        stats->device_ms = ms;
    }
    s->host_step = h.step;
    const bool nonfinite = h.nonfinite != 0;
    // back to drop-in (per-call) mode
    h.run_mode = 0;
    h.done = 0;
    h.want_ws = 1;
    h.resid_every = 1;
    h.T = INFINITY;
    h.max_steps = LLONG_MAX;
    rc = PushState(s);
    if (rc != MPD_OK) return rc;
    if (nonfinite) return Fail(MPD_ERR_NONFINITE, "non-finite value in the state");
    return MPD_OK;
}

// mpd_run's checks of the run parameters.
static int CheckRunParams(const mpd_solver *s, const mpd_run_params *p) {
    if (!p) return Fail(MPD_ERR_INVALID, "run params are NULL");
    if (p->convergence_threshold > 0.0 && !s->with_prev)
        return Fail(MPD_ERR_INVALID, "convergence_threshold > 0 needs a solver created with with_prev");
    if (p->convergence_threshold > 0.0 && p->check_frequency <= 0)
        return Fail(MPD_ERR_INVALID, "check_frequency must be positive");
    if (p->max_steps <= 0) return Fail(MPD_ERR_INVALID, "max_steps must be positive");
    if (p->residual_every < 0 || p->residual_every > 4096)
        return Fail(MPD_ERR_INVALID, "residual_every must be in [0, 4096]");
    if (p->monitor_every < 0) return Fail(MPD_ERR_INVALID, "monitor_every must be >= 0");
    if (p->monitor && p->monitor_every > 0 && p->engine == MPD_ENGINE_PERSISTENT)
        return Fail(MPD_ERR_INVALID, "monitor reports need the graph engine");
    return MPD_OK;
}

// Put the device controller into run mode for `p` (the driver loop's state,
// src/main.cpp:191-223, including the first T clamp).  step0 = step at entry.
static int PrepareRun(mpd_solver *s, const mpd_run_params *p, long long &step0) {
    // dt <= 0: start at the CFL limit of the current state (a warm start that
    // begins at the step the steady state was converged with)
    double ws0 = 0.0;
    if (!(p->dt > 0.0)) {
        const int rw = mpd_max_wave_speed(s, &ws0);
        if (rw != MPD_OK) return rw;
    }
    int rc = SyncState(s);
    if (rc != MPD_OK) return rc;
    mpd::DevState &h = *s->h_st;
    step0 = h.step;
    h.run_mode = 1;
    h.adaptive = p->adaptive ? 1 : 0;
    h.want_ws = p->adaptive ? 1 : 0;
    h.cfl = p->cfl_number;
    h.growth = p->dt_growth_factor;
    h.dt_min = p->dt_min;
    h.dt_max = p->dt_max;
    h.T = p->T;
    h.max_steps = step0 + p->max_steps;
    if (p->monitor && p->monitor_every > 0) {
        // the loop stops at every multiple of monitor_every for a report
        const long long next = (step0 / p->monitor_every + 1) * p->monitor_every;
        if (next < h.max_steps) h.max_steps = next;
    }
    h.resid_tol = p->residual_tol;
    h.resid_every = p->residual_every > 0 ? p->residual_every : 0;
    h.conv_thr = p->convergence_threshold;
    h.check_freq = p->check_frequency;
    h.check_due = 0;
    h.done = 0;
    h.converged = 0;
    h.nonfinite = 0;
    h.t0_ns = 0ull;
    h.done_ns = 0ull;
    double dt = p->dt;
    if (!(dt > 0.0)) {
        const double dx = s->g.dy < s->g.dz ? s->g.dy : s->g.dz;
        dt = p->cfl_number * dx / (ws0 + 1.0e-10);
        dt = dt < p->dt_min ? p->dt_min : (dt > p->dt_max ? p->dt_max : dt);
    }
    if (h.t + dt > h.T) dt = h.T - h.t;  // src/main.cpp:221-223
    h.dt = dt;
    if (!(h.t < h.T)) h.done = 1;
    return PushState(s);
}

// Arguments of the persistent loops for solver s, with a team of `blocks`.
static mpd::PersistArgs PersistArgsOf(const mpd_solver *s, int nstrips, int nbands,
                                      long long nsteps, long long resid_base) {
    mpd::PersistArgs a{};
    a.g = s->g;
    a.buf0 = s->buf[0];
    a.buf1 = s->buf[1];
    a.cphys = s->cphys;
    a.wall0 = s->wall[0];
    a.wall1 = s->wall[1];
    a.len = s->len;
    a.bc = s->bc;
    a.st = s->st;
    a.nstrips = nstrips;
    a.nbands = nbands;
    a.nsteps = nsteps;
    a.resid_base = resid_base;
    return a;
}

// Graph launches until the device controller stops, taking at most `budget`
// steps.  Two launches are kept in flight: after each launch the controller
// state is copied into a pinned slot, and the host reads the older slot while
// the newer launch runs, so the device never waits for the host between
// launches.  Every stop criterion is evaluated on the device (a launch after
// the stop exits at once); launches are capped at the budget, so a fixed-step
// run queues no launch past its last step.
static int GraphLoop(mpd_solver *s, long long budget, int per_graph) {
    const long long cap = budget <= 0 ? 0 : (budget + per_graph - 1) / per_graph;
    if (cap == 0) return MPD_OK;
    long long launched = 0;
    int pending = 0;
    auto launch = [&](int slot) -> int {
        MPD_CK(cudaGraphLaunch(s->graph, s->stream));
        MPD_CK(cudaEventRecord(s->ev_end[slot], s->stream));
        MPD_CK(cudaMemcpyAsync(&s->h_ring[slot], s->st, sizeof(mpd::DevState),
                               cudaMemcpyDeviceToHost, s->stream));
        MPD_CK(cudaEventRecord(s->ev_ring[slot], s->stream));
        ++launched;
        ++pending;
        return MPD_OK;
    };
    int rc = MPD_OK;
    for (int slot = 0; slot < 2 && launched < cap; ++slot) {
        rc = launch(slot);
        if (rc != MPD_OK) return rc;
    }
    long long last_step = -1;
    for (int slot = 0; pending > 0; slot ^= 1) {
        MPD_CK(cudaEventSynchronize(s->ev_ring[slot]));
        --pending;
        const mpd::DevState &r = s->h_ring[slot];
        if (r.wait_fail) {
            MPD_CK(cudaStreamSynchronize(s->stream));
            return Fail(MPD_ERR_TIMEOUT, "a bounded device wait gave up; the state is not valid");
        }
        if (r.done) {  // a launch still in flight exits at once
            s->ev_stop = s->ev_end[slot];
            return MPD_OK;
        }
        if (r.step == last_step) {  // a launch that advanced nothing: stop, don't spin
            MPD_CK(cudaStreamSynchronize(s->stream));
            return Fail(MPD_ERR_TIMEOUT, "run loop made no progress");
        }
        last_step = r.step;
        if (launched < cap) {
            rc = launch(slot);
            if (rc != MPD_OK) return rc;
        }
    }
    MPD_CK(cudaStreamSynchronize(s->stream));
    return Fail(MPD_ERR_TIMEOUT, "run loop ended before the device controller stopped");
}

// The driver loop's periodic report (src/main.cpp:249-281) of the current
// state, handed to the run's monitor callback.  s->h_st is current.
static int Monitor(mpd_solver *s, const mpd_run_params *p) {
    const mpd::DevState h = *s->h_st;
    mpd_monitor_record rec{};
    rec.step = h.step;
    rec.t = h.t;
    rec.dt = h.dt;
    double speed = 0.0;
    if (h.ws_valid && h.step > 0) {
        speed = h.last_ws;
    } else {
        MPD_CK(cudaMemsetAsync(s->red, 0, 2 * sizeof(unsigned long long), s->stream));
        mpd::wave_speed_kernel<<<kRedBlocks, 256, 0, s->stream>>>(Bufs(s), s->red);
        MPD_CK(cudaGetLastError());
        unsigned long long key = 0;
        MPD_CK(cudaMemcpyAsync(&key, s->red, sizeof(key), cudaMemcpyDeviceToHost, s->stream));
        MPD_CK(cudaStreamSynchronize(s->stream));
        std::memcpy(&speed, &key, sizeof(double));
    }
    // Diagnostics::CheckCfl (src/diagnostics.cpp:112-125)
    const double dx = s->g.dz < s->g.dy ? s->g.dz : s->g.dy;
    rec.max_wave_speed = speed;
    rec.dt_cfl = p->cfl_number * dx / (speed + 1.0e-10);
    rec.cfl_warning = h.dt > rec.dt_cfl ? 1 : 0;
    // the checkpoint cell (global l 20, m 40) when the grid has it
    constexpr int kProbeL = 20, kProbeM = 40;
    if (kProbeL < s->L && kProbeM <= s->M) {
        double q[10];
        int rc = mpd_probe(s, kProbeL, kProbeM, q);
        if (rc != MPD_OK) return rc;
        rec.probe[0] = q[0];  // rho
        rec.probe[1] = q[1];  // v_z
        rec.probe[2] = q[3];  // v_phi
        rec.probe[3] = q[4];  // e
        rec.probe[4] = q[9];  // H_phi
    }
    int rc = mpd_integrals(s, rec.integrals);
    if (rc != MPD_OK) return rc;
    p->monitor(&rec, p->monitor_user);
    return MPD_OK;
}

int mpd_run(mpd_solver *s, const mpd_run_params *p, mpd_run_stats *stats) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    rc = CheckRunParams(s, p);
    if (rc != MPD_OK) return rc;
    const bool with_check = p->convergence_threshold > 0.0;
    const bool want_ws = p->adaptive != 0;
    long long step0 = 0;
    rc = PrepareRun(s, p, step0);
    if (rc != MPD_OK) return rc;
    mpd::DevState &h = *s->h_st;

    s->ev_stop = nullptr;
    MPD_CK(cudaEventRecord(s->ev0, s->stream));
    if (!h.done && s->host_step == 0) {
        rc = EnqueueStep(s, true, true, 0.0, with_check, want_ws, p->residual_every == 1);
        if (rc != MPD_OK) return rc;
    }
    if (p->engine == MPD_ENGINE_PERSISTENT && (!s->persist_ok || with_check))
        return Fail(MPD_ERR_INVALID,
                    "the persistent engine needs fast precision, cooperative launch and no "
                    "convergence_threshold");
    // AUTO takes the graph path: on the measured workloads it is the faster one
    // (the persistent engine pays two grid barriers per step and runs the
    // boundary chains of every face inside one phase)
    if (p->engine == MPD_ENGINE_PERSISTENT) {
        // one cooperative launch per chunk of steps; the residual keeps the
        // graph path's schedule: after steps (step - base) % residual_every == 0
        const mpd::PersistArgs a =
            PersistArgsOf(s, s->pplan.nstrips, s->pplan.nbands, 2000,
                          step0 + ((!h.done && s->host_step == 0) ? 1 : 0));
        long long last = -1;
        for (;;) {
            MPD_CK(cudaMemcpyAsync(s->h_st, s->st, sizeof(mpd::DevState), cudaMemcpyDeviceToHost,
                                   s->stream));
            MPD_CK(cudaStreamSynchronize(s->stream));
            if (h.wait_fail)
                return Fail(MPD_ERR_TIMEOUT, "a bounded device wait gave up; the state is not valid");
            if (h.done) break;
            if (h.step == last) return Fail(MPD_ERR_TIMEOUT, "run loop made no progress");
            last = h.step;
            MPD_CK(cudaMemsetAsync(s->gsync, 0, sizeof(mpd::GridSync), s->stream));
            MPD_CK(mpd::launch_lf_persist(s->pplan, s->tmap[0], s->tmap[1], a, s->gsync,
                                          s->stream));
        }
        return FinishRun(s, step0, stats);
    }
    const bool monitored = p->monitor && p->monitor_every > 0;
    // Steps per graph launch: a multiple of the residual interval, so that the
    // residual is evaluated every residual_every steps; with monitor reports,
    // a divisor of monitor_every where the residual interval allows.
    int per_graph = p->steps_per_graph > 0 ? p->steps_per_graph : 100;
    if (monitored && p->monitor_every % per_graph != 0) {
        int a = per_graph, b = p->monitor_every;
        while (b) {
            const int r = a % b;
            a = b;
            b = r;
        }
        per_graph = a;
    }
    if (with_check && p->check_frequency > 0 && per_graph % p->check_frequency != 0 &&
        p->check_frequency < per_graph)
        per_graph = (per_graph / p->check_frequency) * p->check_frequency;
    if (p->residual_every > 0 && per_graph % p->residual_every != 0)
        per_graph = (per_graph / p->residual_every + 1) * p->residual_every;
    rc = BuildGraph(s, per_graph, with_check, want_ws, p->residual_every);
    if (rc != MPD_OK) return rc;
    long long taken_before = (!h.done && s->host_step == 0) ? 1 : 0;  // the exact first step
    const long long end = step0 + p->max_steps;
    for (;;) {
        // steps this segment may take: to the controller's current stop
        long long budget = h.max_steps - h.step - taken_before;
        taken_before = 0;
        rc = GraphLoop(s, h.done ? 0 : budget, per_graph);
        if (rc != MPD_OK) return rc;
        if (!monitored) break;
        rc = SyncState(s);
        if (rc != MPD_OK) return rc;
        if (h.converged || h.nonfinite || !(h.t < h.T) || h.step >= end) {
            if (h.step % p->monitor_every == 0 && h.step > step0) {
                rc = Monitor(s, p);
                if (rc != MPD_OK) return rc;
            }
            break;
        }
        if (h.step % p->monitor_every == 0) {
            rc = Monitor(s, p);
            if (rc != MPD_OK) return rc;
        }
        // next segment: to the next report or the end of the run
        const long long next = (h.step / p->monitor_every + 1) * p->monitor_every;
        h.max_steps = next < end ? next : end;
        h.done = 0;
        rc = PushState(s);
        if (rc != MPD_OK) return rc;
    }
    return FinishRun(s, step0, stats);
}

int mpd_max_wave_speed(mpd_solver *s, double *out) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    if (!out) return Fail(MPD_ERR_INVALID, "out is NULL");
    if (s->hm) {
        // after a step the controller has left the speed in the mapped
        // mirror, the step number last: watch that word for the step this
        // handle issued last (its controller's final write), no copy of the
        // whole state; after 100 ms without it, wait for the stream instead
        const volatile mpd::HostMirror *m = s->hm;
        const long long want = s->host_step;
        bool seen = false;
        if (want > 0) {
            const auto t0 = std::chrono::steady_clock::now();
            for (long long spins = 0;; ++spins) {
                if (m->step >= want || m->wait_fail) {
                    seen = true;
                    break;
                }
                if ((spins & 1023) == 1023 &&
                    std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(100))
                    break;
            }
            std::atomic_thread_fence(std::memory_order_acquire);
        }
        if (!seen) {
            MPD_CK(cudaEventRecord(s->ev_sync, s->stream));
            MPD_CK(cudaEventSynchronize(s->ev_sync));
        }
        if (m->wait_fail)
            return Fail(MPD_ERR_TIMEOUT, "a bounded device wait gave up; the state is not valid");
        if (m->ws_valid && m->step > 0) {
            *out = m->last_ws;
            return MPD_OK;
        }
    }
    rc = SyncState(s);
    if (rc != MPD_OK) return rc;
    if (s->h_st->ws_valid && s->h_st->step > 0) {
        *out = s->h_st->last_ws;
        return MPD_OK;
    }
    MPD_CK(cudaMemsetAsync(s->red, 0, 2 * sizeof(unsigned long long), s->stream));
    mpd::wave_speed_kernel<<<kRedBlocks, 256, 0, s->stream>>>(Bufs(s), s->red);
    MPD_CK(cudaGetLastError());
    unsigned long long key = 0;
    MPD_CK(cudaMemcpyAsync(&key, s->red, sizeof(key), cudaMemcpyDeviceToHost, s->stream));
    MPD_CK(cudaStreamSynchronize(s->stream));
    std::memcpy(out, &key, sizeof(double));
    return MPD_OK;
}

int mpd_compute_dt(mpd_solver *s, double cfl_number, double growth, double dt_min, double dt_max,
                   double dt_current, double *dt_next) {
    double speed = 0.0;
    const int rc = mpd_max_wave_speed(s, &speed);
    if (rc != MPD_OK) return rc;
    if (!dt_next) return Fail(MPD_ERR_INVALID, "dt_next is NULL");
    *dt_next = mpd::compute_dt_from_speed(speed, s->g.dz, s->g.dy, cfl_number, growth, dt_min,
                                          dt_max, dt_current);
    return MPD_OK;
}

static int ChangeImpl(mpd_solver *s, int save, double *out) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    if (!s->with_prev) return Fail(MPD_ERR_INVALID, "solver was created without prev planes");
    mpd::change_kernel<<<kRedBlocks, 256, 0, s->stream>>>(Bufs(s), s->prev, s->partials, save, 0);
    mpd::change_finish_kernel<<<1, 256, 2 * kRedBlocks * sizeof(double), s->stream>>>(
        s->partials, kRedBlocks, s->st, 0);
    MPD_CK(cudaGetLastError());
    rc = SyncState(s);
    if (rc != MPD_OK) return rc;
    if (out) *out = s->h_st->last_change;
    return MPD_OK;
}

int mpd_solution_change(mpd_solver *s, double *out) {
    if (!out) return Fail(MPD_ERR_INVALID, "out is NULL");
    return ChangeImpl(s, 0, out);
}

int mpd_save_prev(mpd_solver *s) { return ChangeImpl(s, 1, nullptr); }

int mpd_integrals(mpd_solver *s, double out7[7]) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    if (!out7) return Fail(MPD_ERR_INVALID, "out is NULL");
    const int nb = s->L < kRedBlocks ? s->L : kRedBlocks;
    mpd::integrals_kernel<<<nb, 256, 0, s->stream>>>(Bufs(s), s->partials);
    mpd::sum_partials_kernel<7><<<1, 256, 7 * nb * sizeof(double), s->stream>>>(s->partials, nb,
                                                                               s->small);
    MPD_CK(cudaGetLastError());
    MPD_CK(cudaMemcpyAsync(out7, s->small, 7 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    MPD_CK(cudaStreamSynchronize(s->stream));
    return MPD_OK;
}

int mpd_outlet(mpd_solver *s, double *mass_flux, double *thrust) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    if (!mass_flux || !thrust) return Fail(MPD_ERR_INVALID, "out is NULL");
    const double inv_8pi = 1.0 / (8.0 * M_PI);
    mpd::outlet_kernel<<<1, mpd::kOutletThreads, 0, s->stream>>>(Bufs(s), inv_8pi, s->small);
    MPD_CK(cudaGetLastError());
    double h[2];
    MPD_CK(cudaMemcpyAsync(h, s->small, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    MPD_CK(cudaStreamSynchronize(s->stream));
    *mass_flux = h[0];
    *thrust = h[1];
    return MPD_OK;
}

int mpd_radial_symmetry(mpd_solver *s, double *out) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    if (!out) return Fail(MPD_ERR_INVALID, "out is NULL");
    MPD_CK(cudaMemsetAsync(s->red, 0, 2 * sizeof(unsigned long long), s->stream));
    mpd::radial_kernel<<<kRedBlocks, 256, 0, s->stream>>>(Bufs(s), s->red);
    MPD_CK(cudaGetLastError());
    unsigned long long key = 0;
    MPD_CK(cudaMemcpyAsync(&key, s->red, sizeof(key), cudaMemcpyDeviceToHost, s->stream));
    MPD_CK(cudaStreamSynchronize(s->stream));
    std::memcpy(out, &key, sizeof(double));
    return MPD_OK;
}

int mpd_residual(mpd_solver *s, double *out) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    if (!out) return Fail(MPD_ERR_INVALID, "out is NULL");
    mpd::residual_kernel<<<s->resid_blocks, 256, 0, s->stream>>>(s->g, s->buf[0], s->buf[1], s->st, 0);
    MPD_CK(cudaGetLastError());
    rc = SyncState(s);
    if (rc != MPD_OK) return rc;
    *out = (s->h_st->step > 0 && s->h_st->resid_valid) ? s->h_st->last_resid : NAN;
    return MPD_OK;
}

int mpd_time(mpd_solver *s, double *t, long long *step) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    rc = SyncState(s);
    if (rc != MPD_OK) return rc;
    if (t) *t = s->h_st->t;
    if (step) *step = s->h_st->step;
    return MPD_OK;
}

static int MaterialisePhysical(mpd_solver *s) {
    if (!s->stage) {
        int rc = DevAlloc(s, &s->stage, 10 * static_cast<size_t>(s->rows) * s->cols);
        if (rc != MPD_OK) return rc;
    }
    if (s->snap_pending) MPD_CK(cudaStreamWaitEvent(s->stream, s->snap_ev, 0));
    mpd::phys_planes_kernel<<<4 * 148, 256, 0, s->stream>>>(Bufs(s), s->stage);
    MPD_CK(cudaGetLastError());
    return MPD_OK;
}

int mpd_download(mpd_solver *s, int which, double *host_plane) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    if (!host_plane || which < 0 || which > 17) return Fail(MPD_ERR_INVALID, "bad download request");
    const double *src;
    if (which < 8) {
        rc = SyncState(s);
        if (rc != MPD_OK) return rc;
        src = s->buf[s->h_st->step & 1] + which * s->ps;
    } else {
        rc = MaterialisePhysical(s);
        if (rc != MPD_OK) return rc;
        src = s->stage + (which - 8) * static_cast<size_t>(s->rows) * s->cols;
        // the staging planes are dense: one contiguous copy
        MPD_CK(cudaMemcpyAsync(host_plane, src,
                               static_cast<size_t>(s->rows) * s->cols * sizeof(double),
                               cudaMemcpyDeviceToHost, s->stream));
        MPD_CK(cudaStreamSynchronize(s->stream));
        return MPD_OK;
    }
    MPD_CK(cudaMemcpy2DAsync(host_plane, s->cols * sizeof(double), src, s->pitch * sizeof(double),
                             s->cols * sizeof(double), s->rows, cudaMemcpyDeviceToHost, s->stream));
    MPD_CK(cudaStreamSynchronize(s->stream));
    return MPD_OK;
}

int mpd_probe(mpd_solver *s, int l_global, int m_global, double out10[10]) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    if (!out10 || l_global < 0 || l_global >= s->L || m_global < 0 || m_global > s->M)
        return Fail(MPD_ERR_INVALID, "probe cell out of range");
    rc = SyncState(s);
    if (rc != MPD_OK) return rc;
    const int l = l_global + 1, m = m_global + 1;
    const size_t i = static_cast<size_t>(l) * s->pitch + m;
    if (s->h_st->step == 0) {
        for (int k = 0; k < 10; ++k)
            MPD_CK(cudaMemcpy(out10 + k, s->ic + k * s->ps + i, sizeof(double), cudaMemcpyDeviceToHost));
        return MPD_OK;
    }
    double u[8], geo[2];
    const double *cur = s->buf[s->h_st->step & 1];
    for (int k = 0; k < 8; ++k)
        MPD_CK(cudaMemcpy(u + k, cur + k * s->ps + i, sizeof(double), cudaMemcpyDeviceToHost));
    MPD_CK(cudaMemcpy(&geo[0], s->g.rin + l, sizeof(double), cudaMemcpyDeviceToHost));
    MPD_CK(cudaMemcpy(&geo[1], s->g.rout + l, sizeof(double), cudaMemcpyDeviceToHost));
    const double frac = (double)(m - 1) * s->g.dy;
    const double r = (1.0 - frac) * geo[0] + frac * geo[1];
    const mpd::Phys q = mpd::recon_exact(u, r, s->g.gamma);
    const double v[10] = {q.rho, q.vz, q.vr, q.vphi, q.e, q.p, q.P, q.Hz, q.Hr, q.Hphi};
    std::memcpy(out10, v, sizeof(v));
    return MPD_OK;
}

int mpd_snapshot_async(mpd_solver *s, double *pinned_phys10) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    if (!pinned_phys10) return Fail(MPD_ERR_INVALID, "snapshot buffer is NULL");
    rc = MaterialisePhysical(s);
    if (rc != MPD_OK) return rc;
    MPD_CK(cudaEventRecord(s->stage_ev, s->stream));
    MPD_CK(cudaStreamWaitEvent(s->side, s->stage_ev, 0));
    const size_t n = static_cast<size_t>(s->rows) * s->cols;
    MPD_CK(cudaMemcpyAsync(pinned_phys10, s->stage, 10 * n * sizeof(double),
                           cudaMemcpyDeviceToHost, s->side));
    MPD_CK(cudaEventRecord(s->snap_ev, s->side));
    s->snap_pending = true;
    return MPD_OK;
}

int mpd_snapshot_wait(mpd_solver *s) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    if (s->snap_pending) MPD_CK(cudaEventSynchronize(s->snap_ev));
    s->snap_pending = false;
    return MPD_OK;
}

int mpd_set_physical(mpd_solver *s, const double *phys10) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    if (!phys10) return Fail(MPD_ERR_INVALID, "phys10 is NULL");
    MPD_CK(cudaStreamSynchronize(s->stream));
    if (s->snap_pending) MPD_CK(cudaEventSynchronize(s->snap_ev));
    s->snap_pending = false;
    if (!s->stage) {  // the dense staging planes of the contiguous upload
        rc = DevAlloc(s, &s->stage, 10 * static_cast<size_t>(s->rows) * s->cols);
        if (rc != MPD_OK) return rc;
    }
    return UploadPhysical(s, phys10);
}

int mpd_set_expression_ic(mpd_solver *s, const char *const exprs[8], int n_vars,
                          const char *const *var_names, const double *var_values) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    if (n_vars < 0 || (n_vars > 0 && (!var_names || !var_values)))
        return Fail(MPD_ERR_INVALID, "mpd_set_expression_ic: bad user variables");
    std::string err;
    mpd::ExprCode code[8];
    rc = mpd::CompileIc(exprs, n_vars, var_names, var_values, code, err);
    if (rc != MPD_OK) return Fail(rc, err);
    int read = -1;
    const int fwd = mpd::IcForwardReference(code, read);
    if (fwd >= 0) {
        static const char *names[8] = {"rho", "v_z", "v_r", "v_phi", "H_z", "H_r", "H_phi", "e"};
        return Fail(MPD_ERR_UNSUPPORTED_IC,
                    std::string("ExpressionIC on the device: the expression for '") + names[fwd] +
                        "' reads '" + names[read] +
                        "', which is evaluated after it; in the reference's sequential sweep "
                        "that reads the previous cell's value (mpd_expression_ic reproduces it)");
    }
    mpd::IcPrograms pr{};
    std::vector<int32_t> all_code;
    std::vector<double> all_consts;
    for (int j = 0; j < 8; ++j) {
        pr.code_off[j] = static_cast<int>(all_code.size());
        pr.const_off[j] = static_cast<int>(all_consts.size());
        all_code.insert(all_code.end(), code[j].code.begin(), code[j].code.end());
        all_consts.insert(all_consts.end(), code[j].consts.begin(), code[j].consts.end());
    }
    if (all_consts.empty()) all_consts.push_back(0.0);
    MPD_CK(cudaStreamSynchronize(s->stream));
    if (s->snap_pending) MPD_CK(cudaEventSynchronize(s->snap_ev));
    s->snap_pending = false;
    int32_t *d_code = nullptr;
    double *d_consts = nullptr;
    if (cudaMalloc(&d_code, all_code.size() * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&d_consts, all_consts.size() * sizeof(double)) != cudaSuccess) {
        cudaFree(d_code);
        cudaGetLastError();
        return Fail(MPD_ERR_NOMEM, "mpd_set_expression_ic: device allocation failed");
    }
    cudaError_t e = cudaMemcpyAsync(d_code, all_code.data(), all_code.size() * sizeof(int32_t),
                                    cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_consts, all_consts.data(), all_consts.size() * sizeof(double),
                            cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->ic, 0, 10 * s->ps * sizeof(double), s->stream);
    if (e == cudaSuccess) {
        pr.code = d_code;
        pr.consts = d_consts;
        mpd::expression_ic_kernel<<<4 * 148, 256, 0, s->stream>>>(s->g, s->ic, pr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    cudaFree(d_code);
    cudaFree(d_consts);
    if (e != cudaSuccess) return Fail(MPD_ERR_CUDA, cudaGetErrorString(e));
    return InitFromIc(s);
}

int mpd_set_ring_overlap(mpd_solver *s, int on) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    MPD_CK(cudaStreamSynchronize(s->stream));
    s->ring_overlap = on ? 1 : 0;
    return MPD_OK;
}

int mpd_ring_overlap_active(mpd_solver *s, int *active) {
    if (!s || !active) return Fail(MPD_ERR_INVALID, "bad arguments");
    *active = (s->precision == MPD_PRECISION_FAST && s->ring_overlap && s->overlap_ok) ? 1 : 0;
    return MPD_OK;
}

int mpd_get_stream(mpd_solver *s, void **stream) {
    if (!s || !stream) return Fail(MPD_ERR_INVALID, "bad arguments");
    *stream = static_cast<void *>(s->stream);
    return MPD_OK;
}

int mpd_profile_kernels(mpd_solver *s, int steps, double dt, double out_ms[2]) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    if (steps <= 0 || !out_ms) return Fail(MPD_ERR_INVALID, "bad profile request");
    // all launches are queued before any is waited for, so each event pair
    // brackets device work only (no host launch gap inside a pair)
    std::vector<cudaEvent_t> ev(3 * static_cast<size_t>(steps), nullptr);
    for (auto &e : ev) MPD_CK(cudaEventCreate(&e));
    for (int i = 0; i < steps && rc == MPD_OK; ++i) {
        const bool first = s->host_step == 0;
        MPD_CK(cudaEventRecord(ev[3 * i], s->stream));
        rc = LaunchInterior(s, first, false, dt, true);
        if (rc != MPD_OK) break;
        MPD_CK(cudaEventRecord(ev[3 * i + 1], s->stream));
        rc = LaunchBoundary(s, false, dt);
        if (rc != MPD_OK) break;
        MPD_CK(cudaEventRecord(ev[3 * i + 2], s->stream));
        s->host_step++;
    }
    double tot[2] = {0.0, 0.0};
    if (rc == MPD_OK) {
        MPD_CK(cudaStreamSynchronize(s->stream));
        for (int i = 0; i < steps; ++i) {
            float a = 0.f, b = 0.f;
            MPD_CK(cudaEventElapsedTime(&a, ev[3 * i], ev[3 * i + 1]));
            MPD_CK(cudaEventElapsedTime(&b, ev[3 * i + 1], ev[3 * i + 2]));
            tot[0] += a;
            tot[1] += b;
        }
    }
    for (auto &e : ev) cudaEventDestroy(e);
    if (rc != MPD_OK) return rc;
    out_ms[0] = tot[0] / steps;
    out_ms[1] = tot[1] / steps;
    return MPD_OK;
}

int mpd_profile_kernel(mpd_solver *s, int which, int launches, double dt, double *ms) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    if (launches <= 0 || !ms ||
        (which != MPD_KERNEL_INTERIOR && which != MPD_KERNEL_RESIDUAL &&
         which != MPD_KERNEL_INTERIOR_PAIR))
        return Fail(MPD_ERR_INVALID, "bad profile request");
    rc = SyncState(s);
    if (rc != MPD_OK) return rc;
    if (s->h_st->step == 0)
        return Fail(MPD_ERR_INVALID, "profile a kernel after the first step");
    MPD_CK(cudaEventRecord(s->ev0, s->stream));
    for (int i = 0; i < launches && rc == MPD_OK; ++i) {
        if (which == MPD_KERNEL_INTERIOR) {
            rc = LaunchInterior(s, false, false, dt, true, 0, true);
        } else if (which == MPD_KERNEL_INTERIOR_PAIR) {
            rc = LaunchInterior(s, false, false, dt, true, 1, true);
        } else {
            mpd::residual_kernel<<<s->resid_blocks, 256, 0, s->stream>>>(s->g, s->buf[0],
                                                                         s->buf[1], s->st, 1);
            MPD_CK(cudaGetLastError());
        }
    }
    if (rc != MPD_OK) return rc;
    MPD_CK(cudaEventRecord(s->ev1, s->stream));
    MPD_CK(cudaEventSynchronize(s->ev1));
    float t = 0.f;
    MPD_CK(cudaEventElapsedTime(&t, s->ev0, s->ev1));
    *ms = static_cast<double>(t) / launches;
    // the interior launches folded this dt's wave speed into the step's
    // accumulator: clear it, so the next step's controller sees only its own
    if (which != MPD_KERNEL_RESIDUAL) {
        MPD_CK(cudaMemsetAsync(&s->st->ws_acc, 0, sizeof(unsigned long long), s->stream));
        MPD_CK(cudaMemsetAsync(&s->st->nf_acc, 0, sizeof(unsigned int), s->stream));
        MPD_CK(cudaStreamSynchronize(s->stream));
    }
    return SyncState(s);
}

int mpd_device_bytes(mpd_solver *s, size_t *bytes) {
    if (!s || !bytes) return Fail(MPD_ERR_INVALID, "bad arguments");
    *bytes = s->dev_bytes;
    return MPD_OK;
}

struct mpd_batch {
    std::vector<mpd_solver *> solvers;
    int device = 0;
    int capacity = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    mpd::PersistArgs *d_solves = nullptr;
    CUtensorMap *d_maps = nullptr;
    int *d_ints = nullptr;            // team_first | solve_first | order
    mpd::GridSync *d_gs = nullptr;    // one per team (at most one per solve)
};

static void FreeBatch(mpd_batch *b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    cudaFree(b->d_solves);
    cudaFree(b->d_maps);
    cudaFree(b->d_ints);
    cudaFree(b->d_gs);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int mpd_batch_create(mpd_solver *const *solvers, int n, mpd_batch **out) {
    if (!out) return Fail(MPD_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!solvers || n <= 0) return Fail(MPD_ERR_INVALID, "a batch needs at least one solver");
    int dev = 0;
    MPD_CK(cudaGetDevice(&dev));
    for (int i = 0; i < n; ++i) {
        const int rc = CheckHandle(solvers[i]);
        if (rc != MPD_OK) return rc;
        if (solvers[i]->precision != MPD_PRECISION_FAST || !solvers[i]->persist_ok)
            return Fail(MPD_ERR_INVALID, "batched solvers must use MPD_PRECISION_FAST on a "
                                         "device with cooperative launch");
        if (solvers[i]->device != dev)
            return Fail(MPD_ERR_INVALID, "batched solvers must live on the current device");
    }
    auto *b = new mpd_batch();
    b->solvers.assign(solvers, solvers + n);
    b->device = dev;
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        mpd::persist_blocks_per_sm(per_sm) != cudaSuccess || per_sm < 1) {
        FreeBatch(b);
        return Fail(MPD_ERR_CUDA, "occupancy query for the batch kernel failed");
    }
    b->capacity = sms * per_sm;
    const size_t nints = 2 * (static_cast<size_t>(n) + 1) + n;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void **>(&b->d_solves), n * sizeof(mpd::PersistArgs)) !=
            cudaSuccess ||
        cudaMalloc(reinterpret_cast<void **>(&b->d_maps), 2 * n * sizeof(CUtensorMap)) !=
            cudaSuccess ||
        cudaMalloc(reinterpret_cast<void **>(&b->d_ints), nints * sizeof(int)) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void **>(&b->d_gs), n * sizeof(mpd::GridSync)) !=
            cudaSuccess) {
        FreeBatch(b);
        return Fail(MPD_ERR_NOMEM, "batch allocation failed");
    }
    *out = b;
    return MPD_OK;
}

void mpd_batch_destroy(mpd_batch *b) { FreeBatch(b); }

int mpd_batch_capacity(mpd_batch *b, int *blocks) {
    if (!b || !blocks) return Fail(MPD_ERR_INVALID, "NULL argument");
    *blocks = b->capacity;
    return MPD_OK;
}

int mpd_batch_run(mpd_batch *b, const mpd_run_params *p, int nteams, const int *team_blocks,
                  const int *solve_team, const double *dt0, mpd_run_stats *stats,
                  double *solve_ms, double *device_ms) {
    if (!b) return Fail(MPD_ERR_INVALID, "batch handle is NULL");
    const int n = static_cast<int>(b->solvers.size());
    if (!team_blocks || !solve_team || nteams < 1 || nteams > n)
        return Fail(MPD_ERR_INVALID, "bad team plan");
    long long used = 0;
    for (int k = 0; k < nteams; ++k) {
        if (team_blocks[k] < 1) return Fail(MPD_ERR_INVALID, "a team needs at least one block");
        used += team_blocks[k];
    }
    if (used > b->capacity)
        return Fail(MPD_ERR_INVALID, "teams need " + std::to_string(used) + " blocks; one wave holds " +
                                         std::to_string(b->capacity));
    for (int i = 0; i < n; ++i)
        if (solve_team[i] < 0 || solve_team[i] >= nteams)
            return Fail(MPD_ERR_INVALID, "solve_team out of range");
    if (p && p->convergence_threshold > 0.0)
        return Fail(MPD_ERR_INVALID, "batched runs take no convergence_threshold");
    const long long chunk = (p && p->steps_per_graph > 0) ? p->steps_per_graph : 5000;

    // every solve: run mode, then the exact first step where the solve has none
    std::vector<long long> step0(n), base(n);
    for (int i = 0; i < n; ++i) {
        mpd_solver *s = b->solvers[i];
        int rc = CheckRunParams(s, p);
        if (rc != MPD_OK) return rc;
        mpd_run_params pi = *p;
        if (dt0) pi.dt = dt0[i];
        rc = PrepareRun(s, &pi, step0[i]);
        if (rc != MPD_OK) return rc;
        MPD_CK(cudaEventRecord(s->ev0, s->stream));
        const bool first = !s->h_st->done && s->host_step == 0;
        if (first) {
            rc = EnqueueStep(s, true, true, 0.0, false, p->adaptive != 0, p->residual_every == 1);
            if (rc != MPD_OK) return rc;
        }
        base[i] = step0[i] + (first ? 1 : 0);
    }
    for (mpd_solver *s : b->solvers) MPD_CK(cudaStreamSynchronize(s->stream));

    // plan: team block ranges, solves grouped by team, per-solve interior tasks
    std::vector<int> team_first(nteams + 1, 0), solve_first(nteams + 1, 0), order;
    for (int k = 0; k < nteams; ++k) team_first[k + 1] = team_first[k] + team_blocks[k];
    for (int k = 0; k < nteams; ++k) {
        solve_first[k] = static_cast<int>(order.size());
        for (int i = 0; i < n; ++i)
            if (solve_team[i] == k) order.push_back(i);
    }
    solve_first[nteams] = static_cast<int>(order.size());
    std::vector<mpd::PersistArgs> args(n);
    std::vector<CUtensorMap> maps(2 * n);
    for (int i = 0; i < n; ++i) {
        mpd_solver *s = b->solvers[i];
        int nstrips = 0, nbands = 0;
        mpd::persist_tasks(s->g, team_blocks[solve_team[i]], nstrips, nbands);
        args[i] = PersistArgsOf(s, nstrips, nbands, chunk, base[i]);
        maps[2 * i] = s->tmap[0];
        maps[2 * i + 1] = s->tmap[1];
    }
    std::vector<int> ints;
    ints.insert(ints.end(), team_first.begin(), team_first.end());
    ints.insert(ints.end(), solve_first.begin(), solve_first.end());
    ints.insert(ints.end(), order.begin(), order.end());
    MPD_CK(cudaMemcpyAsync(b->d_solves, args.data(), n * sizeof(mpd::PersistArgs),
                           cudaMemcpyHostToDevice, b->stream));
    MPD_CK(cudaMemcpyAsync(b->d_maps, maps.data(), 2 * n * sizeof(CUtensorMap),
                           cudaMemcpyHostToDevice, b->stream));
    MPD_CK(cudaMemcpyAsync(b->d_ints, ints.data(), ints.size() * sizeof(int),
                           cudaMemcpyHostToDevice, b->stream));
    mpd::BatchArgs ba{};
    ba.solves = b->d_solves;
    ba.maps = b->d_maps;
    ba.team_first = b->d_ints;
    ba.solve_first = b->d_ints + (nteams + 1);
    ba.order = b->d_ints + 2 * (nteams + 1);
    ba.gs = b->d_gs;
    ba.nteams = nteams;
    const int blocks = team_first[nteams];

    MPD_CK(cudaEventRecord(b->ev0, b->stream));
    long long last = -1;
    int nteams_cur = nteams, blocks_cur = blocks;
    for (;;) {
        MPD_CK(cudaMemsetAsync(b->d_gs, 0, nteams_cur * sizeof(mpd::GridSync), b->stream));
        MPD_CK(mpd::launch_lf_batch(blocks_cur, ba, b->stream));
        long long total = 0;
        bool all_done = true, failed = false;
        for (mpd_solver *s : b->solvers)
            MPD_CK(cudaMemcpyAsync(s->h_st, s->st, sizeof(mpd::DevState), cudaMemcpyDeviceToHost,
                                   b->stream));
        MPD_CK(cudaStreamSynchronize(b->stream));
        for (mpd_solver *s : b->solvers) {
            RefreshMirror(s);
            total += s->h_st->step;
            all_done = all_done && s->h_st->done;
            failed = failed || s->h_st->wait_fail;
        }
        if (failed)
            return Fail(MPD_ERR_TIMEOUT, "a bounded device wait gave up; the state is not valid");
        if (all_done) break;
        if (total == last) return Fail(MPD_ERR_TIMEOUT, "batch run made no progress");
        last = total;
        // Elastic re-plan: once fewer solves are left than teams (the rest
        // would idle for the remaining launches), every remaining solve gets
        // a team of its own and the wave's blocks are split evenly between
        // them, up to the blocks that still give it interior tasks (one
        // 800 x 320 solve on a B200: 50.6 us a step on 64 blocks, 33.8 us on
        // 128).  A solve's results do not depend on its team's size.
        std::vector<int> active;
        for (int i = 0; i < n; ++i)
            if (!b->solvers[i]->h_st->done) active.push_back(i);
        if (!active.empty() && static_cast<int>(active.size()) < nteams_cur) {
            nteams_cur = static_cast<int>(active.size());
            const int share = b->capacity / nteams_cur;
            std::vector<int> tf(nteams_cur + 1, 0), sf(nteams_cur + 1, 0);
            for (int k = 0; k < nteams_cur; ++k) {
                mpd_solver *sv = b->solvers[active[k]];
                const int strips = (sv->M + mpd::kFastCells - 1) / mpd::kFastCells;
                const long long tasks = static_cast<long long>(strips) * sv->L;
                const int want = static_cast<int>((tasks + mpd::kTmaWarps - 1) / mpd::kTmaWarps);
                int nb = share < want ? share : want;
                if (nb < 1) nb = 1;
                tf[k + 1] = tf[k] + nb;
                sf[k + 1] = k + 1;
                int nstrips = 0, nbands = 0;
                mpd::persist_tasks(sv->g, nb, nstrips, nbands);
                args[active[k]].nstrips = nstrips;
                args[active[k]].nbands = nbands;
            }
            std::vector<int> ints2;
            ints2.insert(ints2.end(), tf.begin(), tf.end());
            ints2.insert(ints2.end(), sf.begin(), sf.end());
            ints2.insert(ints2.end(), active.begin(), active.end());
            MPD_CK(cudaMemcpyAsync(b->d_solves, args.data(), n * sizeof(mpd::PersistArgs),
                                   cudaMemcpyHostToDevice, b->stream));
            MPD_CK(cudaMemcpyAsync(b->d_ints, ints2.data(), ints2.size() * sizeof(int),
                                   cudaMemcpyHostToDevice, b->stream));
            MPD_CK(cudaStreamSynchronize(b->stream));
            ba.team_first = b->d_ints;
            ba.solve_first = b->d_ints + (nteams_cur + 1);
            ba.order = b->d_ints + 2 * (nteams_cur + 1);
            ba.nteams = nteams_cur;
            blocks_cur = tf[nteams_cur];
        }
    }
    MPD_CK(cudaEventRecord(b->ev1, b->stream));
    MPD_CK(cudaEventSynchronize(b->ev1));
    float ms = 0.f;
    MPD_CK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    if (device_ms) *device_ms = ms;
    unsigned long long t_first = ~0ull;
    std::vector<unsigned long long> done_ns(n);
    for (int i = 0; i < n; ++i) {
        const mpd::DevState &h = *b->solvers[i]->h_st;
        if (h.t0_ns && h.t0_ns < t_first) t_first = h.t0_ns;
        done_ns[i] = h.done_ns;
    }
    int status = MPD_OK;
    for (int i = 0; i < n; ++i) {
        if (solve_ms)
            solve_ms[i] = (done_ns[i] && t_first != ~0ull) ? (done_ns[i] - t_first) * 1e-6 : NAN;
        const int rc = FinishRun(b->solvers[i], step0[i], stats ? &stats[i] : nullptr);
        if (rc == MPD_ERR_NONFINITE) status = rc;
        else if (rc != MPD_OK) return rc;
    }
    if (status != MPD_OK) return Fail(status, "non-finite value in a batched solve");
    return MPD_OK;
}

}  // extern "C"
