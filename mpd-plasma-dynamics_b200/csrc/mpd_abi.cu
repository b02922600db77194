// C ABI of the B200 solver (include/mpd_b200.h): handle lifetime, the step
// launch sequence, the graph-resident run loop, diagnostics and transfers.
#include <cuda_runtime.h>

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
    unsigned long long *red = nullptr;
    mpd::DevState *st = nullptr;
    mpd::DevState *h_st = nullptr;  // pinned mirror
    mpd::SegDesc *d_seg = nullptr;
    int32_t *d_code = nullptr;
    double *d_consts = nullptr;
    mpd::BcTable bc{};
    int precision = MPD_PRECISION_EXACT;
    int with_prev = 0;
    long long host_step = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0, graph_check = 0;
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
    cudaFree(s->small);
    cudaFree(s->red);
    cudaFree(s->st);
    cudaFree(s->d_seg);
    cudaFree(s->d_code);
    cudaFree(s->d_consts);
    if (s->h_st) cudaFreeHost(s->h_st);
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
int UploadPhysical(mpd_solver *s, const double *phys10) {
    const size_t n = static_cast<size_t>(s->rows) * s->cols;
    MPD_CK(cudaMemsetAsync(s->ic, 0, 10 * s->ps * sizeof(double), s->stream));
    for (int k = 0; k < 10; ++k) {
        const double *src = phys10 + k * n + s->cols + 1;  // (l=1, m=1)
        double *dst = s->ic + k * s->ps + s->pitch + 1;
        MPD_CK(cudaMemcpy2DAsync(dst, s->pitch * sizeof(double), src, s->cols * sizeof(double),
                                 (s->M + 1) * sizeof(double), s->L, cudaMemcpyHostToDevice,
                                 s->stream));
    }
    MPD_CK(cudaMemsetAsync(s->buf[0], 0, 8 * s->ps * sizeof(double), s->stream));
    MPD_CK(cudaMemsetAsync(s->buf[1], 0, 8 * s->ps * sizeof(double), s->stream));
    mpd::init_conservative_kernel<<<4 * 148, 256, 0, s->stream>>>(s->g, s->ic, s->buf[0]);
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
    init.T = INFINITY;
    init.max_steps = LLONG_MAX;
    init.want_ws = 1;
    init.resid_every = 1;
    *s->h_st = init;
    MPD_CK(cudaMemcpyAsync(s->st, s->h_st, sizeof(mpd::DevState), cudaMemcpyHostToDevice,
                           s->stream));
    MPD_CK(cudaStreamSynchronize(s->stream));
    s->host_step = 0;
    return MPD_OK;
}

// One time step: interior kernel, boundary kernel (+ controller), and in run
// mode the guarded relative-L2 convergence check.
int EnqueueStep(mpd_solver *s, bool first, bool use_state_dt, double dt, bool with_check) {
    const mpd::Geo &g = s->g;
    if (first || s->precision == MPD_PRECISION_EXACT) {
        dim3 block(32, 8);
        dim3 grid((g.M - 1 + 31) / 32, (g.L + 7) / 8);
        if (first)
            mpd::lf_exact_kernel<true><<<grid, block, 0, s->stream>>>(
                g, s->buf[0], s->buf[1], s->ic, s->st, dt, use_state_dt ? 1 : 0);
        else
            mpd::lf_exact_kernel<false><<<grid, block, 0, s->stream>>>(
                g, s->buf[0], s->buf[1], s->ic, s->st, dt, use_state_dt ? 1 : 0);
    } else {
        mpd::launch_lf_fast(g, s->buf[0], s->buf[1], s->st, dt, use_state_dt ? 1 : 0, s->stream);
    }
    MPD_CK(cudaGetLastError());
    const int nring = mpd::ring_count(g);
    mpd::bc_kernel<<<(nring + 127) / 128, 128, 0, s->stream>>>(
        g, s->buf[0], s->buf[1], s->ic, s->bc, s->st, dt, use_state_dt ? 1 : 0);
    MPD_CK(cudaGetLastError());
    if (with_check) {
        mpd::change_kernel<<<kRedBlocks, 256, 0, s->stream>>>(Bufs(s), s->prev, s->partials, 1, 1);
        mpd::change_finish_kernel<<<1, 32, 0, s->stream>>>(s->partials, kRedBlocks, s->st, 1);
        MPD_CK(cudaGetLastError());
    }
    return MPD_OK;
}

int SyncState(mpd_solver *s) {
    MPD_CK(cudaMemcpyAsync(s->h_st, s->st, sizeof(mpd::DevState), cudaMemcpyDeviceToHost,
                           s->stream));
    MPD_CK(cudaStreamSynchronize(s->stream));
    return MPD_OK;
}

int PushState(mpd_solver *s) {
    MPD_CK(cudaMemcpyAsync(s->st, s->h_st, sizeof(mpd::DevState), cudaMemcpyHostToDevice,
                           s->stream));
    MPD_CK(cudaStreamSynchronize(s->stream));
    return MPD_OK;
}

int CheckHandle(mpd_solver *s) {
    if (!s) return Fail(MPD_ERR_INVALID, "NULL solver handle");
    MPD_CK(cudaSetDevice(s->device));
    return MPD_OK;
}

int BuildGraph(mpd_solver *s, int steps, bool with_check) {
    if (s->graph && s->graph_steps == steps && s->graph_check == (with_check ? 1 : 0))
        return MPD_OK;
    if (s->graph) {
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
    }
    cudaGraph_t graph = nullptr;
    MPD_CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int rc = MPD_OK;
    for (int i = 0; i < steps && rc == MPD_OK; ++i) rc = EnqueueStep(s, false, true, 0.0, with_check);
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
    s->graph_check = with_check ? 1 : 0;
    return MPD_OK;
}

}  // namespace

extern "C" {

const char *mpd_last_error(void) { return mpd::g_last_error.c_str(); }

int mpd_create(const mpd_config *cfg, const mpd_geometry *geom, const double *phys10,
               mpd_solver **out) {
    std::string err;
    if (!out) return Fail(MPD_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int rc = mpd::ValidateConfig(cfg, geom, err);
    if (rc != MPD_OK) return Fail(rc, err);
    if (!geom || !phys10) return Fail(MPD_ERR_INVALID, "geometry and initial planes are required");
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
    STEP(DevAlloc(s, &s->geo, 5 * static_cast<size_t>(s->rows)));
    STEP(DevAlloc(s, &s->partials, static_cast<size_t>(kRedBlocks) * 8));
    STEP(DevAlloc(s, &s->small, 16));
    STEP(DevAlloc(s, &s->red, 4));
    STEP(DevAlloc(s, &s->st, 1));
    if (cudaMallocHost(reinterpret_cast<void **>(&s->h_st), sizeof(mpd::DevState)) != cudaSuccess) {
        FreeAll(s);
        return Fail(MPD_ERR_NOMEM, "pinned allocation failed");
    }
    // wall profiles + dr (Grid::Build: R = r_outer - r_inner, dr = R / M_max)
    {
        std::vector<double> h(5 * static_cast<size_t>(s->rows));
        for (int l = 0; l < s->rows; ++l) {
            h[0 * s->rows + l] = geom->r_inner[l];
            h[1 * s->rows + l] = geom->r_outer[l];
            h[2 * s->rows + l] = geom->dr_inner_dz[l];
            h[3 * s->rows + l] = geom->dr_outer_dz[l];
            const double R = geom->r_outer[l] - geom->r_inner[l];
            h[4 * s->rows + l] = R / cfg->M_max;
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
    rc = EnqueueStep(s, s->host_step == 0, false, dt, false);
    if (rc != MPD_OK) return rc;
    s->host_step++;
    return MPD_OK;
}

int mpd_run(mpd_solver *s, const mpd_run_params *p, mpd_run_stats *stats) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    if (!p) return Fail(MPD_ERR_INVALID, "run params are NULL");
    if (p->convergence_threshold > 0.0 && !s->with_prev)
        return Fail(MPD_ERR_INVALID, "convergence_threshold > 0 needs a solver created with with_prev");
    if (p->convergence_threshold > 0.0 && p->check_frequency <= 0)
        return Fail(MPD_ERR_INVALID, "check_frequency must be positive");
    if (p->max_steps <= 0) return Fail(MPD_ERR_INVALID, "max_steps must be positive");
    const bool with_check = p->convergence_threshold > 0.0;
    rc = SyncState(s);
    if (rc != MPD_OK) return rc;
    mpd::DevState &h = *s->h_st;
    const long long step0 = h.step;
    h.run_mode = 1;
    h.adaptive = p->adaptive ? 1 : 0;
    h.want_ws = p->adaptive ? 1 : 0;
    h.cfl = p->cfl_number;
    h.growth = p->dt_growth_factor;
    h.dt_min = p->dt_min;
    h.dt_max = p->dt_max;
    h.T = p->T;
    h.max_steps = step0 + p->max_steps;
    h.resid_tol = p->residual_tol;
    h.resid_every = p->residual_every > 0 ? p->residual_every : 0;
    h.conv_thr = p->convergence_threshold;
    h.check_freq = p->check_frequency;
    h.check_due = 0;
    h.done = 0;
    h.converged = 0;
    h.nonfinite = 0;
    double dt = p->dt;
    if (h.t + dt > h.T) dt = h.T - h.t;  // src/main.cpp:221-223
    h.dt = dt;
    if (!(h.t < h.T)) h.done = 1;
    rc = PushState(s);
    if (rc != MPD_OK) return rc;

    MPD_CK(cudaEventRecord(s->ev0, s->stream));
    if (!h.done && s->host_step == 0) {
        rc = EnqueueStep(s, true, true, 0.0, with_check);
        if (rc != MPD_OK) return rc;
    }
    int per_graph = p->steps_per_graph > 0 ? p->steps_per_graph : 100;
    if (with_check && p->check_frequency > 0 && per_graph % p->check_frequency != 0 &&
        p->check_frequency < per_graph)
        per_graph = (per_graph / p->check_frequency) * p->check_frequency;
    rc = BuildGraph(s, per_graph, with_check);
    if (rc != MPD_OK) return rc;
    long long last_step = -1;
    for (;;) {
        MPD_CK(cudaMemcpyAsync(s->h_st, s->st, sizeof(mpd::DevState), cudaMemcpyDeviceToHost,
                               s->stream));
        MPD_CK(cudaStreamSynchronize(s->stream));
        if (h.done) break;
        if (h.step == last_step)  // a launch that advanced nothing: stop, don't spin
            return Fail(MPD_ERR_TIMEOUT, "run loop made no progress");
        last_step = h.step;
        MPD_CK(cudaGraphLaunch(s->graph, s->stream));
    }
    MPD_CK(cudaEventRecord(s->ev1, s->stream));
    MPD_CK(cudaEventSynchronize(s->ev1));
    float ms = 0.f;
    MPD_CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    rc = SyncState(s);
    if (rc != MPD_OK) return rc;
    if (stats) {
        stats->steps = h.step - step0;
        stats->t = h.t;
        stats->dt = h.dt;
        stats->residual = h.last_resid;
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

int mpd_max_wave_speed(mpd_solver *s, double *out) {
    int rc = CheckHandle(s);
    if (rc != MPD_OK) return rc;
    if (!out) return Fail(MPD_ERR_INVALID, "out is NULL");
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
    mpd::change_finish_kernel<<<1, 32, 0, s->stream>>>(s->partials, kRedBlocks, s->st, 0);
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
    mpd::sum_partials_kernel<7><<<1, 32, 0, s->stream>>>(s->partials, nb, s->small);
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
    mpd::outlet_kernel<<<1, 32, 0, s->stream>>>(Bufs(s), inv_8pi, s->small);
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
    rc = SyncState(s);
    if (rc != MPD_OK) return rc;
    *out = s->h_st->resid_valid ? s->h_st->last_resid : NAN;
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
        int rc = DevAlloc(s, &s->stage, 10 * s->ps);
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
        src = s->stage + (which - 8) * s->ps;
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
    for (int k = 0; k < 10; ++k)
        MPD_CK(cudaMemcpy2DAsync(pinned_phys10 + k * n, s->cols * sizeof(double),
                                 s->stage + k * s->ps, s->pitch * sizeof(double),
                                 s->cols * sizeof(double), s->rows, cudaMemcpyDeviceToHost, s->side));
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
    return UploadPhysical(s, phys10);
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
    cudaEvent_t ev[3];
    for (auto &e : ev) MPD_CK(cudaEventCreate(&e));
    double tot[2] = {0.0, 0.0};
    const mpd::Geo &g = s->g;
    for (int i = 0; i < steps; ++i) {
        const bool first = s->host_step == 0;
        MPD_CK(cudaEventRecord(ev[0], s->stream));
        if (first || s->precision == MPD_PRECISION_EXACT) {
            dim3 block(32, 8);
            dim3 grid((g.M - 1 + 31) / 32, (g.L + 7) / 8);
            if (first)
                mpd::lf_exact_kernel<true><<<grid, block, 0, s->stream>>>(g, s->buf[0], s->buf[1],
                                                                           s->ic, s->st, dt, 0);
            else
                mpd::lf_exact_kernel<false><<<grid, block, 0, s->stream>>>(g, s->buf[0], s->buf[1],
                                                                            s->ic, s->st, dt, 0);
        } else {
            mpd::launch_lf_fast(g, s->buf[0], s->buf[1], s->st, dt, 0, s->stream);
        }
        MPD_CK(cudaEventRecord(ev[1], s->stream));
        const int nring = mpd::ring_count(g);
        mpd::bc_kernel<<<(nring + 127) / 128, 128, 0, s->stream>>>(g, s->buf[0], s->buf[1], s->ic,
                                                                   s->bc, s->st, dt, 0);
        MPD_CK(cudaEventRecord(ev[2], s->stream));
        MPD_CK(cudaGetLastError());
        MPD_CK(cudaEventSynchronize(ev[2]));
        float a = 0.f, b = 0.f;
        MPD_CK(cudaEventElapsedTime(&a, ev[0], ev[1]));
        MPD_CK(cudaEventElapsedTime(&b, ev[1], ev[2]));
        tot[0] += a;
        tot[1] += b;
        s->host_step++;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    out_ms[0] = tot[0] / steps;
    out_ms[1] = tot[1] / steps;
    return MPD_OK;
}

int mpd_device_bytes(mpd_solver *s, size_t *bytes) {
    if (!s || !bytes) return Fail(MPD_ERR_INVALID, "bad arguments");
    *bytes = s->dev_bytes;
    return MPD_OK;
}

}  // extern "C"
