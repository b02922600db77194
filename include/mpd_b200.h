/*
 * mpd_b200 — C ABI of the B200 Lax-Friedrichs MHD solver.
 *
 * One opaque handle owns one solve: device-resident structure-of-arrays FP64
 * storage of the eight conserved planes (ping-pong), the initial physical
 * planes, the wall profiles, the compiled boundary-condition table and one
 * CUDA stream.  Every entry point returns an int status (MPD_OK = 0) and never
 * throws; mpd_last_error() gives the message of the calling thread's last
 * failure.  One host thread drives a handle at a time.
 *
 * Index conventions follow the reference exactly (single MPI rank):
 *   planes are (L_max+2) x (M_max+3) doubles, row-major [l][m];
 *   l = 0 and l = L_max+1 are ghost rows, m = 0 and m = M_max+2 ghost columns;
 *   interior l in [1, L_max] (z = (l-1)*dz), m in [1, M_max+1] (m_global = m-1).
 * Host planes passed in or out of this ABI are dense with that shape.
 *
 * The reference exposes C++ classes, not a C API; each entry point below names
 * the reference member it replaces (paths relative to the reference repo).
 */
#ifndef MPD_B200_H
#define MPD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define MPD_OK 0
#define MPD_ERR_INVALID 1        /* bad argument or configuration              */
#define MPD_ERR_CUDA 2           /* a CUDA runtime call failed                  */
#define MPD_ERR_NOMEM 3          /* device or pinned allocation failed / budget */
#define MPD_ERR_UNSUPPORTED_BC 4 /* boundary configuration the device can't run */
#define MPD_ERR_EXPR 5           /* expression failed to compile                */
#define MPD_ERR_NONFINITE 6      /* NaN or Inf seen in the state                */
#define MPD_ERR_TIMEOUT 7        /* a bounded device wait gave up               */
#define MPD_ERR_NO_DEVICE 8      /* no CUDA device / extension unusable         */
#define MPD_ERR_UNSUPPORTED_IC 9 /* initial condition the device can't evaluate */

/* ---- enumerations (values equal the reference's enums) ----------------- */
/* FaceBC::Face, include/face_bc.hpp:52 */
enum { MPD_FACE_L_LO = 0, MPD_FACE_L_HI = 1, MPD_FACE_M_LO = 2, MPD_FACE_M_HI = 3 };
/* FieldCondType, include/field_condition.hpp:92-97 */
enum { MPD_NEUMANN = 0, MPD_DIRICHLET = 1, MPD_EXPRESSION = 2, MPD_AXIS_LF = 3 };
/* Fields physical members, include/fields.hpp:35-37 */
enum {
    MPD_RHO = 0, MPD_V_Z = 1, MPD_V_R = 2, MPD_V_PHI = 3, MPD_E = 4,
    MPD_P_GAS = 5, MPD_P_TOT = 6, MPD_H_Z = 7, MPD_H_R = 8, MPD_H_PHI = 9
};
/* arithmetic of the plain FP64 path */
enum {
    MPD_PRECISION_EXACT = 0, /* same IEEE operations, order and true divides as the
                                reference: bit-for-bit identical fields        */
    MPD_PRECISION_FAST = 1   /* reciprocal multiplies + FMA in the interior update
                                (<= 1e-12 relative L-inf after 1000 steps)     */
};

/* ---- configuration ----------------------------------------------------- */
/* FieldCond, include/field_condition.hpp:100-105 */
typedef struct mpd_field_cond {
    int type;          /* MPD_NEUMANN / MPD_DIRICHLET / MPD_EXPRESSION / MPD_AXIS_LF */
    double value;      /* Neumann offset or Dirichlet value                          */
    const char *expr;  /* expression source (MPD_EXPRESSION only), NUL-terminated    */
} mpd_field_cond;

/* BCSegmentConfig, include/config.hpp:82-95 (same field order) */
typedef struct mpd_bc_segment {
    int global_lo;     /* negative -> face start */
    int global_hi;     /* negative -> face end   */
    mpd_field_cond rho, v_z, v_r, v_phi, e, H_z, H_r, H_phi;
} mpd_bc_segment;

/* The SimConfig fields the hot path reads (include/config.hpp:119-176) plus
 * Grid::r_0 (include/grid.hpp:38).  dz and dy are passed as computed by the
 * caller (SimConfig::Init, src/config.cpp:15-18: 1/L_max, 1/M_max). */
typedef struct mpd_config {
    double gamma, beta, H_z0;
    int L_max, M_max;
    double dz, dy;
    double r_0;
    int n_segments[4];                    /* per face, indexed by MPD_FACE_*  */
    const mpd_bc_segment *segments[4];    /* in config order                  */
    int precision;                        /* MPD_PRECISION_*                  */
    int with_prev;                        /* keep prev planes for SolutionChange */
} mpd_config;

/* IGeometry sampled on the host at z = (l-1)*dz for l = 0..L_max+1
 * (include/igeometry.hpp:16-34, used by Grid::Build src/grid.cpp:20-42). */
typedef struct mpd_geometry {
    const double *r_inner, *r_outer, *dr_inner_dz, *dr_outer_dz;
} mpd_geometry;

typedef struct mpd_solver mpd_solver;

/* ---- lifetime ---------------------------------------------------------- */
/* Replaces the Fields ctor + Fields::InitConservative (src/fields.cpp:40-57),
 * Grid::Build and the Solver ctor (src/solver.cpp:9-16: FaceBC::FromConfig,
 * PerFieldBC validation and expression compile).  phys10 is the initial
 * physical state written by IInitialCondition::Apply: 10 dense host planes in
 * MPD_RHO..MPD_H_PHI order (ghost entries are ignored and treated as 0);
 * NULL starts from all-zero planes, for a state set next by
 * mpd_set_expression_ic or mpd_set_physical. */
int mpd_create(const mpd_config *cfg, const mpd_geometry *geom, const double *phys10,
               mpd_solver **out);
void mpd_destroy(mpd_solver *s);
const char *mpd_last_error(void);

/* ---- the hot path -------------------------------------------------------- */
/* Solver::Advance(double dt), src/solver.cpp:22-37.  Enqueued on the handle's
 * stream; returns without waiting.  Also records the maximum wave speed of the
 * new state (for mpd_compute_dt) and the L-inf residual of the step. */
int mpd_advance(mpd_solver *s, double dt);

/* Graph-resident driver loop of src/main.cpp:191-282: T clamp, adaptive dt
 * (Diagnostics::ComputeDt after every step), the reference's relative-L2
 * convergence check every check_frequency steps, and an L-inf residual
 * criterion.  Runs until t >= T, convergence, or max_steps. */
/* How mpd_run drives the steps.  GRAPH: an interior and a boundary kernel per
 * step, replayed from captured CUDA graphs.  PERSISTENT: one cooperative
 * launch runs many steps with grid barriers between the interior and the
 * boundary phase (fast precision, no SolutionChange checks).  AUTO takes
 * GRAPH.  Both give the same results, bit for bit. */
#define MPD_ENGINE_AUTO 0
#define MPD_ENGINE_GRAPH 1
#define MPD_ENGINE_PERSISTENT 2

/* One report of the reference driver loop's periodic diagnostics
 * (src/main.cpp:249-281), taken by mpd_run after every step whose count is a
 * multiple of mpd_run_params.monitor_every (the reference: 1000). */
typedef struct mpd_monitor_record {
    long long step;        /* step count since the solver's initial state        */
    double t;              /* simulated time after that step                     */
    double dt;             /* dt of the next step (after the adaptive update)    */
    double probe[5];       /* rho, v_z, v_phi, e, H_phi at the global cell
                              (l 20, m 40) (src/main.cpp:196-197,258-270);
                              0 when the grid has no such cell                   */
    double integrals[7];   /* Verification::ComputeIntegrals, src/verification.cpp:16-45 */
    double max_wave_speed; /* Diagnostics::MaxWaveSpeed of the state             */
    double dt_cfl;         /* cfl_number * min(dz, dy) / (max_wave_speed + 1e-10) */
    int cfl_warning;       /* dt > dt_cfl: Diagnostics::CheckCfl's warning
                              condition (src/diagnostics.cpp:112-125)            */
} mpd_monitor_record;

/* Called by mpd_run on its own host thread with the stream idle; the record
 * is valid only during the call. */
typedef void (*mpd_monitor_fn)(const mpd_monitor_record *record, void *user);

typedef struct mpd_run_params {
    double T;                   /* end time (use a huge value for step-limited runs) */
    double dt;                  /* initial dt (SimConfig::dt); <= 0: the CFL limit of
                                   the current state (warm starts)                    */
    int adaptive;               /* SimConfig::adaptive_dt                             */
    double cfl_number, dt_growth_factor, dt_min, dt_max;
    double convergence_threshold; /* relative-L2 change threshold, 0 = off          */
    int check_frequency;          /* steps between SolutionChange checks             */
    double residual_tol;          /* stop when the L-inf residual <= tol, 0 = off    */
    int residual_every;           /* steps between residual evaluations (>= 1)       */
    long long max_steps;
    int steps_per_graph;          /* steps captured per CUDA graph launch (0 = auto) */
    int engine;                   /* MPD_ENGINE_AUTO / _GRAPH / _PERSISTENT           */
    int monitor_every;            /* steps between monitor reports; 0 = none. Needs
                                     the graph engine; the loop then stops at every
                                     multiple of it, and the residual schedule
                                     restarts there                                  */
    mpd_monitor_fn monitor;       /* NULL = no reports                               */
    void *monitor_user;           /* passed to monitor                               */
} mpd_run_params;

typedef struct mpd_run_stats {
    long long steps;     /* steps taken by this call            */
    double t;            /* simulated time reached              */
    double dt;           /* next dt                             */
    double residual;     /* last L-inf residual evaluated       */
    double change;       /* last relative-L2 change evaluated   */
    double max_wave_speed;
    int converged;       /* 1 = residual or change criterion met */
    int status;          /* MPD_OK or MPD_ERR_NONFINITE          */
    double device_ms;    /* device time of the loop (CUDA events on the handle's stream,
                            from before the first launch to the end of the launch the
                            run stopped in) */
} mpd_run_stats;

int mpd_run(mpd_solver *s, const mpd_run_params *p, mpd_run_stats *stats);

/* ---- diagnostics (each waits for the stream) ----------------------------- */
/* Diagnostics::MaxWaveSpeed, src/diagnostics.cpp:14-43 */
int mpd_max_wave_speed(mpd_solver *s, double *out);
/* Diagnostics::ComputeDt, src/diagnostics.cpp:49-65 */
int mpd_compute_dt(mpd_solver *s, double cfl_number, double growth, double dt_min,
                   double dt_max, double dt_current, double *dt_next);
/* Diagnostics::SolutionChange, src/diagnostics.cpp:71-106 (needs with_prev) */
int mpd_solution_change(mpd_solver *s, double *out);
/* Fields::SavePrev, src/fields.cpp:59-74 */
int mpd_save_prev(mpd_solver *s);
/* Verification::ComputeIntegrals, src/verification.cpp:16-45:
 * mass, mom_z, mom_r, mom_phi, energy, mag_flux_z, mag_flux_phi */
int mpd_integrals(mpd_solver *s, double out7[7]);
/* Diagnostics::GetMassFlux / GetThrust, src/integrals.cpp:45-112 */
int mpd_outlet(mpd_solver *s, double *mass_flux, double *thrust);
/* Verification::CheckRadialSymmetry, src/verification.cpp:121-146 */
int mpd_radial_symmetry(mpd_solver *s, double *out);
/* The L-inf residual of the last step (new; no reference counterpart):
 * max_k |u_k^{n+1} - u_k^n|_inf / max(|u_k^n|_inf, 1e-300) over interior cells. */
int mpd_residual(mpd_solver *s, double *out);
/* Physical values at one interior cell (the probe of src/main.cpp:258-275):
 * out10 in MPD_RHO..MPD_H_PHI order, l_global in [0,L_max-1], m_global in [0,M_max]. */
int mpd_probe(mpd_solver *s, int l_global, int m_global, double out10[10]);
/* Simulated time and step count of the handle. */
int mpd_time(mpd_solver *s, double *t, long long *step);

/* ---- state transfer --------------------------------------------------------- */
/* which: 0..7 conserved u0_1..u0_8, 8..17 physical planes MPD_RHO..MPD_H_PHI
 * (the reference's Fields arrays after the step).  Copies one dense plane into
 * host memory and waits. */
int mpd_download(mpd_solver *s, int which, double *host_plane);
/* Snapshot for I/O (IOManager::WriteFrame, src/io_manager.cpp:68-77): enqueue a
 * copy of all 10 physical planes into caller-owned PINNED host memory
 * (10 dense planes) on a side stream and return at once; mpd_snapshot_wait
 * blocks until that copy has landed.  Stepping may continue meanwhile. */
int mpd_snapshot_async(mpd_solver *s, double *pinned_phys10);
int mpd_snapshot_wait(mpd_solver *s);
/* Replace the state by new physical planes (restart; IInitialCondition::Apply
 * + Fields::InitConservative).  Resets step and time to 0. */
int mpd_set_physical(mpd_solver *s, const double *phys10);
/* ExpressionIC::Apply (src/ics/expression_ic.cpp:286-324) evaluated on the
 * device, one thread per cell, with the expressions and user constants of
 * mpd_expression_ic, then Fields::InitConservative; resets step and time to
 * 0.  The planes equal mpd_expression_ic's bit for bit (CUDA's math library
 * stands in for glibc in transcendental functions).  An expression that
 * reads a field evaluated after it (in the reference's sequential sweep, the
 * previous cell's value) is refused with MPD_ERR_UNSUPPORTED_IC. */
int mpd_set_expression_ic(mpd_solver *s, const char *const exprs[8], int n_vars,
                          const char *const *var_names, const double *var_values);

/* Where a fast step's boundary ring runs (new; no reference counterpart: the
 * reference applies the faces after the central update, src/solver.cpp:
 * 22-37, and both forms keep that order of values).  on = 1: beside the
 * interior kernel, in bc_overlap_kernel, which recomputes the
 * central cells the faces read from the step's input state, so the ring's
 * dependent chains overlap the interior and only the end-of-step controller
 * waits for it; the interior kernel then computes rows 2..L-1.  on = 0 (the
 * default): after the interior kernel, reading the central cells it stored.  The two give
 * the same bits.  Takes effect from the next step; exact precision, the first
 * step and grids with L_max < 4 always use the second form.
 * mpd_ring_overlap_active reports whether fast steps of the handle use the
 * first. */
int mpd_set_ring_overlap(mpd_solver *s, int on);
int mpd_ring_overlap_active(mpd_solver *s, int *active);

/* The handle's CUDA stream (a cudaStream_t), for callers that time or order
 * work around the solver. */
int mpd_get_stream(mpd_solver *s, void **stream);
/* Bytes of device memory the handle holds. */
int mpd_device_bytes(mpd_solver *s, size_t *bytes);

/* Measurement support (new; no reference counterpart): advance `steps` steps
 * with time step dt, launching eagerly with CUDA events around each kernel on
 * the handle's stream, and return the mean device time per launch in ms of
 * the interior kernel (out_ms[0]) and the boundary kernel (out_ms[1]). */
int mpd_profile_kernels(mpd_solver *s, int steps, double dt, double out_ms[2]);

/* Measurement support (new; no reference counterpart): the mean device time
 * in ms of one launch of a step kernel, from `launches` back-to-back launches
 * between two events on the handle's stream, with nothing else between them.
 * MPD_KERNEL_INTERIOR: the interior kernel of the handle's precision at time
 * step dt; every launch recomputes the next step's interior cells from the
 * current state (the step counter does not advance; the state stays valid).
 * MPD_KERNEL_RESIDUAL: the L-inf residual pass over the current and previous
 * state.  MPD_KERNEL_INTERIOR_PAIR: the interior kernel's two-point-column-
 * per-lane form (fast precision; the same bits as the default).  Needs a
 * handle that has taken at least one step. */
#define MPD_KERNEL_INTERIOR 0
#define MPD_KERNEL_RESIDUAL 1
#define MPD_KERNEL_INTERIOR_PAIR 2
int mpd_profile_kernel(mpd_solver *s, int which, int launches, double dt, double *ms);

/* ---- conserved integrals without allocating ----------------------------------- */
/* No counterpart in the reference.  For callers that cannot let a library call
 * cudaMalloc: a host whose framework owns every byte of device memory through
 * its own pool (a stray cudaMalloc bypasses the pool's accounting, or fails
 * once the pool has reserved the device), or one that has already handed its
 * device memory budget out.  Computes the same 7 sums as mpd_integrals
 * (Verification::ComputeIntegrals) over caller-owned device memory:
 *   d_u    the 8 conserved planes, plane k at d_u + k*plane_stride, cell (l,m)
 *          at l*pitch + m (ghost layer included, pitch >= M_max+3);
 *   d_dr   the L_max+2 row widths dr[l] = (r_outer - r_inner)/M_max;
 *   d_out7 receives the 7 sums (device memory).
 * Work is enqueued on `stream` (a cudaStream_t; NULL = the default stream)
 * and not waited for.  Its only scratch is a fixed device array of 8192 rows
 * x 7 doubles (458,752 bytes per GPU, kept until the process exits);
 * L_max > 8192 is rejected with MPD_ERR_INVALID.  Under CUDA's lazy module
 * loading (the default) that array is created when the first call on a
 * device loads the library's module, so make a first (warm-up) call on each
 * device before the caller's pool reserves the device's memory, and before
 * any stream capture.  Every call looks the array's address up in the
 * current context (nothing is cached across contexts or device resets).  All
 * calls share the one array and each rewrites the rows it uses: calls whose
 * work overlaps on the GPU race.  Calls no cudaMalloc, cudaFree or allocating
 * library routine. */
int mpd_integrals_noalloc(const double *d_u, size_t plane_stride, int pitch, int L_max,
                          int M_max, const double *d_dr, double dz, double *d_out7,
                          void *stream);

/* ---- batched solves: one persistent cooperative launch ------------------------ */
/* New; the reference runs one solve per process.  A batch groups existing
 * solvers (fast precision, one device) and runs them in one cooperative launch
 * of persistent teams: team k is team_blocks[k] resident blocks (interior
 * tasks of 30-column strips x row bands sized to the team, team-scoped
 * barriers) and runs the solves with solve_team[i] == k one after the other,
 * in increasing i.  Every solve takes exactly the steps, dt and residual
 * schedule mpd_run would give it (same bits).  The plan (team sizes and the
 * assignment) comes from the caller; the Python front end's autotuner times
 * team sizes per grid shape and packs the solves. */
typedef struct mpd_batch mpd_batch;

/* The solvers stay owned by the caller and must outlive the batch. */
int mpd_batch_create(mpd_solver *const *solvers, int n, mpd_batch **out);
void mpd_batch_destroy(mpd_batch *b);
/* Blocks one cooperative wave of the batch kernel holds on this device: the
 * sum of team_blocks may not exceed it. */
int mpd_batch_capacity(mpd_batch *b, int *blocks);
/* Run every solve with the same run parameters (convergence_threshold must be
 * 0; steps_per_graph = steps each solve may take per launch, 0 = 5000).
 * dt0 (n entries, or NULL for p->dt): each solve's initial dt (<= 0: the CFL
 * limit of its state).  stats: n entries.  solve_ms (n entries, or NULL): time from the first step
 * any solve took in this run to this solve's last step.  device_ms (or NULL):
 * the whole run.  The plan holds while every team has work; between launches,
 * once fewer solves are left than teams, the remaining solves are re-planned
 * one per team with the wave's blocks split evenly between them (results do
 * not depend on the plan, only the time does). */
int mpd_batch_run(mpd_batch *b, const mpd_run_params *p, int nteams, const int *team_blocks,
                  const int *solve_team, const double *dt0, mpd_run_stats *stats,
                  double *solve_ms, double *device_ms);

/* ---- surrogate network kernels (learned warm start) -------------------------- */
/* New; the reference has no learned component.  Device pointers, FP32 in
 * global memory; the GEMM rounds its operands to BF16 and accumulates in FP32
 * on the tcgen05 tensor cores:
 *   C[b](m,n) = alpha * sum_k A[b](m,k) B[b](n,k) + beta * C[b](m,n)
 * with element strides per operand (row, k, batch) so transposed operands
 * need no copy.  beta == 0 never reads C.  With work, a GEMM of few output
 * tiles and long K is split over K and the partials summed in a fixed order
 * (deterministic).  Launches on `stream` and returns
 * at once; mpd_nn_wait_status synchronises the stream and reports a tensor-
 * core wait that gave up (MPD_ERR_TIMEOUT). */
typedef struct mpd_gemm_desc {
    int M, N, K, batch;
    const float *A;
    long long sam, sak, sab;
    const float *B;
    long long sbn, sbk, sbb;
    float *C;
    long long scm, scn, scb;
    float alpha, beta;
    float *work;           /* optional scratch for split-K partial sums (or NULL) */
    long long work_floats; /* its size; K is split only when the tiles are few  */
} mpd_gemm_desc;

int mpd_nn_gemm(const mpd_gemm_desc *d, void *stream);
int mpd_nn_wait_status(void *stream);

/* Element-wise and reduction kernels of the network (FP32, deterministic sums):
 * z += bias (per column), out = GELU(z) (act != 0) or z;  g_z = g_out GELU'(z);
 * out[c] = sum over rows of x[r][c] (work: 128 * cols floats of scratch);
 * out (+)= sum of nparts arrays of n;
 * mean squared error of pred vs target into *loss (one double) with
 * grad = 2 (pred - target) / n (grad may be NULL), partial = scratch of
 * 148 * 32 doubles;  one Adam step (bias-corrected, step >= 1). */
int mpd_nn_bias_act(float *z, const float *bias, float *out, long long rows, int cols, int act,
                    void *stream);
int mpd_nn_act_bwd(const float *g_out, const float *z, float *g_z, long long n, void *stream);
int mpd_nn_colsum(const float *x, long long rows, int cols, float *out, float *work,
                  void *stream);
int mpd_nn_sum_parts(const float *parts, int nparts, long long n, float *out, int accumulate,
                     void *stream);
int mpd_nn_mse(const float *pred, const float *target, long long n, float *grad, double *partial,
               double *loss, void *stream);
int mpd_nn_adam(float *p, const float *g, float *m, float *v, long long n, float lr, float b1,
                float b2, float eps, int step, void *stream);

/* ---- restart remap ---------------------------------------------------------- */
/* VtkIC::Apply + Impl::Interp (src/ics/vtk_ic.cpp:137-239) on the device:
 * d_src holds 8 point fields of a snapshot (rho, v_z, v_r, v_phi, H_z, H_r,
 * H_phi, e), ni x nj points each, point (i, j) at i + j ni; the interior cells
 * of the 10 dense physical planes d_out10 ((L_max+2) x (M_max+3), Fields
 * member order) receive the bilinear remap with the reference's index
 * mapping, p and P derived.  Asynchronous on `stream`. */
int mpd_remap_snapshot(const double *d_src, int ni, int nj, int L_max, int M_max, double gamma,
                       double *d_out10, void *stream);

/* ---- the fast path's reciprocal and square root ------------------------------ */
/* New (no reference counterpart): d_rcp[i] = 1/x[i] and d_sqrt[i] = sqrt(x[i])
 * for n device values, evaluated exactly as MPD_PRECISION_FAST evaluates them
 * (hardware seed + polynomial correction), so a test can hold them to their
 * error bound against correctly rounded results.  Asynchronous on `stream`. */
int mpd_fast_math(const double *d_x, long long n, double *d_rcp, double *d_sqrt, void *stream);

/* ---- host-side expression initial condition ---------------------------------- */
/* ExpressionIC::Apply, src/ics/expression_ic.cpp:286-324, evaluated on the host
 * with the library's expression compiler.  exprs: 8 strings in the
 * evaluation order rho, v_z, v_r, v_phi, H_z, H_r, H_phi, e (NULL entries take
 * the reference defaults of src/ics/expression_ic.cpp:263-270); user constants
 * as parallel name/value arrays.  Writes 10 dense physical planes. */
int mpd_expression_ic(const mpd_config *cfg, const mpd_geometry *geom,
                      const char *const exprs[8], int n_vars, const char *const *var_names,
                      const double *var_values, double *phys10_out);

/* Compile and evaluate one expression over named scalars (host).  Used by the
 * config front end to validate expressions early. */
int mpd_eval_expression(const char *src, int n_syms, const char *const *names,
                        const double *values, double *out);

#ifdef __cplusplus
}
#endif
#endif /* MPD_B200_H */
