/*
 * CPU oracle for the Lax-Friedrichs hot path — TEST INFRASTRUCTURE ONLY.
 * See mpd_oracle.h for the layout conventions and how it is pinned.
 *
 * Every arithmetic expression below keeps the operand order and grouping of
 * the reference source it restates (cited per function), because the GPU
 * "exact" mode is checked against it bit for bit.  Build with
 * -ffp-contract=off (oracle/Makefile does).
 */
#include "mpd_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "expr_eval.h"

#define NPH 10
enum { P_RHO, P_VZ, P_VR, P_VPHI, P_E, P_p, P_P, P_HZ, P_HR, P_HPHI };
enum { C_RHO, C_VZ, C_VR, C_VPHI, C_E, C_HZ, C_HR, C_HPHI };
enum { T_NEUMANN, T_DIRICHLET, T_EXPR, T_AXISLF };
enum { F_L_LO, F_L_HI, F_M_LO, F_M_HI };
#define MAX_SEG 16

/* Symbol slots of a segment's expression state (PerFieldBC::ExprImpl members,
 * src/bcs/per_field_bc.cpp:41-59); the values persist between cells and
 * between Apply calls exactly like the reference's mutable members. */
enum {
    S_GAMMA, S_BETA, S_HZ0, S_R0, S_DZ, S_DR, S_R, S_RZ, S_Z, S_RNB, S_RZNB,
    S_RHO_NB, S_VZ_NB, S_VR_NB, S_VPHI_NB, S_E_NB, S_HZ_NB, S_HR_NB, S_HPHI_NB,
    S_RHO, S_VZ, S_VR, S_VPHI, S_HZ, S_HR, S_HPHI, S_E, S_COUNT
};
static const char *k_sym_names[S_COUNT] = {
    "gamma", "beta", "H_z0", "r_0", "dz", "dr", "r", "r_z", "z", "r_nb", "r_z_nb",
    "rho_nb", "v_z_nb", "v_r_nb", "v_phi_nb", "e_nb", "H_z_nb", "H_r_nb", "H_phi_nb",
    "rho", "v_z", "v_r", "v_phi", "H_z", "H_r", "H_phi", "e"};

typedef struct {
    int face, glo, ghi;
    int type[8];
    double value[8];
    oe_expr *expr[8];
    int has_axis, has_expr;
    oe_symtab *st;
    double sym[S_COUNT];
} segment;

struct mo_case {
    int L, M, rows, cols;
    double gamma, beta, H_z0, dz, dy, r_0;
    double *r, *r_z, *dr;
    double *u0[8], *u[8], *ph[NPH], *prev[7];
    int with_prev;
    int nseg[4];
    segment seg[4][MAX_SEG];
};

#define IX(l, m) ((size_t)(l) * (size_t)c->cols + (size_t)(m))

static double *alloc_plane(const mo_case *c) {
    return (double *)calloc((size_t)c->rows * (size_t)c->cols, sizeof(double));
}

/* src/grid.cpp:20-42 (Grid::Build), single rank: l_start = m_start = 0. */
static void build_grid(mo_case *c, const double *rin, const double *rout, const double *drin,
                       const double *drout) {
    for (int l = 0; l < c->rows; ++l) {
        const double R = rout[l] - rin[l];
        c->dr[l] = R / c->M;
        for (int m = 0; m < c->cols; ++m) {
            const int m_global = m - 1;
            const double frac = m_global * c->dy;
            c->r[IX(l, m)] = (1.0 - frac) * rin[l] + frac * rout[l];
            c->r_z[IX(l, m)] = (1.0 - frac) * drin[l] + frac * drout[l];
        }
    }
}

/* src/fields.cpp:40-57 (Fields::InitConservative), interior only. */
static void init_conservative(mo_case *c) {
    double **u0 = c->u0, **ph = c->ph;
    for (int l = 1; l < c->rows - 1; ++l)
        for (int m = 1; m < c->cols - 1; ++m) {
            const size_t i = IX(l, m);
            const double r = c->r[i];
            u0[0][i] = ph[P_RHO][i] * r;
            u0[1][i] = ph[P_RHO][i] * ph[P_VZ][i] * r;
            u0[2][i] = ph[P_RHO][i] * ph[P_VR][i] * r;
            u0[3][i] = ph[P_RHO][i] * ph[P_VPHI][i] * r;
            u0[4][i] = ph[P_RHO][i] * ph[P_E][i] * r;
            u0[5][i] = ph[P_HPHI][i];
            u0[6][i] = ph[P_HZ][i] * r;
            u0[7][i] = ph[P_HR][i] * r;
        }
}

mo_case *mo_new(int L_max, int M_max, const double *params, const double *rin,
                const double *rout, const double *drin, const double *drout,
                const double *phys, int with_prev) {
    mo_case *c = (mo_case *)calloc(1, sizeof(mo_case));
    c->L = L_max;
    c->M = M_max;
    c->rows = L_max + 2;
    c->cols = M_max + 3;
    c->gamma = params[0];
    c->beta = params[1];
    c->H_z0 = params[2];
    c->dz = params[3];
    c->dy = params[4];
    c->r_0 = params[5];
    c->with_prev = with_prev;
    c->r = alloc_plane(c);
    c->r_z = alloc_plane(c);
    c->dr = (double *)calloc((size_t)c->rows, sizeof(double));
    for (int k = 0; k < 8; ++k) {
        c->u0[k] = alloc_plane(c);
        c->u[k] = alloc_plane(c);
    }
    const size_t n = (size_t)c->rows * (size_t)c->cols;
    for (int k = 0; k < NPH; ++k) {
        c->ph[k] = alloc_plane(c);
        /* interior only: ghosts stay zero (IInitialCondition contract,
         * include/iinitial_condition.hpp:21-39) */
        for (int l = 1; l < c->rows - 1; ++l)
            for (int m = 1; m < c->cols - 1; ++m) c->ph[k][IX(l, m)] = phys[k * n + IX(l, m)];
    }
    for (int k = 0; k < 7; ++k) c->prev[k] = with_prev ? alloc_plane(c) : NULL;
    build_grid(c, rin, rout, drin, drout);
    init_conservative(c);
    /* src/main.cpp:150-152: prev snapshot of the initial physical state */
    if (with_prev) mo_save_prev(c);
    return c;
}

void mo_free(mo_case *c) {
    if (!c) return;
    for (int f = 0; f < 4; ++f)
        for (int s = 0; s < c->nseg[f]; ++s) {
            for (int k = 0; k < 8; ++k) oe_free(c->seg[f][s].expr[k]);
            oe_symtab_free(c->seg[f][s].st);
        }
    free(c->r);
    free(c->r_z);
    free(c->dr);
    for (int k = 0; k < 8; ++k) { free(c->u0[k]); free(c->u[k]); }
    for (int k = 0; k < NPH; ++k) free(c->ph[k]);
    for (int k = 0; k < 7; ++k) free(c->prev[k]);
    free(c);
}

/* PerFieldBC constructor validation + ExprImpl compile
 * (src/bcs/per_field_bc.cpp:188-243, 76-181). */
int mo_add_segment(mo_case *c, int face, int global_lo, int global_hi, const int *types,
                   const double *values, const char *const *exprs, char *err, int errlen) {
    if (face < 0 || face > 3 || c->nseg[face] >= MAX_SEG) {
        snprintf(err, (size_t)errlen, "bad face or too many segments");
        return -1;
    }
    segment *s = &c->seg[face][c->nseg[face]];
    memset(s, 0, sizeof(*s));
    s->face = face;
    s->glo = global_lo;
    s->ghi = global_hi;
    for (int k = 0; k < 8; ++k) {
        s->type[k] = types[k];
        s->value[k] = values[k];
        if (types[k] == T_AXISLF) s->has_axis = 1;
        if (types[k] == T_EXPR) s->has_expr = 1;
    }
    if (s->has_axis && face != F_M_LO) {
        snprintf(err, (size_t)errlen, "AxisLF condition is only valid on the M_LO face");
        return -1;
    }
    if (types[C_VR] == T_AXISLF || types[C_VPHI] == T_AXISLF || types[C_HR] == T_AXISLF ||
        types[C_HPHI] == T_AXISLF) {
        snprintf(err, (size_t)errlen, "AxisLF is only valid for rho, v_z, e, and H_z");
        return -1;
    }
    if (s->has_expr) {
        s->st = oe_symtab_new();
        for (int i = 0; i < S_COUNT; ++i) oe_symtab_add_var(s->st, k_sym_names[i], &s->sym[i]);
        oe_symtab_add_const(s->st, "pi", M_PI);
        for (int k = 0; k < 8; ++k) {
            if (types[k] != T_EXPR) continue;
            s->expr[k] = oe_compile(exprs[k], s->st, err, errlen);
            if (!s->expr[k]) return -1;
        }
    }
    c->nseg[face]++;
    return 0;
}

/* ------------------------------------------------------------------ step */

/* src/solver.cpp:59-153 (Solver::ComputeCentralUpdate), one rank. */
static void central_update(mo_case *c, double dt) {
    const int L = c->L, local_M = c->M + 1;
    const double dz = c->dz;
    const int m_lo = 2, m_hi = local_M - 1;
    double *const *u0 = c->u0;
    double *const *u = c->u;
    const double *rho = c->ph[P_RHO], *v_z = c->ph[P_VZ], *v_r = c->ph[P_VR];
    const double *v_phi = c->ph[P_VPHI], *p = c->ph[P_p], *P = c->ph[P_P];
    const double *H_z = c->ph[P_HZ], *H_r = c->ph[P_HR], *H_phi = c->ph[P_HPHI];
    const double *r = c->r;
#pragma omp parallel for collapse(2)
    for (int l = 1; l <= L; ++l) {
        for (int m = m_lo; m <= m_hi; ++m) {
            const size_t C = IX(l, m), N = IX(l + 1, m), S = IX(l - 1, m);
            const size_t E = IX(l, m + 1), W = IX(l, m - 1);
            const double dr_l = c->dr[l];
            const double *a;

            a = u0[0];
            u[0][C] = 0.25 * (a[N] + a[S] + a[E] + a[W])
                    + dt * (-(a[N] * v_z[N] - a[S] * v_z[S]) / (2 * dz)
                            - (a[E] * v_r[E] - a[W] * v_r[W]) / (2 * dr_l));

            a = u0[1];
            u[1][C] = 0.25 * (a[N] + a[S] + a[E] + a[W])
                    + dt * (((H_z[N] * H_z[N] - P[N]) * r[N] - (H_z[S] * H_z[S] - P[S]) * r[S]) / (2 * dz)
                            + (H_z[E] * H_r[E] * r[E] - H_z[W] * H_r[W] * r[W]) / (2 * dr_l)
                            - (a[N] * v_z[N] - a[S] * v_z[S]) / (2 * dz)
                            - (a[E] * v_r[E] - a[W] * v_r[W]) / (2 * dr_l));

            a = u0[2];
            u[2][C] = 0.25 * (a[N] + a[S] + a[E] + a[W])
                    + dt * ((rho[C] * v_phi[C] * v_phi[C] + P[C] - H_phi[C] * H_phi[C])
                            + (H_z[N] * H_r[N] * r[N] - H_z[S] * H_r[S] * r[S]) / (2 * dz)
                            + ((H_r[E] * H_r[E] - P[E]) * r[E] - (H_r[W] * H_r[W] - P[W]) * r[W]) / (2 * dr_l)
                            - (a[N] * v_z[N] - a[S] * v_z[S]) / (2 * dz)
                            - (a[E] * v_r[E] - a[W] * v_r[W]) / (2 * dr_l));

            a = u0[3];
            u[3][C] = 0.25 * (a[N] + a[S] + a[E] + a[W])
                    + dt * ((-rho[C] * v_r[C] * v_phi[C] + H_phi[C] * H_r[C])
                            + (H_phi[N] * H_z[N] * r[N] - H_phi[S] * H_z[S] * r[S]) / (2 * dz)
                            + (H_phi[E] * H_r[E] * r[E] - H_phi[W] * H_r[W] * r[W]) / (2 * dr_l)
                            - (a[N] * v_z[N] - a[S] * v_z[S]) / (2 * dz)
                            - (a[E] * v_r[E] - a[W] * v_r[W]) / (2 * dr_l));

            a = u0[4];
            u[4][C] = 0.25 * (a[N] + a[S] + a[E] + a[W])
                    + dt * (-p[C] * ((v_z[N] * r[N] - v_z[S] * r[S]) / (2 * dz)
                                     + (v_r[E] * r[E] - v_r[W] * r[W]) / (2 * dr_l))
                            - (a[N] * v_z[N] - a[S] * v_z[S]) / (2 * dz)
                            - (a[E] * v_r[E] - a[W] * v_r[W]) / (2 * dr_l));

            a = u0[5];
            u[5][C] = 0.25 * (a[N] + a[S] + a[E] + a[W])
                    + dt * ((H_z[N] * v_phi[N] - H_z[S] * v_phi[S]) / (2 * dz)
                            + (H_r[E] * v_phi[E] - H_r[W] * v_phi[W]) / (2 * dr_l)
                            - (a[N] * v_z[N] - a[S] * v_z[S]) / (2 * dz)
                            - (a[E] * v_r[E] - a[W] * v_r[W]) / (2 * dr_l));

            a = u0[6];
            u[6][C] = 0.25 * (a[N] + a[S] + a[E] + a[W])
                    + dt * ((H_r[E] * v_z[E] * r[E] - H_r[W] * v_z[W] * r[W]) / (2 * dr_l)
                            - (a[E] * v_r[E] - a[W] * v_r[W]) / (2 * dr_l));

            a = u0[7];
            u[7][C] = 0.25 * (a[N] + a[S] + a[E] + a[W])
                    + dt * ((H_z[N] * v_r[N] * r[N] - H_z[S] * v_r[S] * r[S]) / (2 * dz)
                            - (a[N] * v_z[N] - a[S] * v_z[S]) / (2 * dz));
        }
    }
}

/* src/fields.cpp:76-99 (Fields::UpdatePhysicalFromU). */
static void update_physical(mo_case *c, int l_lo, int l_hi, int m_lo, int m_hi) {
    const double gamma = c->gamma;
    double **u = c->u, **ph = c->ph;
#pragma omp parallel for collapse(2)
    for (int l = l_lo; l <= l_hi; ++l) {
        for (int m = m_lo; m <= m_hi; ++m) {
            const size_t i = IX(l, m);
            const double r = c->r[i];
            ph[P_RHO][i] = u[0][i] / r;
            ph[P_VZ][i] = u[1][i] / u[0][i];
            ph[P_VR][i] = u[2][i] / u[0][i];
            ph[P_VPHI][i] = u[3][i] / u[0][i];
            ph[P_HPHI][i] = u[5][i];
            ph[P_HZ][i] = u[6][i] / r;
            ph[P_HR][i] = u[7][i] / r;
            ph[P_E][i] = u[4][i] / u[0][i];
            ph[P_p][i] = (gamma - 1.0) * ph[P_RHO][i] * ph[P_E][i];
            ph[P_P][i] = ph[P_p][i] + 0.5 * (ph[P_HZ][i] * ph[P_HZ][i] + ph[P_HR][i] * ph[P_HR][i]
                                             + ph[P_HPHI][i] * ph[P_HPHI][i]);
        }
    }
}

/* include/physics_utils.hpp:15-24 (RebuildUFromPhysical). */
static void rebuild_u(mo_case *c, int l, int m) {
    const size_t i = IX(l, m);
    const double r = c->r[i];
    double **u = c->u, **ph = c->ph;
    u[0][i] = ph[P_RHO][i] * r;
    u[1][i] = ph[P_RHO][i] * ph[P_VZ][i] * r;
    u[2][i] = ph[P_RHO][i] * ph[P_VR][i] * r;
    u[3][i] = ph[P_RHO][i] * ph[P_VPHI][i] * r;
    u[4][i] = ph[P_RHO][i] * ph[P_E][i] * r;
    u[5][i] = ph[P_HPHI][i];
    u[6][i] = ph[P_HZ][i] * r;
    u[7][i] = ph[P_HR][i] * r;
}

/* src/bcs/per_field_bc.cpp:490-566 (PerFieldBC::AxisLfU1/U2/U5/U7). */
static double axis_u1(const mo_case *c, int l, int m, double dt) {
    const double *u0 = c->u0[0], *vz = c->ph[P_VZ], *vr = c->ph[P_VR], *r = c->r;
    const double dz = c->dz, dr_l = c->dr[l];
    const size_t C = IX(l, m), N = IX(l + 1, m), S = IX(l - 1, m), E = IX(l, m + 1);
    return (0.25 * (u0[N] / r[N] + u0[S] / r[S] + u0[E] / r[E] + u0[C] / r[C])
            + dt * (-(u0[N] / r[N] * vz[N] - u0[S] / r[S] * vz[S]) / (2.0 * dz)
                    - (u0[E] / r[E] * vr[E] - u0[C] / r[C] * vr[E]) / dr_l))
           * r[C];
}

static double axis_u2(const mo_case *c, int l, int m, double dt) {
    const double *u0 = c->u0[1], *vz = c->ph[P_VZ], *vr = c->ph[P_VR], *Hz = c->ph[P_HZ];
    const double *Hr = c->ph[P_HR], *P = c->ph[P_P], *r = c->r;
    const double dz = c->dz, dr_l = c->dr[l];
    const size_t C = IX(l, m), N = IX(l + 1, m), S = IX(l - 1, m), E = IX(l, m + 1);
    return (0.25 * (u0[N] / r[N] + u0[S] / r[S] + u0[E] / r[E] + u0[C] / r[C])
            + dt * (((Hz[N] * Hz[N] - P[N]) - (Hz[S] * Hz[S] - P[S])) / (2.0 * dz)
                    + (Hz[E] * Hr[E] - Hz[C] * Hr[C]) / dr_l
                    - (u0[N] / r[N] * vz[N] - u0[S] / r[S] * vz[S]) / (2.0 * dz)
                    - (u0[E] / r[E] * vr[E] - u0[C] / r[C] * vr[C]) / dr_l))
           * r[C];
}

static double axis_u5(const mo_case *c, int l, int m, double dt) {
    const double *u0 = c->u0[4], *vz = c->ph[P_VZ], *vr = c->ph[P_VR], *p = c->ph[P_p];
    const double *r = c->r;
    const double dz = c->dz, dr_l = c->dr[l];
    const size_t C = IX(l, m), N = IX(l + 1, m), S = IX(l - 1, m), E = IX(l, m + 1);
    return (0.25 * (u0[N] / r[N] + u0[S] / r[S] + u0[E] / r[E] + u0[C] / r[C])
            + dt * (-p[C] * ((vz[N] - vz[S]) / (2.0 * dz) + (vr[E] - vr[C]) / dr_l)
                    - (u0[N] / r[N] * vz[N] - u0[S] / r[S] * vz[S]) / (2.0 * dz)
                    - (u0[E] / r[E] * vr[E] - u0[C] / r[C] * vr[C]) / dr_l))
           * r[C];
}

static double axis_u7(const mo_case *c, int l, int m, double dt) {
    const double *u0 = c->u0[6], *vz = c->ph[P_VZ], *vr = c->ph[P_VR], *Hr = c->ph[P_HR];
    const double *r = c->r;
    const double dr_l = c->dr[l];
    const size_t C = IX(l, m), N = IX(l + 1, m), S = IX(l - 1, m), E = IX(l, m + 1);
    return (0.25 * (u0[N] / r[N] + u0[S] / r[S] + u0[E] / r[E] + u0[C] / r[C])
            + dt * ((Hr[E] * vz[E] - Hr[C] * vz[C]) / dr_l
                    - (u0[E] / r[E] * vr[E] - u0[C] / r[C] * vr[C]) / dr_l))
           * r[C];
}

/* One field: expression value or resolve() (src/bcs/per_field_bc.cpp:286-292). */
static double field_value(segment *s, int k, double cell, double nb) {
    switch (s->type[k]) {
        case T_EXPR: return oe_eval(s->expr[k]);
        case T_NEUMANN: return nb + s->value[k];
        case T_DIRICHLET: return s->value[k];
        default: return cell;
    }
}

/* One boundary cell in the evaluation order rho, v_z, v_r, v_phi, H_z, H_r,
 * H_phi, e (src/bcs/per_field_bc.cpp:319-362, 405-446). */
static void eval_cell(mo_case *c, segment *s, int l, int m, int ln, int mn, double z_l,
                      double dr_l) {
    const size_t i = IX(l, m), nb = IX(ln, mn);
    double **ph = c->ph;
    if (s->has_expr) {
        s->sym[S_DR] = dr_l;
        s->sym[S_R] = c->r[i];
        s->sym[S_RZ] = c->r_z[i];
        s->sym[S_Z] = z_l;
        s->sym[S_RNB] = c->r[nb];
        s->sym[S_RZNB] = c->r_z[nb];
        s->sym[S_RHO_NB] = ph[P_RHO][nb];
        s->sym[S_VZ_NB] = ph[P_VZ][nb];
        s->sym[S_VR_NB] = ph[P_VR][nb];
        s->sym[S_VPHI_NB] = ph[P_VPHI][nb];
        s->sym[S_E_NB] = ph[P_E][nb];
        s->sym[S_HZ_NB] = ph[P_HZ][nb];
        s->sym[S_HR_NB] = ph[P_HR][nb];
        s->sym[S_HPHI_NB] = ph[P_HPHI][nb];
    }
    static const int order_cond[8] = {C_RHO, C_VZ, C_VR, C_VPHI, C_HZ, C_HR, C_HPHI, C_E};
    static const int order_phys[8] = {P_RHO, P_VZ, P_VR, P_VPHI, P_HZ, P_HR, P_HPHI, P_E};
    static const int order_sym[8] = {S_RHO, S_VZ, S_VR, S_VPHI, S_HZ, S_HR, S_HPHI, S_E};
    for (int j = 0; j < 8; ++j) {
        const int k = order_cond[j], pp = order_phys[j];
        const double val = field_value(s, k, ph[pp][i], ph[pp][nb]);
        ph[pp][i] = val;
        if (s->has_expr) s->sym[order_sym[j]] = val;
    }
}

/* src/bcs/per_field_bc.cpp:252-484 (PerFieldBC::Apply), serial cell order. */
static void per_field_apply(mo_case *c, segment *s, int local_lo, int local_hi, double dt) {
    const double dz = c->dz;
    if (s->has_expr) {
        s->sym[S_GAMMA] = c->gamma;
        s->sym[S_BETA] = c->beta;
        s->sym[S_HZ0] = c->H_z0;
        s->sym[S_R0] = c->r_0;
        s->sym[S_DZ] = dz;
        s->sym[S_DR] = 0.0;
    }
    if (s->face == F_L_LO || s->face == F_L_HI) {
        const int l = s->face == F_L_LO ? 1 : c->L;
        const int ln = s->face == F_L_LO ? 2 : c->L - 1;
        const int l_global = l - 1;
        const double z_l = l_global * dz;
        for (int m = local_lo; m <= local_hi; ++m) {
            eval_cell(c, s, l, m, ln, m, z_l, c->dr[l]);
            rebuild_u(c, l, m);
        }
        return;
    }
    const int m = s->face == F_M_LO ? 1 : c->M + 1;
    const int mn = s->face == F_M_LO ? 2 : c->M;
    for (int l = local_lo; l <= local_hi; ++l) {
        const int l_global = l - 1;
        const double z_l = l_global * dz;
        eval_cell(c, s, l, m, l, mn, z_l, c->dr[l]);
        rebuild_u(c, l, m);
        if (s->has_axis) {
            const size_t i = IX(l, m);
            if (s->type[C_RHO] == T_AXISLF) c->u[0][i] = axis_u1(c, l, m, dt);
            if (s->type[C_VZ] == T_AXISLF) c->u[1][i] = axis_u2(c, l, m, dt);
            if (s->type[C_E] == T_AXISLF) c->u[4][i] = axis_u5(c, l, m, dt);
            if (s->type[C_HZ] == T_AXISLF) c->u[6][i] = axis_u7(c, l, m, dt);
        }
    }
}

/* src/face_bc.cpp:104-129 (FaceBC::Apply) with FaceGlobalRange/ClipToLocal
 * for a single rank that owns every face. */
static void face_apply(mo_case *c, int face, double dt) {
    const int is_l = face == F_L_LO || face == F_L_HI;
    const int face_lo = 0, face_hi = is_l ? c->M : c->L - 1;
    const int owned_lo = 0, owned_hi = is_l ? c->M : c->L - 1;
    for (int k = 0; k < c->nseg[face]; ++k) {
        segment *s = &c->seg[face][k];
        const int g_lo = s->glo < 0 ? face_lo : s->glo;
        const int g_hi = s->ghi < 0 ? face_hi : s->ghi;
        const int clo = g_lo > owned_lo ? g_lo : owned_lo;
        const int chi = g_hi < owned_hi ? g_hi : owned_hi;
        if (clo > chi) continue;
        int local_lo = clo - owned_lo + 1, local_hi = chi - owned_lo + 1;
        if (face == F_M_LO) {
            if (local_lo < 2) local_lo = 2;
            if (local_hi > c->L - 1) local_hi = c->L - 1;
            if (local_lo > local_hi) continue;
        }
        per_field_apply(c, s, local_lo, local_hi, dt);
    }
}

/* src/solver.cpp:22-37 (Solver::Advance); ghost exchange is a no-op on one rank. */
void mo_advance(mo_case *c, double dt) {
    central_update(c, dt);
    update_physical(c, 1, c->L, 2, c->M);
    face_apply(c, F_L_LO, dt);
    face_apply(c, F_M_HI, dt);
    face_apply(c, F_M_LO, dt);
    face_apply(c, F_L_HI, dt);
    update_physical(c, 1, c->L, 1, c->M + 1);
    /* src/fields.cpp:102-115 (Fields::CopyUToU0), every cell incl. ghosts */
    const size_t n = (size_t)c->rows * (size_t)c->cols;
    for (int k = 0; k < 8; ++k) memcpy(c->u0[k], c->u[k], n * sizeof(double));
}

/* ------------------------------------------------------------ reductions */

static double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */
static double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */

/* src/diagnostics.cpp:14-43 */
double mo_max_wave_speed(const mo_case *c) {
    double local_max = 0.0;
    double *const *f = c->ph;
    for (int l = 1; l <= c->L; ++l)
        for (int m = 1; m <= c->M + 1; ++m) {
            const size_t i = IX(l, m);
            const double cs = sqrt(c->gamma * f[P_p][i] / f[P_RHO][i]);
            const double ca = sqrt((f[P_HZ][i] * f[P_HZ][i] + f[P_HR][i] * f[P_HR][i]
                                    + f[P_HPHI][i] * f[P_HPHI][i]) / f[P_RHO][i]);
            const double v = sqrt(f[P_VZ][i] * f[P_VZ][i] + f[P_VR][i] * f[P_VR][i]);
            local_max = dmax(local_max, v + cs + ca);
        }
    return local_max;
}

/* src/diagnostics.cpp:49-65 */
double mo_compute_dt(const mo_case *c, double cfl, double growth, double dt_min, double dt_max,
                     double dt_current) {
    const double speed = mo_max_wave_speed(c);
    const double dx = dmin(c->dz, c->dy);
    const double dt_cfl = cfl * dx / (speed + 1.0e-10);
    const double dt_grown = dt_current * growth;
    const double v = dmin(dt_cfl, dt_grown);
    return (v < dt_min) ? dt_min : ((dt_max < v) ? dt_max : v); /* std::clamp */
}

/* src/diagnostics.cpp:71-106, serial summation order */
double mo_solution_change(const mo_case *c) {
    if (!c->with_prev) return 0.0;
    double sum_diff = 0.0, sum_curr = 0.0;
    static const int pk[7] = {P_RHO, P_VZ, P_VR, P_VPHI, P_HZ, P_HR, P_HPHI};
    for (int l = 1; l <= c->L; ++l)
        for (int m = 1; m <= c->M + 1; ++m) {
            const size_t i = IX(l, m);
            double d[7], x[7];
            for (int k = 0; k < 7; ++k) {
                x[k] = c->ph[pk[k]][i];
                d[k] = x[k] - c->prev[k][i];
            }
            sum_diff += d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + d[3] * d[3] + d[4] * d[4]
                      + d[5] * d[5] + d[6] * d[6];
            sum_curr += x[0] * x[0] + x[1] * x[1] + x[2] * x[2] + x[3] * x[3] + x[4] * x[4]
                      + x[5] * x[5] + x[6] * x[6];
        }
    const double norm_diff = sqrt(sum_diff);
    const double norm_curr = sqrt(sum_curr);
    return (norm_curr > 1e-15) ? (norm_diff / norm_curr) : norm_diff;
}

/* src/fields.cpp:59-74 */
void mo_save_prev(mo_case *c) {
    if (!c->with_prev) return;
    static const int pk[7] = {P_RHO, P_VZ, P_VR, P_VPHI, P_HZ, P_HR, P_HPHI};
    const size_t n = (size_t)c->rows * (size_t)c->cols;
    for (int k = 0; k < 7; ++k) memcpy(c->prev[k], c->ph[pk[k]], n * sizeof(double));
}

/* src/verification.cpp:16-45 */
void mo_integrals(const mo_case *c, double *out7) {
    double local[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int l = 1; l <= c->L; ++l) {
        const double cell_area = c->dr[l] * c->dz;
        for (int m = 1; m <= c->M + 1; ++m) {
            const size_t i = IX(l, m);
            local[0] += c->u0[0][i] * cell_area;
            local[1] += c->u0[1][i] * cell_area;
            local[2] += c->u0[2][i] * cell_area;
            local[3] += c->u0[3][i] * cell_area;
            local[4] += c->u0[4][i] * cell_area;
            local[5] += c->u0[6][i] * cell_area;
            local[6] += c->u0[5][i] * cell_area;
        }
    }
    memcpy(out7, local, sizeof(local));
}

/* src/integrals.cpp:45-112 */
void mo_outlet(const mo_case *c, double *mass_flux, double *thrust) {
    const double inv_8pi = 1.0 / (8.0 * M_PI);
    const int l = c->L;
    const double dr_out = c->dr[l];
    double sm = 0.0, st = 0.0;
    double *const *f = c->ph;
    for (int m_local = 1; m_local <= c->M + 1; ++m_local) {
        const int m_global = m_local - 1;
        const double w = (m_global == 0 || m_global == c->M) ? 0.5 : 1.0;
        const size_t i = IX(l, m_local);
        const double fm = f[P_RHO][i] * f[P_VZ][i];
        const double Fm = fm * 2.0 * M_PI * c->r[i];
        sm += w * Fm * dr_out;
        const double v_z2 = f[P_VZ][i] * f[P_VZ][i];
        const double H2 = f[P_HZ][i] * f[P_HZ][i] + f[P_HR][i] * f[P_HR][i]
                        + f[P_HPHI][i] * f[P_HPHI][i];
        const double ft = f[P_RHO][i] * v_z2 + f[P_p][i] + H2 * inv_8pi;
        const double Ft = ft * 2.0 * M_PI * c->r[i];
        st += w * Ft * dr_out;
    }
    *mass_flux = sm;
    *thrust = st;
}

/* src/verification.cpp:121-146 */
double mo_radial_symmetry(const mo_case *c) {
    double local_max = 0.0;
    for (int l = 1; l <= c->L; ++l)
        for (int m = 1; m < c->M + 1; ++m) {
            const double a = c->ph[P_RHO][IX(l, m)];
            const double b = c->ph[P_RHO][IX(l, m + 1)];
            const double mean = 0.5 * (a + b);
            if (mean > 1.0e-15) local_max = dmax(local_max, fabs(b - a) / mean);
        }
    return local_max;
}

void mo_get(const mo_case *c, int which, double *out) {
    const size_t n = (size_t)c->rows * (size_t)c->cols;
    const double *src = NULL;
    if (which >= 0 && which < 8) src = c->u0[which];
    else if (which >= 8 && which < 18) src = c->ph[which - 8];
    else if (which == 18) src = c->r;
    else if (which == 19) src = c->r_z;
    if (src) memcpy(out, src, n * sizeof(double));
}

/* src/main.cpp:191-282 */
void mo_run(mo_case *c, const double *run, double *out) {
    const double T = run[0];
    double dt = run[1];
    const int adaptive = run[2] != 0.0;
    const double cfl = run[3], growth = run[4], dt_min = run[5], dt_max = run[6];
    const double thr = run[7];
    const int check_freq = (int)run[8];
    const long max_steps = (long)run[9];
    double t = 0.0, change = 0.0;
    long step = 0;
    int converged = 0;
    while (t < T && !converged && step < max_steps) {
        if (t + dt > T) dt = T - t;
        mo_advance(c, dt);
        t += dt;
        ++step;
        if (adaptive) dt = mo_compute_dt(c, cfl, growth, dt_min, dt_max, dt);
        if (thr > 0.0 && step % check_freq == 0) {
            change = mo_solution_change(c);
            if (change < thr) converged = 1;
            mo_save_prev(c);
        }
    }
    out[0] = (double)step;
    out[1] = t;
    out[2] = dt;
    out[3] = converged;
    out[4] = change;
}
