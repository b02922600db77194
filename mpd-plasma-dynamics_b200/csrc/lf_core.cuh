// Core per-cell arithmetic of the Lax-Friedrichs hot path.
//
// Every function here is host+device (MPD_HD) so that the exact same source
// runs inside the CUDA kernels and inside the host emulator that the CPU test
// suite drives.  The whole library is compiled with --fmad=false /
// -ffp-contract=off: in the "exact" functions each expression is one IEEE-754
// operation per operator, in the reference's operand order, with true
// divides, which makes them bit-identical to the reference.  The "fast"
// interior kernel (lf_fast.cuh) opts into FMA explicitly.
//
// Storage: conserved planes u_1..u_8 in structure-of-arrays layout, plane k
// at base + k*ps, cell (l, m) at l*pitch + m; the reference's (L+2)x(M+3)
// index space with one ghost layer (single rank: ghosts stay zero).
#pragma once

#include <math.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __CUDACC__
#define MPD_HD __host__ __device__ __forceinline__
#define MPD_HD_NOINLINE __host__ __device__ __noinline__
#else
#define MPD_HD inline
#define MPD_HD_NOINLINE inline
#endif

#include "expr_ops.h"

namespace mpd {

constexpr int kNumCons = 8;
constexpr int kNumPhys = 10;
constexpr int kMaxSegments = 32;  // all faces together

// Physical plane order = Fields members (include/fields.hpp:35-37).
enum PhysIdx { P_RHO = 0, P_VZ, P_VR, P_VPHI, P_E, P_PG, P_PT, P_HZ, P_HR, P_HPHI };
// Boundary field evaluation order (src/bcs/per_field_bc.cpp:319-362):
// rho, v_z, v_r, v_phi, H_z, H_r, H_phi, e.
enum PrimIdx { Q_RHO = 0, Q_VZ, Q_VR, Q_VPHI, Q_HZ, Q_HR, Q_HPHI, Q_E };
enum FaceIdx { FACE_L_LO = 0, FACE_L_HI = 1, FACE_M_LO = 2, FACE_M_HI = 3 };
enum CondType { COND_NEUMANN = 0, COND_DIRICHLET = 1, COND_EXPR = 2, COND_AXIS_LF = 3 };

// Boundary expression symbols (PerFieldBC::ExprImpl, src/bcs/per_field_bc.cpp:81-119).
enum BcSym {
    BS_GAMMA = 0, BS_BETA, BS_HZ0, BS_R0, BS_DZ, BS_DR, BS_R, BS_RZ, BS_Z, BS_RNB, BS_RZNB,
    BS_NB0,            // rho_nb, v_z_nb, v_r_nb, v_phi_nb, e_nb, H_z_nb, H_r_nb, H_phi_nb
    BS_CUR0 = BS_NB0 + 8,  // rho, v_z, v_r, v_phi, H_z, H_r, H_phi, e (evaluation order)
    BS_COUNT = BS_CUR0 + 8
};

// Expression initial-condition symbols (ExpressionIC::Impl,
// src/ics/expression_ic.cpp:84-126): the fields in evaluation order.
enum IcSym { IC_GAMMA = 0, IC_BETA, IC_HZ0, IC_R0, IC_Z, IC_R, IC_RZ, IC_F0, IC_COUNT = IC_F0 + 8 };

struct Phys {
    double rho, vz, vr, vphi, e, p, P, Hz, Hr, Hphi;
};

// Grid geometry: Grid::Build (src/grid.cpp:20-42) recomputed on the fly from
// the wall profiles, so no r plane is stored.
struct Geo {
    int L, M, pitch;
    size_t ps;  // plane stride (doubles)
    double dz, dy, gamma, beta, H_z0, r_0;
    const double *rin, *rout, *drin, *drout, *dr;  // per row l = 0..L+1
    const double *hdr;  // 0.5 / dr per row (the fast interior's r-difference factor)

    MPD_HD size_t ix(int l, int m) const { return (size_t)l * (size_t)pitch + (size_t)m; }
    MPD_HD double r(int l, int m) const {
        const double frac = (double)(m - 1) * dy;
        return (1.0 - frac) * rin[l] + frac * rout[l];
    }
    MPD_HD double rz(int l, int m) const {
        const double frac = (double)(m - 1) * dy;
        return (1.0 - frac) * drin[l] + frac * drout[l];
    }
};

MPD_HD void load_cons(const double *base, size_t ps, size_t i, double u[8]) {
#pragma unroll
    for (int k = 0; k < 8; ++k) u[k] = base[(size_t)k * ps + i];
}

// Fields::UpdatePhysicalFromU (src/fields.cpp:76-99), one cell.
MPD_HD Phys recon_exact(const double u[8], double r, double gamma) {
    Phys q;
    q.rho = u[0] / r;
    q.vz = u[1] / u[0];
    q.vr = u[2] / u[0];
    q.vphi = u[3] / u[0];
    q.Hphi = u[5];
    q.Hz = u[6] / r;
    q.Hr = u[7] / r;
    q.e = u[4] / u[0];
    q.p = (gamma - 1.0) * q.rho * q.e;
    q.P = q.p + 0.5 * (q.Hz * q.Hz + q.Hr * q.Hr + q.Hphi * q.Hphi);
    return q;
}

MPD_HD Phys phys_zero() {
    Phys q;
    q.rho = q.vz = q.vr = q.vphi = q.e = q.p = q.P = q.Hz = q.Hr = q.Hphi = 0.0;
    return q;
}

MPD_HD Phys load_phys(const double *base, size_t ps, size_t i) {
    Phys q;
    q.rho = base[0 * ps + i];
    q.vz = base[1 * ps + i];
    q.vr = base[2 * ps + i];
    q.vphi = base[3 * ps + i];
    q.e = base[4 * ps + i];
    q.p = base[5 * ps + i];
    q.P = base[6 * ps + i];
    q.Hz = base[7 * ps + i];
    q.Hr = base[8 * ps + i];
    q.Hphi = base[9 * ps + i];
    return q;
}

// include/physics_utils.hpp:15-24 (RebuildUFromPhysical), one cell.
MPD_HD void rebuild_u(const Phys &q, double r, double u[8]) {
    u[0] = q.rho * r;
    u[1] = q.rho * q.vz * r;
    u[2] = q.rho * q.vr * r;
    u[3] = q.rho * q.vphi * r;
    u[4] = q.rho * q.e * r;
    u[5] = q.Hphi;
    u[6] = q.Hz * r;
    u[7] = q.Hr * r;
}

// One term of Diagnostics::MaxWaveSpeed (src/diagnostics.cpp:25-35).
MPD_HD double wave_speed(const Phys &q, double gamma) {
    const double cs = sqrt(gamma * q.p / q.rho);
    const double ca = sqrt((q.Hz * q.Hz + q.Hr * q.Hr + q.Hphi * q.Hphi) / q.rho);
    const double v = sqrt(q.vz * q.vz + q.vr * q.vr);
    return v + cs + ca;
}

// Diagnostics::ComputeDt clamp arithmetic (src/diagnostics.cpp:57-64) with
// std::min / std::clamp comparison semantics.
MPD_HD double compute_dt_from_speed(double speed, double dz, double dy, double cfl,
                                    double growth, double dt_min, double dt_max,
                                    double dt_current) {
    const double dx = (dy < dz) ? dy : dz;
    const double dt_cfl = cfl * dx / (speed + 1.0e-10);
    const double dt_grown = dt_current * growth;
    const double v = (dt_grown < dt_cfl) ? dt_grown : dt_cfl;
    return (v < dt_min) ? dt_min : ((dt_max < v) ? dt_max : v);
}

// ---------------------------------------------------------------------------
// Solver::ComputeCentralUpdate (src/solver.cpp:59-153) for one cell, exact.
// Stencil points: 0 = (l,m), 1 = (l+1,m), 2 = (l-1,m), 3 = (l,m+1), 4 = (l,m-1).
// U[p][k] conserved u0 values, Q[p] physical values, R[p] radius.
// ---------------------------------------------------------------------------
MPD_HD void lf_cell_exact(const double U[5][8], const Phys Q[5], const double R[5], double dt,
                          double dz, double dr_l, double out[8]) {
    enum { C = 0, N = 1, S = 2, E = 3, W = 4 };
#define UA(p) U[p][kk]
    {
        const int kk = 0;
        out[0] = 0.25 * (UA(N) + UA(S) + UA(E) + UA(W))
               + dt * (-(UA(N) * Q[N].vz - UA(S) * Q[S].vz) / (2 * dz)
                       - (UA(E) * Q[E].vr - UA(W) * Q[W].vr) / (2 * dr_l));
    }
    {
        const int kk = 1;
        out[1] = 0.25 * (UA(N) + UA(S) + UA(E) + UA(W))
               + dt * (((Q[N].Hz * Q[N].Hz - Q[N].P) * R[N] - (Q[S].Hz * Q[S].Hz - Q[S].P) * R[S]) / (2 * dz)
                       + (Q[E].Hz * Q[E].Hr * R[E] - Q[W].Hz * Q[W].Hr * R[W]) / (2 * dr_l)
                       - (UA(N) * Q[N].vz - UA(S) * Q[S].vz) / (2 * dz)
                       - (UA(E) * Q[E].vr - UA(W) * Q[W].vr) / (2 * dr_l));
    }
    {
        const int kk = 2;
        out[2] = 0.25 * (UA(N) + UA(S) + UA(E) + UA(W))
               + dt * ((Q[C].rho * Q[C].vphi * Q[C].vphi + Q[C].P - Q[C].Hphi * Q[C].Hphi)
                       + (Q[N].Hz * Q[N].Hr * R[N] - Q[S].Hz * Q[S].Hr * R[S]) / (2 * dz)
                       + ((Q[E].Hr * Q[E].Hr - Q[E].P) * R[E] - (Q[W].Hr * Q[W].Hr - Q[W].P) * R[W]) / (2 * dr_l)
                       - (UA(N) * Q[N].vz - UA(S) * Q[S].vz) / (2 * dz)
                       - (UA(E) * Q[E].vr - UA(W) * Q[W].vr) / (2 * dr_l));
    }
    {
        const int kk = 3;
        out[3] = 0.25 * (UA(N) + UA(S) + UA(E) + UA(W))
               + dt * ((-Q[C].rho * Q[C].vr * Q[C].vphi + Q[C].Hphi * Q[C].Hr)
                       + (Q[N].Hphi * Q[N].Hz * R[N] - Q[S].Hphi * Q[S].Hz * R[S]) / (2 * dz)
                       + (Q[E].Hphi * Q[E].Hr * R[E] - Q[W].Hphi * Q[W].Hr * R[W]) / (2 * dr_l)
                       - (UA(N) * Q[N].vz - UA(S) * Q[S].vz) / (2 * dz)
                       - (UA(E) * Q[E].vr - UA(W) * Q[W].vr) / (2 * dr_l));
    }
    {
        const int kk = 4;
        out[4] = 0.25 * (UA(N) + UA(S) + UA(E) + UA(W))
               + dt * (-Q[C].p * ((Q[N].vz * R[N] - Q[S].vz * R[S]) / (2 * dz)
                                  + (Q[E].vr * R[E] - Q[W].vr * R[W]) / (2 * dr_l))
                       - (UA(N) * Q[N].vz - UA(S) * Q[S].vz) / (2 * dz)
                       - (UA(E) * Q[E].vr - UA(W) * Q[W].vr) / (2 * dr_l));
    }
    {
        const int kk = 5;
        out[5] = 0.25 * (UA(N) + UA(S) + UA(E) + UA(W))
               + dt * ((Q[N].Hz * Q[N].vphi - Q[S].Hz * Q[S].vphi) / (2 * dz)
                       + (Q[E].Hr * Q[E].vphi - Q[W].Hr * Q[W].vphi) / (2 * dr_l)
                       - (UA(N) * Q[N].vz - UA(S) * Q[S].vz) / (2 * dz)
                       - (UA(E) * Q[E].vr - UA(W) * Q[W].vr) / (2 * dr_l));
    }
    {
        const int kk = 6;
        out[6] = 0.25 * (UA(N) + UA(S) + UA(E) + UA(W))
               + dt * ((Q[E].Hr * Q[E].vz * R[E] - Q[W].Hr * Q[W].vz * R[W]) / (2 * dr_l)
                       - (UA(E) * Q[E].vr - UA(W) * Q[W].vr) / (2 * dr_l));
    }
    {
        const int kk = 7;
        out[7] = 0.25 * (UA(N) + UA(S) + UA(E) + UA(W))
               + dt * ((Q[N].Hz * Q[N].vr * R[N] - Q[S].Hz * Q[S].vr * R[S]) / (2 * dz)
                       - (UA(N) * Q[N].vz - UA(S) * Q[S].vz) / (2 * dz));
    }
#undef UA
}

// ---------------------------------------------------------------------------
// Fast-mode arithmetic (MPD_PRECISION_FAST, lf_fast.cuh).
//
// Same update as lf_cell_exact, reorganised so that every stencil point is
// evaluated once and its contributions are folded into running sums:
//   out_k(l) = A_k(l) + B_k(l) + 0.25 U_k(l+1) + kz Gz_k(l+1)
// with  A_k(l) = 0.25 U_k(l-1) - kz Gz_k(l-1)          (z neighbour below)
//       B_k(l) = (U_k(m+1)/4 + kr Gr_k(m+1)) + (U_k(m-1)/4 - kr Gr_k(m-1))
//                + dt S_k(l)                           (r neighbours, sources)
// kz = dt / (2 dz), kr = dt / (2 dr_l); Gz / Gr are each equation's z / r
// flux combination at a point (index 6 of Gz, free because u_7 has no z flux,
// carries v_z r; index 7 of Gr, free because u_8 has no r flux, carries v_r r;
// both feed u_5's -p div(r v) source).  Divides become reciprocals: the
// hardware's double-precision seed with one polynomial correction (rcp_nr).
// ---------------------------------------------------------------------------

// 1/x from a seed y0 = (1 - e) / x: y0 (1 + e + e^2) = (1 - e^3) / x, three
// dependent FMAs.  On the device the seed is the hardware's double-precision
// reciprocal approximation (rcp.approx.ftz.f64: no conversions, any normal
// double), measured on a B200 at |e| <= 2^-19.9 over 2^28 inputs across
// exponents -60..60, so e^3 <= 2^-59 is below double rounding; on the host a
// single-precision reciprocal (|e| <= 2^-24).
MPD_HD double rcp_nr(double x) {
#ifdef __CUDA_ARCH__
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
#else
    double y = (double)(1.0f / (float)x);
#endif
    const double e = fma(-x, y, 1.0);
    return fma(y, fma(e, e, e), y);
}

// sqrt(a) (0 -> 0, a < 0 -> NaN) from a 1/sqrt seed y0: with t = a y0 and
// d = 1 - t y0, sqrt(a) = t (1 - d)^(-1/2) = t (1 + d/2 + 3 d^2 / 8 + ...); the
// two terms kept leave 5 d^3 / 16.  Device seed: rsqrt.approx.ftz.f64, measured
// at 2^-20.0 relative (d <= 2^-19, so 5 d^3 / 16 <= 2^-58); host seed: single
// precision.
MPD_HD double sqrt_nr(double a) {
#ifdef __CUDA_ARCH__
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
#else
    double y = (double)(1.0f / sqrtf((float)a));
#endif
    const double t = a * y;
    const double d = fma(-t, y, 1.0);
    const double out = fma(t, d * fma(d, 0.375, 0.5), t);
    return a > 0.0 ? out : (a == 0.0 ? 0.0 : NAN);
}

// Primitive values of one point (Fields::UpdatePhysicalFromU with reciprocals).
struct FastPrim {
    double rho, vz, vr, vphi, e, Hphi, Hz, Hr, p, P;
    double ir;  // 1 / r of the point
};

// zero_iu: a ghost point (U = 0): 1/u_1 taken as 0, so that every value is 0.
MPD_HD FastPrim fast_prim(const double U[8], double r, double gm1, bool zero_iu = false) {
    FastPrim q;
    const double ir = rcp_nr(r);
    const double iu = zero_iu ? 0.0 : rcp_nr(U[0]);
    q.rho = U[0] * ir;
    q.vz = U[1] * iu;
    q.vr = U[2] * iu;
    q.vphi = U[3] * iu;
    q.e = U[4] * iu;
    q.Hphi = U[5];
    q.Hz = U[6] * ir;
    q.Hr = U[7] * ir;
    q.p = gm1 * q.rho * q.e;
    q.P = fma(0.5, fma(q.Hz, q.Hz, fma(q.Hr, q.Hr, q.Hphi * q.Hphi)), q.p);
    q.ir = ir;
    return q;
}

// z flux combination of each equation at a point (Gz[6] = v_z r).
MPD_HD void fast_gz(const double U[8], const FastPrim &q, double r, double Gz[8]) {
    Gz[0] = -U[0] * q.vz;
    Gz[1] = fma(fma(q.Hz, q.Hz, -q.P), r, -U[1] * q.vz);
    Gz[2] = fma(q.Hz * q.Hr, r, -U[2] * q.vz);
    Gz[3] = fma(q.Hphi * q.Hz, r, -U[3] * q.vz);
    Gz[4] = -U[4] * q.vz;
    Gz[5] = fma(q.Hz, q.vphi, -U[5] * q.vz);
    Gz[6] = q.vz * r;
    Gz[7] = fma(q.Hz * q.vr, r, -U[7] * q.vz);
}

// r flux combination of each equation at a point (Gr[7] = v_r r).
MPD_HD void fast_gr(const double U[8], const FastPrim &q, double r, double Gr[8]) {
    Gr[0] = -U[0] * q.vr;
    Gr[1] = fma(q.Hz * q.Hr, r, -U[1] * q.vr);
    Gr[2] = fma(fma(q.Hr, q.Hr, -q.P), r, -U[2] * q.vr);
    Gr[3] = fma(q.Hphi * q.Hr, r, -U[3] * q.vr);
    Gr[4] = -U[4] * q.vr;
    Gr[5] = fma(q.Hr, q.vphi, -U[5] * q.vr);
    Gr[6] = fma(q.Hr * q.vz, r, -U[6] * q.vr);
    Gr[7] = q.vr * r;
}

// A(l+1) from point row l: A[k] = U/4 - kz Gz (u_7: U/4); A[8] = v_z r.
MPD_HD void fast_a(const double U[8], const double Gz[8], double kz, double A[9]) {
#pragma unroll
    for (int k = 0; k < 8; ++k) A[k] = (k == 6) ? 0.25 * U[6] : fma(-kz, Gz[k], 0.25 * U[k]);
    A[8] = Gz[6];
}

// A point's shares of its r neighbours' B: ce (seen from the cell to its west,
// as that cell's east neighbour) = U/4 + kr Gr and cw (seen from the cell to
// its east) = U/4 - kr Gr; for u_8, U/4 alone (its r term is u_5's source).
MPD_HD void fast_rc(const double U[8], const double Gr[8], double kr, double ce[8],
                    double cw[8]) {
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        const double q = 0.25 * U[k];
        ce[k] = fma(kr, Gr[k], q);
        cw[k] = fma(-kr, Gr[k], q);
    }
    ce[7] = cw[7] = 0.25 * U[7];
}

// B(l) from the east neighbour's ce, the west neighbour's cw, their v_r r
// (g7e, g7w) and the point's own sources; B[8] = p.
MPD_HD void fast_b(const double ce_e[8], const double cw_w[8], double g7e, double g7w,
                   const FastPrim &q, double kr, double dt, double B[9]) {
#pragma unroll
    for (int k = 0; k < 8; ++k) B[k] = ce_e[k] + cw_w[k];
    B[2] = fma(dt, fma(q.rho * q.vphi, q.vphi, q.P) - q.Hphi * q.Hphi, B[2]);
    B[3] = fma(dt, fma(-q.rho * q.vr, q.vphi, q.Hphi * q.Hr), B[3]);
    // r part of u_5's source -p kr (v_r r)_e - (v_r r)_w
    B[4] = fma(-q.p * kr, g7e - g7w, B[4]);
    B[8] = q.p;
}

// The running sums of cell row l once its own point row has been folded in:
// S[k] = A[k] + B[k] (k < 8), S[8] = p (B[8]), S[9] = v_z r of the point row
// below (A[8]).
MPD_HD void fast_sum(const double A[9], const double B[9], double S[10]) {
#pragma unroll
    for (int k = 0; k < 8; ++k) S[k] = A[k] + B[k];
    S[8] = B[8];
    S[9] = A[8];
}

// Close cell row l (sums S) with point row l+1 (U, Gz).
MPD_HD void fast_finish(const double S[10], const double Un[8], const double Gzn[8], double kz,
                        double out[8]) {
#pragma unroll
    for (int k = 0; k < 8; ++k)
        out[k] = (k == 6) ? fma(0.25, Un[6], S[k]) : fma(kz, Gzn[k], fma(0.25, Un[k], S[k]));
    // z part of u_5's source: -p kz ((v_z r)_n - (v_z r)_s)
    out[4] = fma(-S[8] * kz, Gzn[6] - S[9], out[4]);
}

// Wave speed |v| + c_s + c_a of a new cell state at radius r (ir = 1 / r),
// with reciprocals and seeded square roots (rcp_nr, sqrt_speed):
//   |v|^2 = (u_2^2 + u_3^2) / u_1^2,  c_s^2 = gamma (gamma - 1) u_5 / u_1,
//   c_a^2 = (H_z^2 + H_r^2 + H_phi^2) r / u_1   (u_1 = rho r, u_5 = rho e r).
// The wave speed's square roots, without special cases: the argument is
// nudged by 1e-300, which leaves every argument above 1e-284 unchanged (it is
// below half an ulp), turns 0 into a root of 1e-150 that vanishes in the
// sum, and keeps a negative argument's NaN (an unphysical state, caught by
// the non-finite check).
MPD_HD double sqrt_speed(double a) {
    a += 1e-300;
#ifdef __CUDA_ARCH__
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
#else
    double y = (double)(1.0f / sqrtf((float)a));
#endif
    const double t = a * y;
    const double d = fma(-t, y, 1.0);
    return fma(t, d * fma(d, 0.375, 0.5), t);
}

MPD_HD double fast_wave_speed(const double u[8], double r, double ir, double gamma) {
    const double iu = rcp_nr(u[0]);
    const double vz = u[1] * iu, vr = u[2] * iu;
    const double Hz = u[6] * ir, Hr = u[7] * ir, Hphi = u[5];
    const double cs2 = gamma * (gamma - 1.0) * u[4] * iu;
    const double ca2 = fma(Hz, Hz, fma(Hr, Hr, Hphi * Hphi)) * (r * iu);
    const double v2 = fma(vz, vz, vr * vr);
    return sqrt_speed(v2) + sqrt_speed(cs2) + sqrt_speed(ca2);
}

// ---------------------------------------------------------------------------
// Expression bytecode interpreter (codes from expr.cpp).
// ---------------------------------------------------------------------------
MPD_HD double eval_code(const int32_t *code, const double *consts, const double *sym) {
    double st[kExprMaxStack];
    int sp = 0;
    for (int pc = 0;; ++pc) {
        const int32_t ins = code[pc];
        const int op = ins & 0xff;
        const int arg = ins >> 8;
        switch (op) {
            case OP_END: return sp > 0 ? st[sp - 1] : 0.0;
            case OP_CONST: st[sp++] = consts[arg]; break;
            case OP_VAR: st[sp++] = sym[arg]; break;
            case OP_NEG: st[sp - 1] = -st[sp - 1]; break;
            case OP_ADD: st[sp - 2] = st[sp - 2] + st[sp - 1]; --sp; break;
            case OP_SUB: st[sp - 2] = st[sp - 2] - st[sp - 1]; --sp; break;
            case OP_MUL: st[sp - 2] = st[sp - 2] * st[sp - 1]; --sp; break;
            case OP_DIV: st[sp - 2] = st[sp - 2] / st[sp - 1]; --sp; break;
            case OP_MOD: st[sp - 2] = fmod(st[sp - 2], st[sp - 1]); --sp; break;
            case OP_POW: st[sp - 2] = pow(st[sp - 2], st[sp - 1]); --sp; break;
            case OP_ATAN2: st[sp - 2] = atan2(st[sp - 2], st[sp - 1]); --sp; break;
            case OP_MIN2: {
                const double y = st[sp - 1], x = st[sp - 2];
                st[sp - 2] = y < x ? y : x;
                --sp;
                break;
            }
            case OP_MAX2: {
                const double y = st[sp - 1], x = st[sp - 2];
                st[sp - 2] = y > x ? y : x;
                --sp;
                break;
            }
            case OP_CLAMP: {
                const double lo = st[sp - 3], v = st[sp - 2], hi = st[sp - 1];
                st[sp - 3] = v < lo ? lo : (v > hi ? hi : v);
                sp -= 2;
                break;
            }
            case OP_FN1: {
                const double x = st[sp - 1];
                double y;
                switch (arg) {
                    case FN_SIN: y = sin(x); break;
                    case FN_COS: y = cos(x); break;
                    case FN_TAN: y = tan(x); break;
                    case FN_ASIN: y = asin(x); break;
                    case FN_ACOS: y = acos(x); break;
                    case FN_ATAN: y = atan(x); break;
                    case FN_EXP: y = exp(x); break;
                    case FN_LOG: y = log(x); break;
                    case FN_LOG2: y = log2(x); break;
                    case FN_LOG10: y = log10(x); break;
                    case FN_SQRT: y = sqrt(x); break;
                    case FN_ABS: y = fabs(x); break;
                    default: y = x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); break;
                }
                st[sp - 1] = y;
                break;
            }
            default: return NAN;
        }
    }
}

// ---------------------------------------------------------------------------
// Boundary conditions (FaceBC + PerFieldBC) for one boundary cell.
// ---------------------------------------------------------------------------

// One segment, compiled: local inclusive range along the face's free axis
// after FaceBC::Apply's sentinel resolution, ClipToLocal and the M_LO corner
// policy (src/face_bc.cpp:104-129); conditions in evaluation order.
// Closed forms of expression fields, found by the host compiler: a folded
// constant, or one binary operation on two operands (symbols or constants).
// Anything else runs through the bytecode interpreter.
enum ExprForm { EF_GENERAL = 0, EF_CONST = 1, EF_BIN = 2 };

struct SegDesc {
    int lo, hi;
    int has_axis;
    int pad;
    int type[8];
    int code[8];      // offset of the expression's bytecode, -1 if none
    double value[8];
    int form[8];      // ExprForm of an expression field
    int fop[8];       // OP_ADD / OP_SUB / OP_MUL / OP_DIV for EF_BIN
    int fa[8], fb[8]; // operand symbols (BcSym), -1 for a constant operand
    double ca[8], cb[8];  // constant operands; ca is the value of EF_CONST
};

struct BcTable {
    int nseg[4];
    int first[4];             // index of the face's first segment in seg[]
    const SegDesc *seg;
    const int32_t *code;
    const double *consts;
    int nseg_total, ncode, nconst;
};

// Values of the cells the boundary faces read, laid out as "lines" along one
// grid row or column (field stride len).
//   central lines (the interior kernel's new conserved values, 8 fields, of
//   the cells the faces read; the boundary kernel reconstructs them):
//   0 = row 2 by m, 1 = row L-1 by m, 2 = column 2 by l, 3 = column M by l
//   (its entries l = 1 and l = L are (1,M) and (L,M) before the L faces
//   overwrite them);
//   wall lines (10 physical fields in Phys order, line stride 10 * len: the
//   previous step's full reconstruction of the wall columns, written by the
//   boundary kernel; the initial condition on step 0):
//   0 = column 1 by l, 1 = column M+1 by l.
constexpr int kCentralLines = 4;
constexpr int kWallLines = 2;

MPD_HD int line_len(int L, int M) { return (L + 2 > M + 3) ? L + 2 : M + 3; }

MPD_HD Phys line_phys(const double *lines, int len, int line, int idx) {
    const double *b = lines + (size_t)line * 10 * len + idx;
    Phys q;
    q.rho = b[0 * len];
    q.vz = b[1 * len];
    q.vr = b[2 * len];
    q.vphi = b[3 * len];
    q.e = b[4 * len];
    q.p = b[5 * len];
    q.P = b[6 * len];
    q.Hz = b[7 * len];
    q.Hr = b[8 * len];
    q.Hphi = b[9 * len];
    return q;
}

MPD_HD void store_line_phys(double *lines, int len, int line, int idx, const Phys &q) {
    double *b = lines + (size_t)line * 10 * len + idx;
    b[0 * len] = q.rho;
    b[1 * len] = q.vz;
    b[2 * len] = q.vr;
    b[3 * len] = q.vphi;
    b[4 * len] = q.e;
    b[5 * len] = q.p;
    b[6 * len] = q.P;
    b[7 * len] = q.Hz;
    b[8 * len] = q.Hr;
    b[9 * len] = q.Hphi;
}

// Which central line (and index) holds cell (l, m), or -1.
MPD_HD int central_line(int L, int M, int l, int m, int &idx) {
    if (l == 2) { idx = m; return 0; }
    if (l == L - 1) { idx = m; return 1; }
    if (m == 2) { idx = l; return 2; }
    if (m == M) { idx = l; return 3; }
    idx = 0;
    return -1;
}

// Store the new conserved values of a freshly updated central cell into every
// central line that holds it (line stride 8 * len, field stride len).
MPD_HD void store_central(double *cl, int len, int L, int M, int l, int m, const double u[8]) {
    const int lines[4] = {l == 2 ? 0 : -1, l == L - 1 ? 1 : -1, m == 2 ? 2 : -1, m == M ? 3 : -1};
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        if (lines[t] < 0) continue;
        double *b = cl + (size_t)lines[t] * 8 * len + (t < 2 ? m : l);
#pragma unroll
        for (int k = 0; k < 8; ++k) b[(size_t)k * len] = u[k];
    }
}

MPD_HD bool wants_central(int L, int M, int l, int m) {
    return l == 2 || l == L - 1 || m == 2 || m == M;
}

// Point (n, p) of the step's input state as the fast interior's warp sees it:
// conserved values, primitives and radius (ghost rows: U = 0, r = 1, every
// primitive 0).
MPD_HD void fast_point(const Geo &g, const double *u0, int n, int p, double gm1, double U[8],
                       FastPrim &q, double &r) {
    const bool gh = n <= 0 || n >= g.L + 1 || p > g.M + 1;
    load_cons(u0, g.ps, g.ix(n, p), U);
    r = gh ? 1.0 : g.r(n, p);
    q = fast_prim(U, r, gm1, gh);
}

// The fast interior's new conserved values of cell (l, m), 1 <= l <= L,
// 2 <= m <= M, computed on their own from the step's input state u0: the
// operations of lf_tma_kernel's warp in the same order (A from point row
// l-1; B from the east and west points' shares, which the warp moves by
// shuffles, and the point's own sources; closed with point row l+1), so the
// result is bit-identical to the value that kernel stores for the cell.
MPD_HD void fast_cell_alone(const Geo &g, const double *u0, double dt, int l, int m,
                            double out[8]) {
    const double gm1 = g.gamma - 1.0;
    const double kz = dt * (0.5 / g.dz);
    double U[8], Gz[8], A[9], B[9], S[10];
    FastPrim q;
    double r;
    fast_point(g, u0, l - 1, m, gm1, U, q, r);
    fast_gz(U, q, r, Gz);
    fast_a(U, Gz, kz, A);
    const double kr = dt * g.hdr[l];
    {
        double Ue[8], Uw[8], Gre[8], Grw[8], re, rw;
        FastPrim qe, qw;
        fast_point(g, u0, l, m + 1, gm1, Ue, qe, re);
        fast_gr(Ue, qe, re, Gre);
        fast_point(g, u0, l, m - 1, gm1, Uw, qw, rw);
        fast_gr(Uw, qw, rw, Grw);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const double ce = (k == 7) ? 0.25 * Ue[7] : fma(kr, Gre[k], 0.25 * Ue[k]);
            const double cw = (k == 7) ? 0.25 * Uw[7] : fma(-kr, Grw[k], 0.25 * Uw[k]);
            B[k] = ce + cw;
        }
        const double d7 = Gre[7] - Grw[7];
        fast_point(g, u0, l, m, gm1, U, q, r);
        B[2] = fma(dt, fma(q.rho * q.vphi, q.vphi, q.P) - q.Hphi * q.Hphi, B[2]);
        B[3] = fma(dt, fma(-q.rho * q.vr, q.vphi, q.Hphi * q.Hr), B[3]);
        B[4] = fma(-q.p * kr, d7, B[4]);
        B[8] = q.p;
    }
    fast_sum(A, B, S);
    fast_point(g, u0, l + 1, m, gm1, U, q, r);
    fast_gz(U, q, r, Gz);
    fast_finish(S, U, Gz, kz, out);
}

// Everything one boundary step reads.
struct BcView {
    Geo g;
    const double *u0;     // conserved state at the start of the step
    double *u;            // new state (interior written by the LF kernel)
    const double *ic;     // initial physical planes (first step only)
    const double *cphys;  // central lines of this step (conserved values)
    const double *wphys;  // wall lines at the start of this step
    int len;              // line length
    int first;            // step 0: "old" physical values are the IC planes
    int fast;             // MPD_PRECISION_FAST: reconstruct with reciprocals
    double dt;
    BcTable bc;
    // The faces run beside the fast interior instead of after it: central
    // cells they read are recomputed from u0 (fast_cell_alone) instead of
    // read from the central lines, and ring cells no face covers take that
    // value too (the interior then writes neither).
    int recompute = 0;
};

// Fields::UpdatePhysicalFromU of one cell on the boundary path: the exact
// divides in exact mode, the interior kernel's reciprocal form in fast mode.
MPD_HD Phys recon_bc(const BcView &v, const double u[8], double r) {
    if (!v.fast) return recon_exact(u, r, v.g.gamma);
    const FastPrim f = fast_prim(u, r, v.g.gamma - 1.0);
    Phys q;
    q.rho = f.rho;
    q.vz = f.vz;
    q.vr = f.vr;
    q.vphi = f.vphi;
    q.e = f.e;
    q.p = f.p;
    q.P = f.P;
    q.Hz = f.Hz;
    q.Hr = f.Hr;
    q.Hphi = f.Hphi;
    return q;
}

// Primitive values in evaluation order.
struct Prim {
    double v[8];
};

MPD_HD Prim prim_of(const Phys &q) {
    Prim p;
    p.v[Q_RHO] = q.rho;
    p.v[Q_VZ] = q.vz;
    p.v[Q_VR] = q.vr;
    p.v[Q_VPHI] = q.vphi;
    p.v[Q_HZ] = q.Hz;
    p.v[Q_HR] = q.Hr;
    p.v[Q_HPHI] = q.Hphi;
    p.v[Q_E] = q.e;
    return p;
}

// Physical value of a cell as the previous step's full reconstruction left
// it (or the initial condition on the first step).
// The boundary faces only ever ask for wall cells (m = 1 or M+1) here.
MPD_HD Phys old_phys(const BcView &v, int l, int m) {
    if (m == 1) return line_phys(v.wphys, v.len, 0, l);
    if (m == v.g.M + 1) return line_phys(v.wphys, v.len, 1, l);
    const size_t i = v.g.ix(l, m);
    if (v.first) return load_phys(v.ic, v.g.ps, i);
    double u[8];
    load_cons(v.u0, v.g.ps, i, u);
    return recon_bc(v, u, v.g.r(l, m));
}

// Physical value of a central cell after this step's central update
// (UpdateCentralPhysical, src/solver.cpp:155-159).  The faces only ask for
// cells the central lines hold.
MPD_HD Phys central_phys(const BcView &v, int l, int m) {
    int idx;
    const int line = central_line(v.g.L, v.g.M, l, m, idx);
    double u[8];
    if (v.recompute) {
        fast_cell_alone(v.g, v.u0, v.dt, l, m, u);
        return recon_bc(v, u, v.g.r(l, m));
    }
    if (line >= 0) {
        const double *b = v.cphys + (size_t)line * 8 * v.len + idx;
#pragma unroll
        for (int k = 0; k < 8; ++k) u[k] = b[(size_t)k * v.len];
        return recon_bc(v, u, v.g.r(l, m));
    }
    load_cons(v.u, v.g.ps, v.g.ix(l, m), u);
    return recon_bc(v, u, v.g.r(l, m));
}

// Last segment of `face` whose range covers free index k, or -1.
MPD_HD int last_cover(const BcView &v, int face, int k, int limit) {
    const int base = v.bc.first[face];
    for (int s = limit; s >= 0; --s) {
        const SegDesc &d = v.bc.seg[base + s];
        if (k >= d.lo && k <= d.hi) return s;
    }
    return -1;
}

// Value of boundary expression symbol `idx` at cell (l, m) with neighbour
// (ln, mn); out holds the fields already evaluated in this cell.
MPD_HD double bc_sym(const BcView &v, int idx, int l, int m, int ln, int mn, const Prim &nb,
                     const Prim &out) {
    switch (idx) {
        case BS_GAMMA: return v.g.gamma;
        case BS_BETA: return v.g.beta;
        case BS_HZ0: return v.g.H_z0;
        case BS_R0: return v.g.r_0;
        case BS_DZ: return v.g.dz;
        case BS_DR: return v.g.dr[l];
        case BS_R: return v.g.r(l, m);
        case BS_RZ: return v.g.rz(l, m);
        case BS_Z: return (double)(l - 1) * v.g.dz;
        case BS_RNB: return v.g.r(ln, mn);
        case BS_RZNB: return v.g.rz(ln, mn);
        // *_nb symbols in the reference's SetNeighbors order:
        // rho, v_z, v_r, v_phi, e, H_z, H_r, H_phi
        case BS_NB0 + 0: return nb.v[Q_RHO];
        case BS_NB0 + 1: return nb.v[Q_VZ];
        case BS_NB0 + 2: return nb.v[Q_VR];
        case BS_NB0 + 3: return nb.v[Q_VPHI];
        case BS_NB0 + 4: return nb.v[Q_E];
        case BS_NB0 + 5: return nb.v[Q_HZ];
        case BS_NB0 + 6: return nb.v[Q_HR];
        case BS_NB0 + 7: return nb.v[Q_HPHI];
        case BS_CUR0 + 0: return out.v[0];
        case BS_CUR0 + 1: return out.v[1];
        case BS_CUR0 + 2: return out.v[2];
        case BS_CUR0 + 3: return out.v[3];
        case BS_CUR0 + 4: return out.v[4];
        case BS_CUR0 + 5: return out.v[5];
        case BS_CUR0 + 6: return out.v[6];
        case BS_CUR0 + 7: return out.v[7];
        default: return NAN;
    }
}

// An expression field the closed forms don't cover: full symbol table and
// the bytecode interpreter.  Inlined: an out-of-line call takes the view by
// reference, which puts the whole BcView in local memory for every caller
// and turns each of its fields into a load on the boundary chains (the
// boundary kernels' stacks shrink from 992 to 720 bytes, the batched
// engine's spills from 594 to 314 bytes).
MPD_HD double bc_eval_general(const BcView &v, int code, int l, int m, int ln, int mn,
                              Prim nb, Prim out) {
    double sym[BS_COUNT];
    for (int t = 0; t < BS_COUNT; ++t) sym[t] = bc_sym(v, t, l, m, ln, mn, nb, out);
    return eval_code(v.bc.code + code, v.bc.consts, sym);
}

MPD_HD double bc_binop(int op, double a, double b) {
    switch (op) {
        case OP_ADD: return a + b;
        case OP_SUB: return a - b;
        case OP_MUL: return a * b;
        default: return a / b;
    }
}

// PerFieldBC::Apply's per-cell field evaluation (src/bcs/per_field_bc.cpp:
// 286-292 resolve, 311-360 / 393-446 expression path): writes the 8 new
// primitives of cell (l, m) given its neighbour's primitives and the values
// to keep (AxisLF fields keep the cell's current value).
#ifndef MPD_SEG_UNROLL
#define MPD_SEG_UNROLL 0
#endif
MPD_HD void eval_segment(const BcView &v, const SegDesc &d, int l, int m, int ln, int mn,
                         const Prim &nb, const Prim &keep, Prim &out) {
#if MPD_SEG_UNROLL
#pragma unroll
#else
#pragma unroll 1
#endif
    for (int j = 0; j < 8; ++j) {
        double val;
        switch (d.type[j]) {
            case COND_NEUMANN: val = nb.v[j] + d.value[j]; break;
            case COND_DIRICHLET: val = d.value[j]; break;
            case COND_EXPR: {
                const int form = d.form[j];
                if (form == EF_CONST) {
                    val = d.ca[j];
                } else if (form == EF_BIN) {
                    const double a = d.fa[j] < 0 ? d.ca[j] : bc_sym(v, d.fa[j], l, m, ln, mn, nb, out);
                    const double b = d.fb[j] < 0 ? d.cb[j] : bc_sym(v, d.fb[j], l, m, ln, mn, nb, out);
                    val = bc_binop(d.fop[j], a, b);
                } else {
                    val = bc_eval_general(v, d.code[j], l, m, ln, mn, nb, out);
                }
                break;
            }
            default: val = keep.v[j]; break;
        }
        out.v[j] = val;
    }
}

// Physical primitives of (1, m) after the L_LO face; covered = false if no
// L_LO segment covers m (then the cell keeps its value).
MPD_HD bool l_lo_out(const BcView &v, int m, Prim &out) {
    const int s = last_cover(v, FACE_L_LO, m, v.bc.nseg[FACE_L_LO] - 1);
    if (s < 0) return false;
    const Prim nb = prim_of((m >= 2 && m <= v.g.M) ? central_phys(v, 2, m) : old_phys(v, 2, m));
    eval_segment(v, v.bc.seg[v.bc.first[FACE_L_LO] + s], 1, m, 2, m, nb, nb, out);
    return true;
}

// Primitives of (l, M+1) after the M_HI face (applied after L_LO).
MPD_HD bool m_hi_out(const BcView &v, int l, Prim &out) {
    const int s = last_cover(v, FACE_M_HI, l, v.bc.nseg[FACE_M_HI] - 1);
    if (s < 0) return false;
    const int M = v.g.M;
    Prim nb;
    if (l == 1) {
        if (!l_lo_out(v, M, nb)) nb = prim_of(central_phys(v, 1, M));
    } else {
        nb = prim_of(central_phys(v, l, M));
    }
    eval_segment(v, v.bc.seg[v.bc.first[FACE_M_HI] + s], l, M + 1, l, M, nb, nb, out);
    return true;
}

// Primitives of (l, 1), 2 <= l <= L-1, after the M_LO segments 0..limit have
// been applied in order (each covering segment starts from the previous
// one's result; AxisLF fields keep it).  Returns the last applied segment or -1.
MPD_HD int m_lo_after(const BcView &v, int l, int limit, Prim &out) {
    out = prim_of(old_phys(v, l, 1));
    const int base = v.bc.first[FACE_M_LO];
    int last = -1;
    bool have_nb = false;
    Prim nb;
    for (int s = 0; s <= limit; ++s) {
        const SegDesc &d = v.bc.seg[base + s];
        if (l < d.lo || l > d.hi) continue;
        if (!have_nb) {
            nb = prim_of(central_phys(v, l, 2));
            have_nb = true;
        }
        const Prim keep = out;
        eval_segment(v, d, l, 1, l, 2, nb, keep, out);
        last = s;
    }
    return last;
}

// Primitives of (L, m) after the L_HI face (applied last).
MPD_HD bool l_hi_out(const BcView &v, int m, Prim &out) {
    const int s = last_cover(v, FACE_L_HI, m, v.bc.nseg[FACE_L_HI] - 1);
    if (s < 0) return false;
    const int L = v.g.L, M = v.g.M;
    Prim nb;
    if (m >= 2 && m <= M) {
        nb = prim_of(central_phys(v, L - 1, m));
    } else if (m == 1) {
        if (m_lo_after(v, L - 1, v.bc.nseg[FACE_M_LO] - 1, nb) < 0)
            nb = prim_of(old_phys(v, L - 1, 1));
    } else {
        if (!m_hi_out(v, L - 1, nb)) nb = prim_of(old_phys(v, L - 1, M + 1));
    }
    eval_segment(v, v.bc.seg[v.bc.first[FACE_L_HI] + s], L, m, L - 1, m, nb, nb, out);
    return true;
}

// Values AxisLF reads at the four stencil points of (l, 1).
struct AxisPoint {
    double u0, r, vz, vr, Hz, Hr, P, p;
};

// PerFieldBC::AxisLfU1/U2/U5/U7 (src/bcs/per_field_bc.cpp:490-566).
// Points: C = (l,1), N = (l+1,1), S = (l-1,1), E = (l,2).
MPD_HD double axis_u1(const AxisPoint &C, const AxisPoint &N, const AxisPoint &S,
                      const AxisPoint &E, double dt, double dz, double dr_l) {
    return (0.25 * (N.u0 / N.r + S.u0 / S.r + E.u0 / E.r + C.u0 / C.r)
            + dt * (-(N.u0 / N.r * N.vz - S.u0 / S.r * S.vz) / (2.0 * dz)
                    - (E.u0 / E.r * E.vr - C.u0 / C.r * E.vr) / dr_l))
           * C.r;
}
MPD_HD double axis_u2(const AxisPoint &C, const AxisPoint &N, const AxisPoint &S,
                      const AxisPoint &E, double dt, double dz, double dr_l) {
    return (0.25 * (N.u0 / N.r + S.u0 / S.r + E.u0 / E.r + C.u0 / C.r)
            + dt * (((N.Hz * N.Hz - N.P) - (S.Hz * S.Hz - S.P)) / (2.0 * dz)
                    + (E.Hz * E.Hr - C.Hz * C.Hr) / dr_l
                    - (N.u0 / N.r * N.vz - S.u0 / S.r * S.vz) / (2.0 * dz)
                    - (E.u0 / E.r * E.vr - C.u0 / C.r * C.vr) / dr_l))
           * C.r;
}
MPD_HD double axis_u5(const AxisPoint &C, const AxisPoint &N, const AxisPoint &S,
                      const AxisPoint &E, double dt, double dz, double dr_l) {
    return (0.25 * (N.u0 / N.r + S.u0 / S.r + E.u0 / E.r + C.u0 / C.r)
            + dt * (-C.p * ((N.vz - S.vz) / (2.0 * dz) + (E.vr - C.vr) / dr_l)
                    - (N.u0 / N.r * N.vz - S.u0 / S.r * S.vz) / (2.0 * dz)
                    - (E.u0 / E.r * E.vr - C.u0 / C.r * C.vr) / dr_l))
           * C.r;
}
MPD_HD double axis_u7(const AxisPoint &C, const AxisPoint &N, const AxisPoint &S,
                      const AxisPoint &E, double dt, double dz, double dr_l) {
    (void)N;
    (void)S;
    (void)dz;
    return (0.25 * (N.u0 / N.r + S.u0 / S.r + E.u0 / E.r + C.u0 / C.r)
            + dt * ((E.Hr * E.vz - C.Hr * C.vz) / dr_l
                    - (E.u0 / E.r * E.vr - C.u0 / C.r * C.vr) / dr_l))
           * C.r;
}

// Final conserved values of M_LO cell (l, 1): rebuild from the primitives of
// the last covering segment, then that segment's AxisLF overwrites.  The
// neighbours (l-1,1) / (l+1,1) are seen as the serial segment loop leaves
// them: l-1 already processed by the same segment, l+1 not yet.
MPD_HD void m_lo_final_u(const BcView &v, int l, int s_last, const Prim &q, double u[8]) {
    const Geo &g = v.g;
    Phys cur;
    cur.rho = q.v[Q_RHO];
    cur.vz = q.v[Q_VZ];
    cur.vr = q.v[Q_VR];
    cur.vphi = q.v[Q_VPHI];
    cur.Hz = q.v[Q_HZ];
    cur.Hr = q.v[Q_HR];
    cur.Hphi = q.v[Q_HPHI];
    cur.e = q.v[Q_E];
    const double rc = g.r(l, 1);
    rebuild_u(cur, rc, u);
    const SegDesc &d = v.bc.seg[v.bc.first[FACE_M_LO] + s_last];
    if (!d.has_axis) return;

    // old physical state of the cell supplies p and P (never written by BCs)
    const Phys oc = old_phys(v, l, 1);
    // neighbour l-1
    Prim qs;
    if (l - 1 == 1) {
        if (!l_lo_out(v, 1, qs)) qs = prim_of(old_phys(v, 1, 1));
    } else {
        const int lim = (l - 1 >= d.lo && l - 1 <= d.hi) ? s_last : s_last - 1;
        m_lo_after(v, l - 1, lim, qs);
    }
    // neighbour l+1
    Prim qn;
    if (l + 1 == g.L) {
        qn = prim_of(old_phys(v, g.L, 1));
    } else {
        m_lo_after(v, l + 1, s_last - 1, qn);
    }
    const Phys os = old_phys(v, l - 1, 1);
    const Phys on = old_phys(v, l + 1, 1);
    const Phys ce = central_phys(v, l, 2);

    AxisPoint C, N, S, E;
    C.r = rc;
    C.vz = cur.vz;
    C.vr = cur.vr;
    C.Hz = cur.Hz;
    C.Hr = cur.Hr;
    C.P = oc.P;
    C.p = oc.p;
    N.r = g.r(l + 1, 1);
    N.vz = qn.v[Q_VZ];
    N.vr = qn.v[Q_VR];
    N.Hz = qn.v[Q_HZ];
    N.Hr = qn.v[Q_HR];
    N.P = on.P;
    N.p = on.p;
    S.r = g.r(l - 1, 1);
    S.vz = qs.v[Q_VZ];
    S.vr = qs.v[Q_VR];
    S.Hz = qs.v[Q_HZ];
    S.Hr = qs.v[Q_HR];
    S.P = os.P;
    S.p = os.p;
    E.r = g.r(l, 2);
    E.vz = ce.vz;
    E.vr = ce.vr;
    E.Hz = ce.Hz;
    E.Hr = ce.Hr;
    E.P = ce.P;
    E.p = ce.p;
    const size_t ic = g.ix(l, 1), in = g.ix(l + 1, 1), is = g.ix(l - 1, 1), ie = g.ix(l, 2);
    const double dr_l = g.dr[l];
    // u0 planes: u_1 = k 0, u_2 = k 1, u_5 = k 4, u_7 = k 6
    const int kcons[4] = {0, 1, 4, 6};
    const int kprim[4] = {Q_RHO, Q_VZ, Q_E, Q_HZ};
    for (int t = 0; t < 4; ++t) {
        if (d.type[kprim[t]] != COND_AXIS_LF) continue;
        const size_t off = (size_t)kcons[t] * g.ps;
        C.u0 = v.u0[off + ic];
        N.u0 = v.u0[off + in];
        S.u0 = v.u0[off + is];
        E.u0 = v.u0[off + ie];
        double val;
        switch (t) {
            case 0: val = axis_u1(C, N, S, E, v.dt, g.dz, dr_l); break;
            case 1: val = axis_u2(C, N, S, E, v.dt, g.dz, dr_l); break;
            case 2: val = axis_u5(C, N, S, E, v.dt, g.dz, dr_l); break;
            default: val = axis_u7(C, N, S, E, v.dt, g.dz, dr_l); break;
        }
        u[kcons[t]] = val;
    }
}

MPD_HD void phys_to_prim_u(const Prim &q, double r, double u[8]) {
    Phys p;
    p.rho = q.v[Q_RHO];
    p.vz = q.v[Q_VZ];
    p.vr = q.v[Q_VR];
    p.vphi = q.v[Q_VPHI];
    p.Hz = q.v[Q_HZ];
    p.Hr = q.v[Q_HR];
    p.Hphi = q.v[Q_HPHI];
    p.e = q.v[Q_E];
    p.p = p.P = 0.0;
    rebuild_u(p, r, u);
}

// Ring slots: the edge cells of rows l = 1 and l = L (m = 2..M) and of
// columns m = 1 and m = M+1 (l = 2..L-1), then the four corners, each at the
// start of its own 32-slot group (the other slots of a group are idle).  The
// corners run the longest recomputation chains; alone in their warps they do
// not serialise behind the edge cells' code paths.
constexpr int kRingGroup = 32;

MPD_HD int ring_edges(const Geo &g) { return 2 * (g.M - 1) + 2 * (g.L - 2); }

MPD_HD int ring_count(const Geo &g) {
    const int e = ring_edges(g);
    return (e + kRingGroup - 1) / kRingGroup * kRingGroup + 4 * kRingGroup;
}

// Cell of ring slot i; false for an idle slot.
MPD_HD bool ring_cell(const Geo &g, int i, int &l, int &m) {
    const int inner = g.M - 1;
    const int e = ring_edges(g);
    if (i < e) {
        if (i < inner) { l = 1; m = 2 + i; return true; }
        i -= inner;
        if (i < inner) { l = g.L; m = 2 + i; return true; }
        i -= inner;
        if (i < g.L - 2) { l = 2 + i; m = 1; return true; }
        i -= g.L - 2;
        l = 2 + i;
        m = g.M + 1;
        return true;
    }
    const int c = i - (e + kRingGroup - 1) / kRingGroup * kRingGroup;
    if (c < 0 || c % kRingGroup != 0) return false;
    switch (c / kRingGroup) {
        case 0: l = 1; m = 1; return true;
        case 1: l = 1; m = g.M + 1; return true;
        case 2: l = g.L; m = 1; return true;
        case 3: l = g.L; m = g.M + 1; return true;
        default: return false;
    }
}

// Final conserved values of boundary-ring cell (l, m) after the four faces
// L_LO, M_HI, M_LO, L_HI have been applied in that order
// (src/solver.cpp:29-32).  The last face that covers the cell decides it;
// cells no face covers keep the central update (interior columns) or the
// zero the reference's never-written u arrays hold (wall columns).
MPD_HD void bc_ring_final(const BcView &v, int l, int m, double u[8]) {
    const Geo &g = v.g;
    const int L = g.L, M = g.M;
    Prim q;
    if (l == L && l_hi_out(v, m, q)) {
        phys_to_prim_u(q, g.r(l, m), u);
        return;
    }
    if (m == 1 && l >= 2 && l <= L - 1) {
        const int s_last = m_lo_after(v, l, v.bc.nseg[FACE_M_LO] - 1, q);
        if (s_last >= 0) {
            m_lo_final_u(v, l, s_last, q, u);
            return;
        }
    }
    if (m == M + 1 && m_hi_out(v, l, q)) {
        phys_to_prim_u(q, g.r(l, m), u);
        return;
    }
    if (l == 1 && l_lo_out(v, m, q)) {
        phys_to_prim_u(q, g.r(l, m), u);
        return;
    }
    if (m >= 2 && m <= M) {
        if (v.recompute)
            fast_cell_alone(g, v.u0, v.dt, l, m, u);
        else
            load_cons(v.u, g.ps, g.ix(l, m), u);
        return;
    }
    for (int k = 0; k < 8; ++k) u[k] = 0.0;
}

}  // namespace mpd
