// Host emulation of one device time step — built only into libmpd_emu.so for
// the CPU test suite (the product library libmpd_b200.so has no host path).
//
// It runs the kernels' own per-cell functions from lf_core.cuh over every
// cell in a plain loop: the exact interior cell (lf_exact_kernel), the fast
// interior cell (lf_tma_kernel: fast_prim / fast_a / fast_rc / fast_b / fast_finish), the boundary ring
// (bc_kernel's bc_ring_final).  That lets the CPU suite check the boundary
// dependency logic and the fast-mode rounding against the oracle before any
// GPU time is spent.
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mpd_b200.h"
#include "bc_compile.hpp"
#include "lf_core.cuh"

namespace mpd {
namespace {
thread_local std::string g_emu_error;
}
void SetLastError(const std::string &msg) { g_emu_error = msg; }
}  // namespace mpd

namespace {

struct EmuSolver {
    mpd::Geo g{};
    int rows = 0, cols = 0;
    std::vector<double> buf[2], ic, geo;
    mpd::CompiledBc cbc;
    mpd::BcTable bc{};
    int precision = 0;
    long long step = 0;
    int len = 0;
    std::vector<double> cphys, wall[2];
};

}  // namespace

extern "C" {

const char *mpd_emu_last_error(void) { return mpd::g_emu_error.c_str(); }

int mpd_emu_create(const mpd_config *cfg, const mpd_geometry *geom, const double *phys10,
                   void **out) {
    std::string err;
    int rc = mpd::ValidateConfig(cfg, geom, err);
    if (rc != MPD_OK) {
        mpd::SetLastError(err);
        return rc;
    }
    auto *s = new EmuSolver();
    rc = mpd::CompileBc(*cfg, s->cbc, err);
    if (rc != MPD_OK) {
        mpd::SetLastError(err);
        delete s;
        return rc;
    }
    const int L = cfg->L_max, M = cfg->M_max;
    s->rows = L + 2;
    s->cols = M + 3;
    const size_t ps = static_cast<size_t>(s->rows) * s->cols;
    s->buf[0].assign(8 * ps, 0.0);
    s->buf[1].assign(8 * ps, 0.0);
    s->ic.assign(10 * ps, 0.0);
    s->geo.assign(6 * static_cast<size_t>(s->rows), 0.0);
    for (int l = 0; l < s->rows; ++l) {
        s->geo[0 * s->rows + l] = geom->r_inner[l];
        s->geo[1 * s->rows + l] = geom->r_outer[l];
        s->geo[2 * s->rows + l] = geom->dr_inner_dz[l];
        s->geo[3 * s->rows + l] = geom->dr_outer_dz[l];
        const double R = geom->r_outer[l] - geom->r_inner[l];
        s->geo[4 * s->rows + l] = R / M;
        s->geo[5 * s->rows + l] = 0.5 / s->geo[4 * s->rows + l];
    }
    mpd::Geo &g = s->g;
    g.L = L;
    g.M = M;
    g.pitch = s->cols;
    g.ps = ps;
    g.dz = cfg->dz;
    g.dy = cfg->dy;
    g.gamma = cfg->gamma;
    g.beta = cfg->beta;
    g.H_z0 = cfg->H_z0;
    g.r_0 = cfg->r_0;
    g.rin = s->geo.data();
    g.rout = s->geo.data() + s->rows;
    g.drin = s->geo.data() + 2 * s->rows;
    g.drout = s->geo.data() + 3 * s->rows;
    g.dr = s->geo.data() + 4 * s->rows;
    g.hdr = s->geo.data() + 5 * s->rows;
    for (int k = 0; k < 10; ++k)
        for (int l = 1; l <= L; ++l)
            for (int m = 1; m <= M + 1; ++m) s->ic[k * ps + g.ix(l, m)] = phys10[k * ps + g.ix(l, m)];
    for (int l = 1; l <= L; ++l)
        for (int m = 1; m <= M + 1; ++m) {
            double u[8];
            mpd::rebuild_u(mpd::load_phys(s->ic.data(), ps, g.ix(l, m)), g.r(l, m), u);
            for (int k = 0; k < 8; ++k) s->buf[0][k * ps + g.ix(l, m)] = u[k];
        }
    s->len = mpd::line_len(L, M);
    s->cphys.assign(static_cast<size_t>(mpd::kCentralLines) * 8 * s->len, 0.0);
    s->wall[0].assign(static_cast<size_t>(mpd::kWallLines) * 10 * s->len, 0.0);
    s->wall[1].assign(static_cast<size_t>(mpd::kWallLines) * 10 * s->len, 0.0);
    for (int l = 1; l <= L; ++l) {
        mpd::store_line_phys(s->wall[0].data(), s->len, 0, l,
                             mpd::load_phys(s->ic.data(), ps, g.ix(l, 1)));
        mpd::store_line_phys(s->wall[0].data(), s->len, 1, l,
                             mpd::load_phys(s->ic.data(), ps, g.ix(l, M + 1)));
    }
    for (int f = 0; f < 4; ++f) {
        s->bc.nseg[f] = s->cbc.nseg[f];
        s->bc.first[f] = s->cbc.first[f];
    }
    s->bc.seg = s->cbc.seg.data();
    s->bc.code = s->cbc.code.data();
    s->bc.consts = s->cbc.consts.data();
    s->bc.nseg_total = static_cast<int>(s->cbc.seg.size());
    s->bc.ncode = static_cast<int>(s->cbc.code.size());
    s->bc.nconst = static_cast<int>(s->cbc.consts.size());
    s->precision = cfg->precision;
    *out = s;
    return MPD_OK;
}

void mpd_emu_destroy(void *h) { delete static_cast<EmuSolver *>(h); }

// order: 0 = compute every ring cell, then write them; 1 = write each as it is
// computed, in ring order; 2 = the same in reverse order.  All three must give
// the same state, which is what makes the one-thread-per-cell device kernel
// free of read/write hazards.
int mpd_emu_advance(void *h, double dt, int order) {
    auto *s = static_cast<EmuSolver *>(h);
    const mpd::Geo &g = s->g;
    const bool first = s->step == 0;
    const double *u0 = s->buf[s->step & 1].data();
    double *u = s->buf[(s->step + 1) & 1].data();
    const double gm1 = g.gamma - 1.0;
    for (int l = 1; l <= g.L; ++l) {
        for (int m = 2; m <= g.M; ++m) {
            const int ls[5] = {l, l + 1, l - 1, l, l};
            const int ms[5] = {m, m, m, m + 1, m - 1};
            double U[5][8], R[5];
            for (int p = 0; p < 5; ++p) {
                R[p] = g.r(ls[p], ms[p]);
                mpd::load_cons(u0, g.ps, g.ix(ls[p], ms[p]), U[p]);
            }
            double out[8];
            if (first || s->precision == MPD_PRECISION_EXACT) {
                mpd::Phys Q[5];
                for (int p = 0; p < 5; ++p) {
                    if (ls[p] == 0 || ls[p] == g.L + 1) Q[p] = mpd::phys_zero();
                    else if (first) Q[p] = mpd::load_phys(s->ic.data(), g.ps, g.ix(ls[p], ms[p]));
                    else Q[p] = mpd::recon_exact(U[p], R[p], g.gamma);
                }
                mpd::lf_cell_exact(U, Q, R, dt, g.dz, g.dr[l], out);
            } else {
                // the fast kernel's arithmetic, point by point (ghost rows are zero)
                const double kz = dt * (0.5 / g.dz), kr = dt * (0.5 / g.dr[l]);
                mpd::FastPrim q[5];
                double Gz[5][8], Gr[5][8];
                for (int p = 0; p < 5; ++p) {
                    if (ls[p] == 0 || ls[p] == g.L + 1) {
                        q[p] = mpd::FastPrim{};
                        for (int k = 0; k < 8; ++k) Gz[p][k] = Gr[p][k] = 0.0;
                    } else {
                        q[p] = mpd::fast_prim(U[p], R[p], gm1);
                        mpd::fast_gz(U[p], q[p], R[p], Gz[p]);
                        mpd::fast_gr(U[p], q[p], R[p], Gr[p]);
                    }
                }
                double A[9], B[9], S[10], ce[8], cw[8], ce_e[8], cw_w[8];
                mpd::fast_a(U[2], Gz[2], kz, A);
                mpd::fast_rc(U[3], Gr[3], kr, ce_e, cw);   // east neighbour's ce
                mpd::fast_rc(U[4], Gr[4], kr, ce, cw_w);   // west neighbour's cw
                mpd::fast_b(ce_e, cw_w, Gr[3][7], Gr[4][7], q[0], kr, dt, B);
                mpd::fast_sum(A, B, S);
                mpd::fast_finish(S, U[1], Gz[1], kz, out);
            }
            for (int k = 0; k < 8; ++k) u[k * g.ps + g.ix(l, m)] = out[k];
            if (mpd::wants_central(g.L, g.M, l, m))
                mpd::store_central(s->cphys.data(), s->len, g.L, g.M, l, m, out);
        }
    }
    mpd::BcView v;
    v.g = g;
    v.u0 = u0;
    v.u = u;
    v.ic = s->ic.data();
    v.cphys = s->cphys.data();
    v.wphys = s->wall[s->step & 1].data();
    v.len = s->len;
    v.first = first ? 1 : 0;
    v.fast = s->precision == MPD_PRECISION_FAST ? 1 : 0;
    v.dt = dt;
    v.bc = s->bc;
    const int nring = mpd::ring_count(g);
    std::vector<double> ring(8 * static_cast<size_t>(nring));
    for (int t = 0; t < nring; ++t) {
        const int i = order == 2 ? nring - 1 - t : t;
        int l, m;
        if (!mpd::ring_cell(g, i, l, m)) continue;
        double *uf = &ring[8 * static_cast<size_t>(i)];
        mpd::bc_ring_final(v, l, m, uf);
        if (m == 1 || m == g.M + 1)
            mpd::store_line_phys(s->wall[(s->step + 1) & 1].data(), s->len, m == 1 ? 0 : 1, l,
                                 mpd::recon_bc(v, uf, g.r(l, m)));
        if (order != 0)
            for (int k = 0; k < 8; ++k) u[k * g.ps + g.ix(l, m)] = uf[k];
    }
    if (order == 0) {
        for (int i = 0; i < nring; ++i) {
            int l, m;
            if (!mpd::ring_cell(g, i, l, m)) continue;
            for (int k = 0; k < 8; ++k) u[k * g.ps + g.ix(l, m)] = ring[8 * static_cast<size_t>(i) + k];
        }
    }
    s->step++;
    return MPD_OK;
}

// which: 0..7 conserved, 8..17 physical (initial condition before any step).
int mpd_emu_download(void *h, int which, double *out) {
    auto *s = static_cast<EmuSolver *>(h);
    const mpd::Geo &g = s->g;
    const size_t n = g.ps;
    const double *cur = s->buf[s->step & 1].data();
    if (which < 8) {
        std::memcpy(out, cur + which * n, n * sizeof(double));
        return MPD_OK;
    }
    std::memset(out, 0, n * sizeof(double));
    for (int l = 1; l <= g.L; ++l)
        for (int m = 1; m <= g.M + 1; ++m) {
            mpd::Phys q;
            if (s->step == 0) {
                q = mpd::load_phys(s->ic.data(), n, g.ix(l, m));
            } else {
                double u[8];
                mpd::load_cons(cur, n, g.ix(l, m), u);
                q = mpd::recon_exact(u, g.r(l, m), g.gamma);
            }
            const double v[10] = {q.rho, q.vz, q.vr, q.vphi, q.e, q.p, q.P, q.Hz, q.Hr, q.Hphi};
            out[g.ix(l, m)] = v[which - 8];
        }
    return MPD_OK;
}

double mpd_emu_wave_speed(void *h) {
    auto *s = static_cast<EmuSolver *>(h);
    const mpd::Geo &g = s->g;
    const double *cur = s->buf[s->step & 1].data();
    double mx = 0.0;
    for (int l = 1; l <= g.L; ++l)
        for (int m = 1; m <= g.M + 1; ++m) {
            mpd::Phys q;
            if (s->step == 0) {
                q = mpd::load_phys(s->ic.data(), g.ps, g.ix(l, m));
            } else {
                double u[8];
                mpd::load_cons(cur, g.ps, g.ix(l, m), u);
                q = mpd::recon_exact(u, g.r(l, m), g.gamma);
            }
            const double w = mpd::wave_speed(q, g.gamma);
            mx = (mx < w) ? w : mx;
        }
    return mx;
}

}  // extern "C"
