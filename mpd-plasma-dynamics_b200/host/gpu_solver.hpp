// GpuSolver — drop-in for the reference's Solver (include/solver.hpp:24-53)
// on one B200, over the C ABI of include/mpd_b200.h.
//
// A maintainer adds this header to the reference and replaces
//     Solver solver(cfg, mpi, grid, fields);
// by
//     GpuSolver solver(cfg, mpi, grid, fields);
// keeping config.yaml, the IGeometry registry, the IInitialCondition and the
// per-field boundary configuration unchanged.  The state lives on the GPU;
// Download() copies it back into the host Fields before anything on the host
// (IOManager::WriteFrame, probes) reads them.  Errors throw
// std::runtime_error, like the reference's constructors.
#pragma once

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "config.hpp"
#include "fields.hpp"
#include "grid.hpp"
#include "mpd_b200.h"
#include "mpi_manager.hpp"
#include "verification.hpp"

class GpuSolver {
public:
    GpuSolver(const SimConfig &cfg, const MPIManager &mpi, const Grid &grid, Fields &f,
              int precision = MPD_PRECISION_FAST)
        : cfg_(cfg), f_(f) {
        if (mpi.size != 1)
            throw std::runtime_error("GpuSolver: one GPU owns the whole grid; run with one MPI rank");
        const BCFaceConfig *faces[4] = {&cfg.bc_l_lo, &cfg.bc_l_hi, &cfg.bc_m_lo, &cfg.bc_m_hi};
        mpd_config c{};
        c.gamma = cfg.gamma;
        c.beta = cfg.beta;
        c.H_z0 = cfg.H_z0;
        c.L_max = cfg.L_max;
        c.M_max = cfg.M_max;
        c.dz = cfg.dz;
        c.dy = cfg.dy;
        c.r_0 = grid.r_0;
        c.precision = precision;
        c.with_prev = f.has_prev ? 1 : 0;
        for (int k = 0; k < 4; ++k) {
            for (const BCSegmentConfig &s : faces[k]->segments) {
                mpd_bc_segment d{};
                d.global_lo = s.global_lo;
                d.global_hi = s.global_hi;
                d.rho = Cond(s.rho);
                d.v_z = Cond(s.v_z);
                d.v_r = Cond(s.v_r);
                d.v_phi = Cond(s.v_phi);
                d.e = Cond(s.e);
                d.H_z = Cond(s.H_z);
                d.H_r = Cond(s.H_r);
                d.H_phi = Cond(s.H_phi);
                segs_[k].push_back(d);
            }
            c.n_segments[k] = static_cast<int>(segs_[k].size());
            c.segments[k] = segs_[k].data();
        }
        // wall profiles at z = (l-1) dz, the rows Grid::Build samples
        const int rows = cfg.L_max + 2;
        std::vector<double> prof(4 * static_cast<size_t>(rows));
        for (int l = 0; l < rows; ++l) {
            const double z = (l - 1) * cfg.dz;
            prof[l] = grid.geom.RInner(z);
            prof[rows + l] = grid.geom.ROuter(z);
            prof[2 * rows + l] = grid.geom.DrInnerDz(z);
            prof[3 * rows + l] = grid.geom.DrOuterDz(z);
        }
        mpd_geometry g{prof.data(), prof.data() + rows, prof.data() + 2 * rows,
                       prof.data() + 3 * rows};
        const Array2D *phys[10] = {&f.rho, &f.v_z, &f.v_r, &f.v_phi, &f.e,
                                   &f.p,   &f.P,   &f.H_z, &f.H_r, &f.H_phi};
        const size_t n = f.rho.Size();
        std::vector<double> planes(10 * n);
        for (int k = 0; k < 10; ++k)
            std::copy(phys[k]->Flat(), phys[k]->Flat() + n, planes.begin() + k * n);
        Check(mpd_create(&c, &g, planes.data(), &h_));
    }

    ~GpuSolver() { mpd_destroy(h_); }
    GpuSolver(const GpuSolver &) = delete;
    GpuSolver &operator=(const GpuSolver &) = delete;

    /// Solver::Advance(dt) (src/solver.cpp:22-37).  Asynchronous.
    void Advance(double dt) { Check(mpd_advance(h_, dt)); }

    /// Diagnostics::ComputeDt (src/diagnostics.cpp:49-65) of the device state.
    double ComputeDt(double dt_current) {
        double dt = 0.0;
        Check(mpd_compute_dt(h_, cfg_.cfl_number, cfg_.dt_growth_factor, cfg_.dt_min, cfg_.dt_max,
                             dt_current, &dt));
        return dt;
    }
    /// Diagnostics::SolutionChange / Fields::SavePrev of the device state.
    double SolutionChange() {
        double c = 0.0;
        Check(mpd_solution_change(h_, &c));
        return c;
    }
    void SavePrev() { Check(mpd_save_prev(h_)); }

    /// Verification::ComputeIntegrals (src/verification.cpp:16-45) of the device state.
    Verification::ConservedIntegrals ComputeIntegrals() {
        double q[7];
        Check(mpd_integrals(h_, q));
        Verification::ConservedIntegrals c;
        c.mass = q[0];
        c.momentum_z = q[1];
        c.momentum_r = q[2];
        c.momentum_phi = q[3];
        c.energy = q[4];
        c.mag_flux_z = q[5];
        c.mag_flux_phi = q[6];
        return c;
    }

    /// Diagnostics::CheckCfl (src/diagnostics.cpp:112-125) of the device state:
    /// the same warning, printed under the same condition.
    void CheckCfl(double dt, int step_count) {
        double speed = 0.0;
        Check(mpd_max_wave_speed(h_, &speed));
        const double dx = cfg_.dz < cfg_.dy ? cfg_.dz : cfg_.dy;
        const double dt_max = cfg_.cfl_number * dx / (speed + 1.0e-10);
        if (dt > dt_max && step_count % 1000 == 0)
            std::printf("WARNING [step %d]: dt=%.6e exceeds CFL limit dt_max=%.6e "
                        "(max_speed=%.3f, CFL=%.2f)\n",
                        step_count, dt, dt_max, speed, dt / dt_max * cfg_.cfl_number);
    }

    /// The physical values of one global cell (rho, v_z, v_r, v_phi, e, p, P,
    /// H_z, H_r, H_phi), e.g. the driver's checkpoint cell (src/main.cpp:258-270).
    void Probe(int l_global, int m_global, double out10[10]) {
        Check(mpd_probe(h_, l_global, m_global, out10));
    }

    /// Copy the device state into the host Fields (u0_*, u_* and the physical arrays).
    void Download() {
        Array2D *u0[8] = {&f_.u0_1, &f_.u0_2, &f_.u0_3, &f_.u0_4,
                          &f_.u0_5, &f_.u0_6, &f_.u0_7, &f_.u0_8};
        Array2D *u[8] = {&f_.u_1, &f_.u_2, &f_.u_3, &f_.u_4, &f_.u_5, &f_.u_6, &f_.u_7, &f_.u_8};
        Array2D *phys[10] = {&f_.rho, &f_.v_z, &f_.v_r, &f_.v_phi, &f_.e,
                             &f_.p,   &f_.P,   &f_.H_z, &f_.H_r, &f_.H_phi};
        for (int k = 0; k < 8; ++k) {
            Check(mpd_download(h_, k, u0[k]->Flat()));
            std::copy(u0[k]->Flat(), u0[k]->Flat() + u0[k]->Size(), u[k]->Flat());
        }
        for (int k = 0; k < 10; ++k) Check(mpd_download(h_, 8 + k, phys[k]->Flat()));
    }

    mpd_solver *Handle() { return h_; }

private:
    static mpd_field_cond Cond(const FieldCond &fc) {
        mpd_field_cond c{};
        c.type = static_cast<int>(fc.type);
        c.value = fc.value;
        c.expr = fc.type == FieldCondType::Expression ? fc.expr_str.c_str() : nullptr;
        return c;
    }
    static void Check(int rc) {
        if (rc != MPD_OK) throw std::runtime_error(std::string("mpd_b200: ") + mpd_last_error());
    }

    const SimConfig &cfg_;
    Fields &f_;
    std::vector<mpd_bc_segment> segs_[4];
    mpd_solver *h_ = nullptr;
};
