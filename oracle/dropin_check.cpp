// Drop-in check — TEST INFRASTRUCTURE ONLY (built by `make -C oracle dropin`).
//
// Runs the reference's own driver pattern (src/main.cpp:185-247: Solver,
// Diagnostics::ComputeDt after every step, the relative-L2 check every
// check_frequency steps) twice from the same SimConfig, IGeometry plugin and
// ExpressionIC: once with the reference's Solver on the CPU, once with
// GpuSolver (mpd-plasma-dynamics_b200/host/gpu_solver.hpp) on the GPU in
// exact mode, and compares every Fields array bit for bit.
// The configuration is the reference's config.yaml at a reduced grid,
// filled in code because src/config.cpp needs yaml-cpp.
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "config.hpp"
#include "diagnostics.hpp"
#include "fields.hpp"
#include "geometry_registry.hpp"
#include "gpu_solver.hpp"
#include "grid.hpp"
#include "ics/expression_ic.hpp"
#include "igeometry.hpp"
#include "mpi_manager.hpp"
#include "solver.hpp"

#include <yaml-cpp/yaml.h>

void SimConfig::Init() {
    dz = 1.0 / L_max;
    dy = 1.0 / M_max;
}

namespace {

FieldCond FC(FieldCondType t, double v = 0.0, const char *e = "") {
    FieldCond c;
    c.type = t;
    c.value = v;
    c.expr_str = e;
    return c;
}

SimConfig MakeConfig(int L, int M) {
    using T = FieldCondType;
    SimConfig cfg;
    cfg.gamma = 1.67;
    cfg.beta = 0.01;
    cfg.H_z0 = 0.25;
    cfg.L_max = L;
    cfg.M_max = M;
    cfg.dz = 1.0 / L;
    cfg.dy = 1.0 / M;
    cfg.dt = 1.0e-7;
    cfg.adaptive_dt = true;
    cfg.cfl_number = 0.45;
    cfg.dt_growth_factor = 1.10;
    cfg.dt_min = 1.0e-10;
    cfg.dt_max = 5.0e-5;
    cfg.convergence_threshold = 1e-30;
    cfg.check_frequency = 50;
    BCSegmentConfig lo;
    lo.v_z = FC(T::Dirichlet, 0.0);
    lo.H_z = FC(T::Expression, 0.0, "H_z0");
    lo.H_r = FC(T::Dirichlet, 0.0);
    lo.H_phi = FC(T::Expression, 0.0, "r_0 / r");
    cfg.bc_l_lo.segments = {lo};
    cfg.bc_l_hi.segments = {BCSegmentConfig{}};
    BCSegmentConfig hi;
    hi.v_r = FC(T::Expression, 0.0, "v_z * r_z");
    hi.H_r = FC(T::Expression, 0.0, "H_z * r_z");
    cfg.bc_m_hi.segments = {hi};
    BCSegmentConfig w, tip, axis;
    w.global_lo = 0;
    w.global_hi = 235 * L / 800;
    w.v_r = FC(T::Expression, 0.0, "v_z_nb * r_z_nb");
    w.H_r = FC(T::Expression, 0.0, "H_z_nb * r_z_nb");
    tip.global_lo = 236 * L / 800;
    tip.global_hi = 263 * L / 800;
    tip.rho = FC(T::Dirichlet, 0.1);
    tip.v_phi = FC(T::Dirichlet, 0.0);
    tip.e = FC(T::Expression, 0.0, "beta / (2 * (gamma - 1))");
    tip.H_r = FC(T::Expression, 0.0, "H_z_nb * r_z_nb");
    axis.global_lo = 264 * L / 800;
    axis.global_hi = -1;
    axis.rho = FC(T::AxisLF);
    axis.v_z = FC(T::AxisLF);
    axis.v_r = FC(T::Dirichlet, 0.0);
    axis.v_phi = FC(T::Dirichlet, 0.0);
    axis.e = FC(T::AxisLF);
    axis.H_z = FC(T::AxisLF);
    axis.H_r = FC(T::Dirichlet, 0.0);
    axis.H_phi = FC(T::Dirichlet, 0.0);
    cfg.bc_m_lo.segments = {w, tip, axis};
    return cfg;
}

YAML::Node Params(std::initializer_list<std::pair<const char *, const char *>> kv) {
    YAML::Node n = YAML::Node::MakeMap();
    for (const auto &p : kv) n.Set(p.first, YAML::Node::MakeScalar(p.second));
    return n;
}

bool Same(const Array2D &a, const Array2D &b, const char *what) {
    if (std::memcmp(a.Flat(), b.Flat(), a.Size() * sizeof(double)) == 0) return true;
    std::printf("MISMATCH in %s\n", what);
    return false;
}

}  // namespace

int main(int argc, char **argv) {
    const int L = argc > 1 ? std::atoi(argv[1]) : 80;
    const int M = argc > 2 ? std::atoi(argv[2]) : 40;
    const int steps = argc > 3 ? std::atoi(argv[3]) : 300;
    SimConfig cfg = MakeConfig(L, M);
    int ac = 0;
    char **av = nullptr;
    MPIManager mpi(ac, av, cfg);
    RegisterAllGeometries();
    auto geom = GeometryRegistry::Instance().Create(
        "short_cathode_cosine",
        Params({{"z_center", "0.31"}, {"transition_half_width", "0.02"}, {"r_inner_before", "0.200"},
                {"r_inner_after", "0.005"}, {"r_outer", "0.800"}}));
    ExpressionIC ic(Params({{"rho", "0.1"}, {"v_z", "0.1"}, {"v_r", "0.1"}, {"v_phi", "0.0"},
                            {"H_z", "H_z0"}, {"H_r", "H_z * r_z"},
                            {"H_phi", "(1 - 0.9 * z) * r_0 / r"},
                            {"e", "beta / (2 * (gamma - 1))"}}));
    Grid grid(cfg, mpi.local_L_with_ghosts, mpi.l_start, mpi.local_M_with_ghosts, mpi.m_start, *geom);
    Fields fc(mpi.local_L_with_ghosts, mpi.local_M_with_ghosts, true);
    Fields fg(mpi.local_L_with_ghosts, mpi.local_M_with_ghosts, true);
    for (Fields *f : {&fc, &fg}) {
        f->InitPhysical(ic, cfg, grid, mpi.l_start);
        f->InitConservative(grid);
        f->SavePrev();
    }
    Solver cpu(cfg, mpi, grid, fc);
    GpuSolver gpu(cfg, mpi, grid, fg, MPD_PRECISION_EXACT);

    double dt_c = cfg.dt, dt_g = cfg.dt;
    for (int step = 1; step <= steps; ++step) {
        cpu.Advance(dt_c);
        gpu.Advance(dt_g);
        dt_c = Diagnostics::ComputeDt(fc, cfg, mpi.local_L, mpi.local_M, mpi, dt_c);
        dt_g = gpu.ComputeDt(dt_g);
        if (dt_c != dt_g) {
            std::printf("MISMATCH dt at step %d: %.17g vs %.17g\n", step, dt_c, dt_g);
            return 1;
        }
        if (step % cfg.check_frequency == 0) {
            const double cc = Diagnostics::SolutionChange(fc, mpi.local_L, mpi.local_M);
            const double cg = gpu.SolutionChange();
            fc.SavePrev();
            gpu.SavePrev();
            if (std::abs(cc - cg) > 1e-12 * std::abs(cc)) {
                std::printf("MISMATCH change at step %d: %.17g vs %.17g\n", step, cc, cg);
                return 1;
            }
        }
    }
    gpu.Download();
    bool ok = Same(fc.u0_1, fg.u0_1, "u0_1") && Same(fc.u0_2, fg.u0_2, "u0_2") &&
              Same(fc.u0_3, fg.u0_3, "u0_3") && Same(fc.u0_4, fg.u0_4, "u0_4") &&
              Same(fc.u0_5, fg.u0_5, "u0_5") && Same(fc.u0_6, fg.u0_6, "u0_6") &&
              Same(fc.u0_7, fg.u0_7, "u0_7") && Same(fc.u0_8, fg.u0_8, "u0_8") &&
              Same(fc.rho, fg.rho, "rho") && Same(fc.v_z, fg.v_z, "v_z") &&
              Same(fc.v_r, fg.v_r, "v_r") && Same(fc.v_phi, fg.v_phi, "v_phi") &&
              Same(fc.e, fg.e, "e") && Same(fc.p, fg.p, "p") && Same(fc.P, fg.P, "P") &&
              Same(fc.H_z, fg.H_z, "H_z") && Same(fc.H_r, fg.H_r, "H_r") &&
              Same(fc.H_phi, fg.H_phi, "H_phi");
    // the driver's 1000-step report through GpuSolver: the integrals
    // (Verification::ComputeIntegrals, sums in another order: 1e-13) and the
    // checkpoint cell (bit for bit)
    const Verification::ConservedIntegrals ic_c = Verification::ComputeIntegrals(fc, grid, cfg, mpi);
    const Verification::ConservedIntegrals ic_g = gpu.ComputeIntegrals();
    const double qc[7] = {ic_c.mass, ic_c.momentum_z, ic_c.momentum_r, ic_c.momentum_phi,
                          ic_c.energy, ic_c.mag_flux_z, ic_c.mag_flux_phi};
    const double qg[7] = {ic_g.mass, ic_g.momentum_z, ic_g.momentum_r, ic_g.momentum_phi,
                          ic_g.energy, ic_g.mag_flux_z, ic_g.mag_flux_phi};
    for (int k = 0; k < 7; ++k)
        if (std::abs(qc[k] - qg[k]) > 1e-13 * std::abs(qc[k])) {
            std::printf("MISMATCH integral %d: %.17g vs %.17g\n", k, qc[k], qg[k]);
            ok = false;
        }
    if (L > 20 && M >= 40) {
        double q[10];
        gpu.Probe(20, 40, q);
        const double want[5] = {fc.rho[21][41], fc.v_z[21][41], fc.v_phi[21][41], fc.e[21][41],
                                fc.H_phi[21][41]};
        const double got[5] = {q[0], q[1], q[3], q[4], q[9]};
        for (int k = 0; k < 5; ++k)
            if (got[k] != want[k]) {
                std::printf("MISMATCH probe %d: %.17g vs %.17g\n", k, got[k], want[k]);
                ok = false;
            }
    }
    gpu.CheckCfl(dt_g, steps);
    std::printf("%s after %d steps of %dx%d (dt=%.17g)\n", ok ? "DROPIN OK" : "DROPIN FAIL", steps,
                L, M, dt_c);
    return ok ? 0 : 1;
}
