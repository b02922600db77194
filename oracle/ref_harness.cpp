/*
 * C entry points around the reference's own solver classes — TEST
 * INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile together with the
 * reference's unmodified translation units into oracle/_ref/libmpd_ref.so.
 *
 * It restates only what src/main.cpp does around the solver (main.cpp
 * depends on yaml-cpp and VTK, which are absent): a SimConfig filled
 * directly, one MPI rank, a Grid over tabulated wall profiles, the initial
 * physical planes copied in, Fields::InitConservative, Solver, and the time
 * loop of src/main.cpp:191-282.  The API mirrors oracle/mpd_oracle.h so the
 * tests can drive both with the same inputs.
 */
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "config.hpp"
#include "diagnostics.hpp"
#include "fields.hpp"
#include "geometry_registry.hpp"
#include "grid.hpp"
#include "ics/expression_ic.hpp"
#include "igeometry.hpp"
#include "integrals.hpp"
#include "mpi_manager.hpp"
#include "solver.hpp"
#include "verification.hpp"

#include <yaml-cpp/yaml.h>

// src/config.cpp is not compiled (it needs yaml-cpp), but SimConfig's
// constructor calls its private Init(); restated from src/config.cpp:15-18.
void SimConfig::Init() {
    dz = 1.0 / L_max;
    dy = 1.0 / M_max;
}

namespace {

// Wall profiles sampled on the host at z = (l-1)*dz, l = 0..L_max+1.
class ProfileGeometry : public IGeometry {
public:
    ProfileGeometry(double dz, const double *rin, const double *rout, const double *drin,
                    const double *drout, int n)
        : dz_(dz), rin_(rin, rin + n), rout_(rout, rout + n), drin_(drin, drin + n),
          drout_(drout, drout + n) {}
    [[nodiscard]] auto RInner(double z) const -> double override { return rin_.at(Idx(z)); }
    [[nodiscard]] auto ROuter(double z) const -> double override { return rout_.at(Idx(z)); }
    [[nodiscard]] auto DrInnerDz(double z) const -> double override { return drin_.at(Idx(z)); }
    [[nodiscard]] auto DrOuterDz(double z) const -> double override { return drout_.at(Idx(z)); }
    [[nodiscard]] auto Name() const -> std::string override { return "profile"; }

private:
    [[nodiscard]] std::size_t Idx(double z) const {
        return static_cast<std::size_t>(std::llround(z / dz_) + 1);
    }
    double dz_;
    std::vector<double> rin_, rout_, drin_, drout_;
};

struct RefCase {
    SimConfig cfg;
    std::unique_ptr<MPIManager> mpi;
    std::unique_ptr<ProfileGeometry> geom;
    std::unique_ptr<Grid> grid;
    std::unique_ptr<Fields> fields;
    std::unique_ptr<Solver> solver;
};

Array2D *PhysPlane(Fields &f, int k) {
    Array2D *p[10] = {&f.rho, &f.v_z, &f.v_r, &f.v_phi, &f.e, &f.p, &f.P, &f.H_z, &f.H_r, &f.H_phi};
    return p[k];
}

FieldCond MakeCond(int type, double value, const char *expr) {
    FieldCond fc;
    fc.type = static_cast<FieldCondType>(type);
    fc.value = value;
    if (type == static_cast<int>(FieldCondType::Expression) && expr) fc.expr_str = expr;
    return fc;
}

void CopyErr(const std::exception &e, char *err, int errlen) {
    if (err && errlen > 0) {
        std::strncpy(err, e.what(), static_cast<std::size_t>(errlen - 1));
        err[errlen - 1] = 0;
    }
}

YAML::Node MapFromKv(const char *const *keys, const char *const *vals, int n) {
    YAML::Node node = YAML::Node::MakeMap();
    for (int i = 0; i < n; ++i) node.Set(keys[i], YAML::Node::MakeScalar(vals[i]));
    return node;
}

}  // namespace

extern "C" {

void *ref_new(int L_max, int M_max, const double *params, const double *rin, const double *rout,
              const double *drin, const double *drout, const double *phys, int with_prev) {
    auto *c = new RefCase();
    c->cfg.gamma = params[0];
    c->cfg.beta = params[1];
    c->cfg.H_z0 = params[2];
    c->cfg.L_max = L_max;
    c->cfg.M_max = M_max;
    c->cfg.dz = params[3];
    c->cfg.dy = params[4];
    c->cfg.mpi_dims_l = 1;
    c->cfg.mpi_dims_m = 1;
    int argc = 0;
    char **argv = nullptr;
    c->mpi = std::make_unique<MPIManager>(argc, argv, c->cfg);
    c->geom = std::make_unique<ProfileGeometry>(c->cfg.dz, rin, rout, drin, drout, L_max + 2);
    c->grid = std::make_unique<Grid>(c->cfg, c->mpi->local_L_with_ghosts, c->mpi->l_start,
                                     c->mpi->local_M_with_ghosts, c->mpi->m_start, *c->geom);
    c->fields = std::make_unique<Fields>(c->mpi->local_L_with_ghosts, c->mpi->local_M_with_ghosts,
                                         with_prev != 0);
    const int rows = c->fields->rows, cols = c->fields->cols;
    const std::size_t n = static_cast<std::size_t>(rows) * cols;
    for (int k = 0; k < 10; ++k) {
        Array2D &a = *PhysPlane(*c->fields, k);
        for (int l = 1; l < rows - 1; ++l)
            for (int m = 1; m < cols - 1; ++m) a[l][m] = phys[k * n + static_cast<std::size_t>(l) * cols + m];
    }
    c->fields->InitConservative(*c->grid);
    if (with_prev) c->fields->SavePrev();
    return c;
}

void ref_free(void *h) { delete static_cast<RefCase *>(h); }

int ref_add_segment(void *h, int face, int global_lo, int global_hi, const int *types,
                    const double *values, const char *const *exprs) {
    auto *c = static_cast<RefCase *>(h);
    BCSegmentConfig s;
    s.global_lo = global_lo;
    s.global_hi = global_hi;
    s.rho = MakeCond(types[0], values[0], exprs[0]);
    s.v_z = MakeCond(types[1], values[1], exprs[1]);
    s.v_r = MakeCond(types[2], values[2], exprs[2]);
    s.v_phi = MakeCond(types[3], values[3], exprs[3]);
    s.e = MakeCond(types[4], values[4], exprs[4]);
    s.H_z = MakeCond(types[5], values[5], exprs[5]);
    s.H_r = MakeCond(types[6], values[6], exprs[6]);
    s.H_phi = MakeCond(types[7], values[7], exprs[7]);
    BCFaceConfig *faces[4] = {&c->cfg.bc_l_lo, &c->cfg.bc_l_hi, &c->cfg.bc_m_lo, &c->cfg.bc_m_hi};
    faces[face]->segments.push_back(s);
    return 0;
}

/* Builds the Solver (FaceBC::FromConfig + PerFieldBC validation/compile). */
int ref_finalize(void *h, char *err, int errlen) {
    auto *c = static_cast<RefCase *>(h);
    try {
        c->solver = std::make_unique<Solver>(c->cfg, *c->mpi, *c->grid, *c->fields);
    } catch (const std::exception &e) {
        CopyErr(e, err, errlen);
        return -1;
    }
    return 0;
}

void ref_advance(void *h, double dt) { static_cast<RefCase *>(h)->solver->Advance(dt); }

double ref_grid_r0(void *h) { return static_cast<RefCase *>(h)->grid->r_0; }

double ref_max_wave_speed(void *h) {
    auto *c = static_cast<RefCase *>(h);
    return Diagnostics::MaxWaveSpeed(*c->fields, c->cfg, c->mpi->local_L, c->mpi->local_M, *c->mpi);
}

double ref_compute_dt(void *h, double cfl, double growth, double dt_min, double dt_max,
                      double dt_current) {
    auto *c = static_cast<RefCase *>(h);
    c->cfg.cfl_number = cfl;
    c->cfg.dt_growth_factor = growth;
    c->cfg.dt_min = dt_min;
    c->cfg.dt_max = dt_max;
    return Diagnostics::ComputeDt(*c->fields, c->cfg, c->mpi->local_L, c->mpi->local_M, *c->mpi,
                                  dt_current);
}

double ref_solution_change(void *h) {
    auto *c = static_cast<RefCase *>(h);
    return Diagnostics::SolutionChange(*c->fields, c->mpi->local_L, c->mpi->local_M);
}

void ref_save_prev(void *h) { static_cast<RefCase *>(h)->fields->SavePrev(); }

void ref_integrals(void *h, double *out7) {
    auto *c = static_cast<RefCase *>(h);
    const auto q = Verification::ComputeIntegrals(*c->fields, *c->grid, c->cfg, *c->mpi);
    const double v[7] = {q.mass, q.momentum_z, q.momentum_r, q.momentum_phi,
                         q.energy, q.mag_flux_z, q.mag_flux_phi};
    std::memcpy(out7, v, sizeof(v));
}

void ref_outlet(void *h, double *mass_flux, double *thrust) {
    auto *c = static_cast<RefCase *>(h);
    *mass_flux = Diagnostics::GetMassFlux(*c->fields, *c->grid, c->cfg, *c->mpi);
    *thrust = Diagnostics::GetThrust(*c->fields, *c->grid, c->cfg, *c->mpi);
}

double ref_radial_symmetry(void *h) {
    auto *c = static_cast<RefCase *>(h);
    return Verification::CheckRadialSymmetry(*c->fields, *c->mpi);
}

void ref_get(void *h, int which, double *out) {
    auto *c = static_cast<RefCase *>(h);
    Fields &f = *c->fields;
    Array2D *u0[8] = {&f.u0_1, &f.u0_2, &f.u0_3, &f.u0_4, &f.u0_5, &f.u0_6, &f.u0_7, &f.u0_8};
    const Array2D *src = nullptr;
    if (which >= 0 && which < 8) src = u0[which];
    else if (which >= 8 && which < 18) src = PhysPlane(f, which - 8);
    else if (which == 18) src = &c->grid->r;
    else if (which == 19) src = &c->grid->r_z;
    if (src) std::memcpy(out, src->Flat(), src->Size() * sizeof(double));
}

/* src/main.cpp:191-282, without printing and I/O. */
void ref_run(void *h, const double *run, double *out) {
    auto *c = static_cast<RefCase *>(h);
    c->cfg.T = run[0];
    c->cfg.dt = run[1];
    c->cfg.adaptive_dt = run[2] != 0.0;
    c->cfg.cfl_number = run[3];
    c->cfg.dt_growth_factor = run[4];
    c->cfg.dt_min = run[5];
    c->cfg.dt_max = run[6];
    c->cfg.convergence_threshold = run[7];
    c->cfg.check_frequency = static_cast<int>(run[8]);
    const long max_steps = static_cast<long>(run[9]);
    double t = 0.0, dt = c->cfg.dt, change = 0.0;
    long step = 0;
    bool converged = false;
    while (t < c->cfg.T && !converged && step < max_steps) {
        if (t + dt > c->cfg.T) dt = c->cfg.T - t;
        c->solver->Advance(dt);
        t += dt;
        ++step;
        if (c->cfg.adaptive_dt)
            dt = Diagnostics::ComputeDt(*c->fields, c->cfg, c->mpi->local_L, c->mpi->local_M,
                                        *c->mpi, dt);
        if (c->cfg.convergence_threshold > 0.0 && step % c->cfg.check_frequency == 0) {
            change = Diagnostics::SolutionChange(*c->fields, c->mpi->local_L, c->mpi->local_M);
            if (change < c->cfg.convergence_threshold) converged = true;
            c->fields->SavePrev();
        }
    }
    out[0] = static_cast<double>(step);
    out[1] = t;
    out[2] = dt;
    out[3] = converged ? 1.0 : 0.0;
    out[4] = change;
}

/* The reference's geometry plugins through its own registry
 * (src/geometry_registry.cpp:15-65), sampled at z = (l-1)*dz. */
int ref_geometry_profile(const char *type, const char *const *keys, const char *const *vals,
                         int nkv, int L_max, double dz, double *rin, double *rout, double *drin,
                         double *drout, char *err, int errlen) {
    try {
        RegisterAllGeometries();
        YAML::Node params = nkv > 0 ? MapFromKv(keys, vals, nkv) : YAML::Node();
        auto geom = GeometryRegistry::Instance().Create(type, params);
        for (int l = 0; l < L_max + 2; ++l) {
            const int l_global = l - 1;
            const double z = l_global * dz;
            rin[l] = geom->RInner(z);
            rout[l] = geom->ROuter(z);
            drin[l] = geom->DrInnerDz(z);
            drout[l] = geom->DrOuterDz(z);
        }
    } catch (const std::exception &e) {
        CopyErr(e, err, errlen);
        return -1;
    }
    return 0;
}

/* The reference's ExpressionIC (src/ics/expression_ic.cpp:255-324) on a
 * Grid over tabulated profiles; writes the 10 physical planes. */
int ref_expression_ic(const char *const *keys, const char *const *vals, int nkv, int L_max,
                      int M_max, const double *params, const double *rin, const double *rout,
                      const double *drin, const double *drout, double *phys_out, char *err,
                      int errlen) {
    try {
        SimConfig cfg;
        cfg.gamma = params[0];
        cfg.beta = params[1];
        cfg.H_z0 = params[2];
        cfg.L_max = L_max;
        cfg.M_max = M_max;
        cfg.dz = params[3];
        cfg.dy = params[4];
        ProfileGeometry geom(cfg.dz, rin, rout, drin, drout, L_max + 2);
        Grid grid(cfg, L_max + 2, 0, M_max + 3, 0, geom);
        Fields f(L_max + 2, M_max + 3, false);
        YAML::Node node = nkv > 0 ? MapFromKv(keys, vals, nkv) : YAML::Node();
        ExpressionIC ic(node);
        ic.Apply(f, grid, cfg, 0);
        const std::size_t n = static_cast<std::size_t>(f.rows) * f.cols;
        for (int k = 0; k < 10; ++k) std::memcpy(phys_out + k * n, PhysPlane(f, k)->Flat(), n * sizeof(double));
    } catch (const std::exception &e) {
        CopyErr(e, err, errlen);
        return -1;
    }
    return 0;
}

}  // extern "C"
