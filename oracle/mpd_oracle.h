/*
 * CPU oracle for the Lax-Friedrichs hot path — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference solver's time step, boundary
 * conditions and reductions, used by tests/ and by the CPU-baseline leg of
 * bench.py as the checker.  Nothing in the product path links or calls it.
 *
 * Pinned against the reference itself: oracle/Makefile builds the
 * reference's own translation units (src/solver.cpp, src/fields.cpp,
 * src/face_bc.cpp, src/bcs/per_field_bc.cpp, src/diagnostics.cpp, ...) with
 * single-rank MPI / YAML / exprtk-API shims into oracle/_ref/, and
 * tests/test_oracle_pin.py checks this restatement bit-for-bit against that
 * build; tests/golden/ holds the fixtures generated from it.
 *
 * Storage follows the reference (include/array2d.hpp:6-55, src/mpi_manager.cpp
 * single rank): every plane is (L_max+2) x (M_max+3) doubles, row-major
 * [l][m], l = 0 and l = L_max+1 ghost rows, m = 0 and m = M_max+2 ghost
 * columns, interior l in [1, L_max], m in [1, M_max+1].
 *
 * Physical plane order (Fields members, include/fields.hpp:35-37):
 *   0 rho, 1 v_z, 2 v_r, 3 v_phi, 4 e, 5 p, 6 P, 7 H_z, 8 H_r, 9 H_phi
 * Field-condition order (BCSegmentConfig, include/config.hpp:82-92):
 *   0 rho, 1 v_z, 2 v_r, 3 v_phi, 4 e, 5 H_z, 6 H_r, 7 H_phi
 * Faces (FaceBC::Face, include/face_bc.hpp:52): 0 L_LO, 1 L_HI, 2 M_LO, 3 M_HI
 * Condition types (FieldCondType, include/field_condition.hpp:92-97):
 *   0 Neumann, 1 Dirichlet, 2 Expression, 3 AxisLF
 */
#ifndef MPD_ORACLE_H
#define MPD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mo_case mo_case;

/* params: gamma, beta, H_z0, dz, dy, r_0.  rin/rout/drin/drout: geometry
 * profiles at z = (l-1)*dz for l = 0..L_max+1 (IGeometry evaluated on the
 * host, src/grid.cpp:20-42).  phys: 10 planes of the initial physical state
 * (IInitialCondition::Apply output); u0 is built from it by
 * Fields::InitConservative (src/fields.cpp:40-57). */
mo_case *mo_new(int L_max, int M_max, const double *params, const double *rin,
                const double *rout, const double *drin, const double *drout,
                const double *phys, int with_prev);
void mo_free(mo_case *c);

/* Append one segment to a face (FaceBC::FromConfig, src/face_bc.cpp:23-36).
 * types/values/exprs are in field-condition order. Returns 0 or -1 (err). */
int mo_add_segment(mo_case *c, int face, int global_lo, int global_hi, const int *types,
                   const double *values, const char *const *exprs, char *err, int errlen);

void mo_advance(mo_case *c, double dt);                      /* Solver::Advance */
double mo_max_wave_speed(const mo_case *c);                  /* Diagnostics::MaxWaveSpeed */
double mo_compute_dt(const mo_case *c, double cfl, double growth, double dt_min,
                     double dt_max, double dt_current);     /* Diagnostics::ComputeDt */
double mo_solution_change(const mo_case *c);                 /* Diagnostics::SolutionChange */
void mo_save_prev(mo_case *c);                               /* Fields::SavePrev */
void mo_integrals(const mo_case *c, double *out7);           /* Verification::ComputeIntegrals */
void mo_outlet(const mo_case *c, double *mass_flux, double *thrust); /* GetMassFlux / GetThrust */
double mo_radial_symmetry(const mo_case *c);                 /* Verification::CheckRadialSymmetry */

/* which: 0..7 -> u0_1..u0_8, 8..17 -> physical planes 0..9, 18 -> grid r,
 * 19 -> grid r_z.  Copies the full (L+2)*(M+3) plane. */
void mo_get(const mo_case *c, int which, double *out);

/* Restatement of the driver loop src/main.cpp:191-282 (T clamp, adaptive dt,
 * relative-L2 convergence every check_frequency steps).  run[]: T, dt0,
 * adaptive, cfl, growth, dt_min, dt_max, conv_threshold, check_frequency,
 * max_steps.  out[]: steps, t, dt (next), converged, last change. */
void mo_run(mo_case *c, const double *run, double *out);

#ifdef __cplusplus
}
#endif
#endif
