/*
 * dn_oracle.h -- CPU restatement of the reference CHNS time step (TEST INFRASTRUCTURE ONLY).
 *
 * This library is the checker for the CUDA path: a single-threaded plain-C restatement of
 * Hygc0627/ding_nsch_core_solver's coupled time step (the src/core/coupled sources and
 * src/core/linear_algebra/ch_sparse_krylov.hpp), written to reproduce the reference's FP64
 * arithmetic order so that it agrees with the reference build bit for bit.  Only the tests,
 * the smoke check and the CPU-baseline leg of the benchmark may load it; the product path never
 * links or calls it.
 */
#ifndef DN_ORACLE_H
#define DN_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* boundary-condition types, config.hpp:24-28 */
enum { ORC_BC_UNSET = 0, ORC_BC_DIRICHLET = 1, ORC_BC_NEUMANN = 2 };
/* sides, config.hpp:17-22 */
enum { ORC_LEFT = 0, ORC_RIGHT = 1, ORC_BOTTOM = 2, ORC_TOP = 3 };
/* Config::mode values that change the step (solver.cpp:59-67) */
enum { ORC_MODE_COUPLED = 0, ORC_MODE_SINGLE_PHASE = 1, ORC_MODE_ADVECTION_ONLY = 2 };
/* pressure_scheme values handled here (pressure.cpp:1031-1071, aliases folded) */
enum {
  ORC_P_JACOBI = 0,
  ORC_P_ICPCG = 1,
  ORC_P_ILDLT_PCG = 2,
  ORC_P_SPLIT_ICPCG = 3,
  ORC_P_SPLIT_ILDLT_PCG = 4,
  ORC_P_SPLIT_DCDM_ICPCG = 5
};

typedef struct {
  int type;
  double value;
} orc_bc;

/* Numeric mirror of ding::Config (config.hpp:35-136) restricted to the keys the step reads. */
typedef struct {
  int nx, ny, ghost;
  int mode;
  int freeze_ch;
  int pressure_scheme;
  int phase_initializer; /* 0 default, 1 zalesak_disk */
  int velocity_profile;  /* 0 default, 1 solid_body_rotation */
  int invert_phase;
  int periodic_x, periodic_y;
  int ch_inner_iterations, momentum_iterations, poisson_iterations;
  int surface_tension_smoothing_passes;
  double dt, lx, ly, re, ca, pe, cn, density_ratio, viscosity_ratio;
  double surface_tension_multiplier, surface_tension_smoothing_weight;
  double ch_tolerance, pressure_tolerance, momentum_tolerance;
  double body_force_x, body_force_y;
  double interface_center_x, interface_center_y, interface_radius, interface_amplitude, interface_wavenumber;
  double zalesak_slot_width, zalesak_slot_depth;
  double advect_u, advect_v, rotation_center_x, rotation_center_y, angular_velocity;
  double top_wall_velocity_x, bottom_wall_velocity_x;
  orc_bc p_bc[4], u_bc[4], v_bc[4]; /* indexed by ORC_LEFT..ORC_TOP */
  int dcdm_direction_mode;           /* 0 icc_preconditioned, 1 identity (config.hpp:51) */
  int dcdm_history_size, dcdm_max_stored_directions, dcdm_restart_interval; /* config.hpp:72-74 */
} orc_config;

/* Field identifiers (Solver members, solver.hpp:64-91). */
enum {
  ORC_F_C = 0, ORC_F_C_PREV, ORC_F_C_PREV2, ORC_F_MU, ORC_F_RHO, ORC_F_ETA, ORC_F_RHO_PREV, ORC_F_ETA_PREV,
  ORC_F_RHO_MID, ORC_F_ETA_MID, ORC_F_P, ORC_F_P_PREV, ORC_F_P_CORR, ORC_F_U, ORC_F_V, ORC_F_U_PREV, ORC_F_V_PREV,
  ORC_F_U_STAR, ORC_F_V_STAR, ORC_F_SFX_CELL, ORC_F_SFY_CELL, ORC_F_SFX_U, ORC_F_SFY_V, ORC_F_E_PREV,
  ORC_F_HU_PREV, ORC_F_HV_PREV, ORC_F_COUNT
};

/* Per-step report (the Solver::last_* members and Diagnostics the step writes). */
typedef struct {
  int ch_iterations, momentum_iterations, pressure_iterations, coupling_iterations;
  int ch_preconditioner; /* 0 diagonal, 1 ILDLT, 2 diagonal fallback, -1 not used */
  double ch_residual, ch_equation_residual, momentum_residual, pressure_residual;
  double boundary_speed_pre, boundary_speed_post;
} orc_report;

typedef struct {
  double mass, mass_drift, divergence_l2, max_divergence, max_abs_mu, max_velocity, kinetic_energy;
  double total_free_energy, rho_min, rho_max, eta_min, eta_max;
  double dt_limit_advective, dt_limit_capillary, dt_limit_ch_explicit, dt_limit_active, dt_limit_ratio;
} orc_diag;

typedef struct orc_solver orc_solver;

orc_solver *orc_create(const orc_config *cfg);
void orc_destroy(orc_solver *s);
const char *orc_last_error(const orc_solver *s);

/* Field access: ghosted Field2D storage, j contiguous (field.hpp:23-33). */
double *orc_field(orc_solver *s, int id, int *nx, int *ny, int *ghost);
void orc_set_initial_mass(orc_solver *s, double mass);

/* Entry points; each returns 0 on success, non-zero with orc_last_error() set on failure. */
int orc_initialize(orc_solver *s);                 /* Solver::initialize, solver.cpp:69-113 */
int orc_step(orc_solver *s, int step);             /* Solver::advance_one_timestep, solver.cpp:224-283 */
int orc_begin_step(orc_solver *s, int step);       /* history copies, solver.cpp:225-231 */
int orc_phase(orc_solver *s, int step);            /* advance_phase_state, phase_field.cpp:258-281 */
int orc_momentum(orc_solver *s, int step);         /* momentum.cpp:55-85 + 157-502 */
int orc_pressure(orc_solver *s);                   /* solve_pressure_correction, pressure.cpp:1031-1089 */
int orc_correct(orc_solver *s);                    /* apply_pressure_velocity_correction, operators.cpp:480-534 */
int orc_finish_step(orc_solver *s);                /* refresh mu, solver.cpp:274 */
int orc_refresh_derived(orc_solver *s);            /* restart-load rebuild of derived fields, io.cpp:412-436 */
int orc_ch_linear_solve(orc_solver *s, const double *rhs_field, double alpha0, double *c_state,
                        double *iterate_residual, double *equation_residual); /* phase_field.cpp:437-503 */
/* The CH advective term -div(u c) with WENO5 face values (build_phase_advection_fluxes,
 * phase_field.cpp:283-311) of Field2D arrays c (cell), u, v (faces) into rhs (cell, interior + ghosts). */
int orc_advection(orc_solver *s, const double *c, const double *u, const double *v, double *rhs);
/* The CH explicit operator E (build_phase_explicit_operator, phase_field.cpp:354-396) of Field2D arrays c
 * (cell; its ghosts are refilled by the scalar BC), u, v (faces) into E (cell, interior + ghosts). */
int orc_explicit_operator(orc_solver *s, const double *c, const double *u, const double *v, double *E);
/* The CG monitor's per-iteration record of the pressure solve (abs, rel, iterate residual, alpha). */
void orc_set_pressure_monitor(orc_solver *s, int capacity);
int orc_pressure_monitor(const orc_solver *s, double *out, int capacity);
void orc_get_report(const orc_solver *s, orc_report *r);
void orc_diagnostics(orc_solver *s, orc_diag *d); /* diagnostics.cpp:114-167 */
double orc_compute_mass(orc_solver *s, int field_id);

#ifdef __cplusplus
}
#endif
#endif
