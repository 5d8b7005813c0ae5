/*
 * dn_cuda.h -- C-ABI of the B200 (sm_100a) CHNS time-step library, libdn_cuda.so.
 *
 * The library replaces, as a drop-in backend, the hot path of Hygc0627/ding_nsch_core_solver's coupled
 * solver: one time step on the 2D MAC grid (Cahn-Hilliard implicit solve, momentum predictor, pressure
 * correction).  Every entry point is `extern "C"`, takes plain pointers and sizes, returns a dn_status and
 * never throws or aborts.  A handle owns its device memory and one CUDA stream; calls on one handle must
 * be serialised by the caller, different handles are independent.
 *
 * Field arrays exchanged with the host use the reference's Field2D layout (src/core/base/field.hpp:9-36):
 * FP64, (nx'+2g) x (ny'+2g) values with j (the y index) contiguous, where nx' = nx+1 for u-type fields,
 * ny' = ny+1 for v-type fields, and g = ghost (3).
 */
#ifndef DN_CUDA_H
#define DN_CUDA_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  Messages (dn_status_string) mirror the reference's std::runtime_error texts. */
typedef enum {
  DN_OK = 0,
  DN_ERR_INVALID_ARGUMENT = 1,   /* bad size / pointer / config value                                  */
  DN_ERR_CONFIG = 2,             /* config.cpp:49-208 parse errors, operators.cpp:11-34 BC validation  */
  DN_ERR_CUDA = 3,               /* a CUDA runtime call failed                                           */
  DN_ERR_ICC_FAILED = 4,         /* pressure.cpp:36-38  "ICC preconditioner construction failed"       */
  DN_ERR_ILDLT_FAILED = 5,       /* pressure.cpp:44-46  "ILDLT preconditioner construction failed"     */
  DN_ERR_PCG_BREAKDOWN = 6,      /* ch_sparse_krylov.hpp:566-568, 588-590, 631-633                      */
  DN_ERR_BICGSTAB_BREAKDOWN = 7, /* ch_sparse_krylov.hpp:887-938                                       */
  DN_ERR_TIMEOUT = 8,            /* a device-side wait (grid barrier / wavefront flag) gave up         */
  DN_ERR_NONFINITE = 9,          /* solver.cpp:355-364 "non-finite diagnostic detected"                */
  DN_ERR_UNSUPPORTED = 10        /* a config the CUDA path does not implement (see message)            */
} dn_status;

typedef enum { DN_BC_UNSET = 0, DN_BC_DIRICHLET = 1, DN_BC_NEUMANN = 2 } dn_bc_type;          /* config.hpp:24-28 */
typedef enum { DN_LEFT = 0, DN_RIGHT = 1, DN_BOTTOM = 2, DN_TOP = 3 } dn_side;                 /* config.hpp:17-22 */
typedef enum { DN_MODE_COUPLED = 0, DN_MODE_SINGLE_PHASE = 1, DN_MODE_ADVECTION_ONLY = 2 } dn_mode;
/* pressure_scheme (pressure.cpp:1031-1071; reference aliases liu_/paper_ fold onto these; the new config
 * values cuda_icpcg / cuda_ildlt_pcg / cuda_split_icpcg / cuda_split_ildlt_pcg select the same schemes). */
typedef enum {
  DN_P_JACOBI = 0,
  DN_P_ICPCG = 1,
  DN_P_ILDLT_PCG = 2,
  DN_P_SPLIT_ICPCG = 3,
  DN_P_SPLIT_ILDLT_PCG = 4,
  DN_P_SPLIT_DCDM_ICPCG = 5 /* conjugate directions (pressure.cpp:367-468) */
} dn_pressure_scheme;
/* arithmetic of the Krylov inner loops: plain FP64, or FP32 inner solves wrapped in FP64 defect correction */
typedef enum { DN_PRECISION_FP64 = 0, DN_PRECISION_MIXED = 1 } dn_precision;
typedef enum { DN_MIXED_PREC_MULTIGRID = 0, DN_MIXED_PREC_IC = 1 } dn_mixed_preconditioner;

typedef struct {
  int type; /* dn_bc_type */
  double value;
} dn_bc;

/* Numeric image of ding::Config (config.hpp:35-136), keys the time step reads. */
typedef struct {
  int nx, ny, ghost;
  int mode;            /* dn_mode */
  int freeze_ch;
  int pressure_scheme; /* dn_pressure_scheme */
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
  dn_bc p_bc[4], u_bc[4], v_bc[4]; /* indexed by dn_side */
  int precision;                   /* dn_precision */
  double mixed_inner_tolerance;    /* relative tolerance of each FP32 inner solve (mixed form) */
  int device_share;                /* handles meant to run concurrently on one device (dn_step_batch): each
                                      persistent launch takes at most 1/device_share of the SMs, never fewer
                                      CTAs than its wavefront needs; 1 = the whole device */
  int dcdm_direction_mode;         /* split_dcdm_icpcg directions: 0 icc_preconditioned, 1 identity (config.hpp:51) */
  int dcdm_history_size, dcdm_max_stored_directions, dcdm_restart_interval; /* config.hpp:72-74 */
  int pcg_rows_per_cta;            /* launch shape of the pressure PCG: rows per CTA of its SpMV / update
                                      phases (0: 512) -- see dn_autotune_pressure */
  int sweep_warps_per_cta;         /* sweep warps per CTA of the staged wavefront (0: as many as fit, up to 4) */
  int device_wait_limit;           /* polls after which a device-side wait (grid barrier, wavefront hand-over)
                                      gives up and the call returns DN_ERR_TIMEOUT (0: the default, 2^22, well
                                      under a few seconds) */
  int mixed_preconditioner;        /* dn_mixed_preconditioner: preconditioner of the FP32 inner CG of the mixed
                                      form (0: geometric multigrid V-cycle where the grid coarsens to <= 128
                                      cells, else the scheme's own IC(0)/ILDLT(0); 1: always IC/ILDLT).  With 0
                                      the CH solve also runs the mixed form (FP32 CG, two V-cycles of the
                                      shifted Laplacian K + sqrt(alpha0/beta2) I as preconditioner); with 1 it
                                      stays FP64 ILDLT-PCG */
  int mg_cluster_cells;            /* level-0 grids up to this many cells run each multigrid inner CG solve as
                                      one thread-block cluster launch (0 or negative: never, a launch per
                                      phase recorded in the solve's graph) */
  /* pressure analysis (config.hpp:36-133; run_pressure_analysis_from_snapshot, pressure_analysis.cpp:156-328) */
  int analysis_enabled;            /* analysis_enabled */
  int analysis_mode;               /* dn_analysis_mode, from the analysis_mode string */
  int analysis_trigger_step;       /* the step (1-based, current_step_index + 1) that is analysed */
  double analysis_interface_band_multiplier;
  char name[128];                  /* case name: output_dir/name/pressure_analysis/name_<mode>_step_NNNNNN_* */
  char output_dir[512];
  char analysis_case_group[128];
  char analysis_initial_guess[64];
  char analysis_nullspace_treatment[64];
  char analysis_spectrum_iterations[256]; /* iterations whose residual field is written ("final" ignored) */
} dn_config;

/* analysis_mode: "online" after the step's pressure solve, "frozen" before it, "both"; anything else off */
typedef enum { DN_ANALYSIS_OFF = 0, DN_ANALYSIS_ONLINE = 1, DN_ANALYSIS_FROZEN = 2, DN_ANALYSIS_BOTH = 3 } dn_analysis_mode;

/* Fields (Solver members, src/core/coupled/solver.hpp:64-91). */
typedef enum {
  DN_F_C = 0, DN_F_C_PREV, DN_F_C_PREV2, DN_F_MU, DN_F_RHO, DN_F_ETA, DN_F_RHO_PREV, DN_F_ETA_PREV,
  DN_F_RHO_MID, DN_F_ETA_MID, DN_F_P, DN_F_P_PREV, DN_F_P_CORR, DN_F_U, DN_F_V, DN_F_U_PREV, DN_F_V_PREV,
  DN_F_U_STAR, DN_F_V_STAR, DN_F_SFX_CELL, DN_F_SFY_CELL, DN_F_SFX_U, DN_F_SFY_V, DN_F_E_PREV,
  DN_F_HU_PREV, DN_F_HV_PREV, DN_F_COUNT
} dn_field;

/* What one step (or one backend call) reports: Solver::last_* members (solver.hpp:93-108). */
typedef struct {
  int ch_iterations, momentum_iterations, pressure_iterations, coupling_iterations;
  int ch_preconditioner; /* 0 diagonal, 1 ILDLT, 2 diagonal fallback after a breakdown, -1 not used,
                            3 mixed form: FP32 CG preconditioned by (K + s I)^-2 V-cycles */
  double ch_residual, ch_equation_residual, momentum_residual, pressure_residual;
  double boundary_speed_pre, boundary_speed_post;
  int refinement_cycles; /* mixed form: outer FP64 defect-correction cycles of the pressure solve */
  int mixed_inner_multigrid; /* mixed form: 1 when the inner solves started with the multigrid preconditioner */
} dn_report;

/* Diagnostics (src/core/base/diagnostics.hpp; computed as in diagnostics.cpp:114-167). */
typedef struct {
  double mass, mass_drift, divergence_l2, max_divergence, max_abs_mu, max_velocity, kinetic_energy;
  double total_free_energy, rho_min, rho_max, eta_min, eta_max;
  double dt_limit_advective, dt_limit_capillary, dt_limit_ch_explicit, dt_limit_active, dt_limit_ratio;
} dn_diag;

typedef struct dn_handle dn_handle;

/* ---- configuration ------------------------------------------------------------------------------- */
/* Defaults of struct Config (config.hpp:35-136). */
void dn_config_default(dn_config *cfg);
/* Parse a reference case file (`key = value`, `#` comments) -- replaces ding::load_config (config.cpp:49-208).
 * Accepts the reference's pressure_scheme spellings and the new cuda_* values.  `err` may be NULL. */
dn_status dn_config_parse(const char *text, dn_config *cfg, char *err, size_t err_len);

/* ---- lifetime ------------------------------------------------------------------------------------ */
/* Replaces ding::Solver::Solver (solver.cpp:25-57): allocates every field on `device` (-1 = current). */
dn_status dn_create(const dn_config *cfg, int device, dn_handle **out);
dn_status dn_destroy(dn_handle *h);
const char *dn_status_string(dn_status s);
/* Message of the last failure on this handle (reference wording where one exists). */
const char *dn_last_error(const dn_handle *h);

/* ---- state ----------------------------------------------------------------------------------------- */
/* Solver::initialize (solver.cpp:69-113) on the device: built-in phase / velocity initialisers. */
dn_status dn_initialize(dn_handle *h);
/* Host <-> device copy of one Field2D-layout field (`count` doubles, checked against the field size). */
dn_status dn_set_field(dn_handle *h, int field, const double *host, size_t count);
dn_status dn_get_field(dn_handle *h, int field, double *host, size_t count);
/* Device-pointer access for callers that keep their own device buffers (same layout). */
dn_status dn_field_device_ptr(dn_handle *h, int field, double **dev_ptr, size_t *count);
void dn_set_initial_mass(dn_handle *h, double mass);
/* After injecting c, c_prev, p, p_prev, u, v, E_prev, H_prev with dn_set_field, rebuild the derived fields
 * exactly as a restart does (io.cpp:412-436): BC ghosts, rho/eta (n and n-1), midpoint materials, mu. */
dn_status dn_refresh_derived(dn_handle *h);

/* ---- the time step and its phases (each replaces the cited reference member) ------------------------ */
/* Solver::advance_one_timestep (solver.cpp:224-283). */
dn_status dn_step(dn_handle *h, int step, dn_report *rep);
/* Batched ensemble (the reference runs one Solver per process; here many handles share the device): one
 * dn_step of each of `count` distinct handles, run concurrently -- each on its own stream from a host worker
 * thread -- so that many small instances fill the GPU.  steps[a] is handle a's step index (NULL: 0);
 * reports (NULL allowed) receives one dn_report per handle.  Each handle's result equals its dn_step alone.
 * Returns the first failing handle's status (its message via dn_last_error).  The CUDA runtime maps streams
 * onto CUDA_DEVICE_MAX_CONNECTIONS hardware queues (8 unless the environment sets it before the process
 * creates its CUDA context; up to 32), and streams that share a queue serialise.  When every handle has
 * captured steps enabled (dn_set_step_graph) and its step can be captured, the batch is instead one CUDA
 * graph holding every handle's step as a branch, recorded on the first such call for this list of handles
 * and launched once per call. */
dn_status dn_step_batch(dn_handle *const *handles, int count, const int *steps, dn_report *reports);
/* Captured steps (no reference counterpart): with enable != 0, a step of index >= 1 that follows an eager
 * step of index >= 1 is recorded once into a CUDA graph and replayed from then on.  The graph holds every
 * launch of the step; the loops of the solves run on the device as conditional graph nodes, whose
 * conditions kernels set from the same residual checks as the eager step.  The host reads the step's
 * results once, after the replay.  Results, iteration counts and reports equal the eager step's.  Steps
 * that need host decisions run eagerly: step 0; a changed CH operator; the DCDM and Jacobi schemes; the
 * pressure analysis; an active pressure monitor.  A launch-shape change (dn_autotune_pressure) records the
 * step again. */
dn_status dn_set_step_graph(dn_handle *h, int enable);
/* history copies at the start of advance_one_timestep (solver.cpp:225-231) */
dn_status dn_begin_step(dn_handle *h, int step);
/* Solver::advance_phase_state (phase_field.cpp:258-281): CH solve, materials, surface force */
dn_status dn_phase(dn_handle *h, int step, dn_report *rep);
/* compute_momentum_fluxes + solve_momentum_predictor (momentum.cpp:55-85, 157-502) */
dn_status dn_momentum(dn_handle *h, int step, dn_report *rep);
/* Solver::solve_pressure_correction (pressure.cpp:1031-1089) for the configured scheme */
dn_status dn_pressure(dn_handle *h, dn_report *rep);
/* Solver::apply_pressure_velocity_correction (operators.cpp:480-534) */
dn_status dn_correct(dn_handle *h, dn_report *rep);

/* ---- backend entry points with host buffers (what a reference-side binding calls) ------------------ */
/* CH backend: replaces Solver::solve_phase_linear_system_eq25 (phase_field.cpp:437-503) for
 * ch_solver = cuda_sparse_pcg.  rhs_field, c_state: Field2D layout (nx x ny cell field); c_state in/out. */
dn_status dn_ch_linear_solve(dn_handle *h, const double *rhs_field, double alpha0, double *c_state,
                             double *iterate_residual, double *equation_residual, int *iterations);
/* Pressure backend: replaces Solver::solve_pressure_correction_{icpcg,ildlt_pcg,liu_split_icpcg,
 * liu_split_ildlt_pcg} (pressure.cpp:302-365, 470-491).  Inputs u_star, v_star, rho_mid, p, p_prev
 * (Field2D layout), step index (split extrapolation); output p_corr (Field2D, ghosts filled). */
dn_status dn_pressure_solve(dn_handle *h, int step, const double *u_star, const double *v_star,
                            const double *rho_mid, const double *p, const double *p_prev, double *p_corr,
                            int *iterations, double *relative_residual);

/* Size of the fixed device array that dn_pressure_solve_static works in (16 MiB; the grid's operator,
 * factor, Krylov vectors and sync words need about 165 bytes per cell, so up to about 100,000 cells). */
#define DN_STATIC_SCRATCH_BYTES (16u * 1024u * 1024u)
/* No counterpart in the reference.  The pressure solve of dn_pressure_solve for callers that cannot
 * allocate device memory at the point of the solve (a caching pool that already holds the GPU's memory,
 * a loop that must not stall on cudaMalloc, code holding only raw device pointers and no handle).  No
 * handle and no allocation: inputs u_star, v_star, rho_mid, p, p_prev and the output p_corr are the
 * caller's DEVICE buffers in Field2D layout for `cfg`'s grid; the work runs on `stream` (a cudaStream_t,
 * NULL for the default stream), which must belong to the current device (else DN_ERR_INVALID_ARGUMENT).
 * The call reads status words back and synchronises the stream in the middle of the solve and before it
 * returns, so it cannot be used inside stream capture at all.  Scratch lives in one static device array
 * of DN_STATIC_SCRATCH_BYTES that every GPU loading the library holds until exit; grids that need more
 * return DN_ERR_UNSUPPORTED.  Each call looks the array's device address up with the current device's
 * context (so a re-created context is safe).  All calls share the array, so calls overlapping in time on
 * one device race.  The launch shape is the default a handle would use for `cfg` (device_share
 * included); shapes picked by dn_autotune_pressure are not reproduced.  On error a message goes to `err`
 * (`err_len` bytes, may be NULL). */
dn_status dn_pressure_solve_static(const dn_config *cfg, int step, const double *u_star, const double *v_star,
                                   const double *rho_mid, const double *p, const double *p_prev, double *p_corr,
                                   void *stream, int *iterations, double *relative_residual, char *err,
                                   size_t err_len);

/* ---- differentiation of the projection ---------------------------------------------------------------- */
/* The pressure projection of one step on caller DEVICE buffers (Field2D layouts of the handle's u, v and
 * cell fields): u_star, v_star, p, p_prev in; u, v, p_new and p_prev_new (= p) out, as
 * solve_pressure_correction + apply_pressure_velocity_correction (pressure.cpp:1031-1089,
 * operators.cpp:480-534) compute them, with the handle's rho_mid.  Uses the handle's fields as work space.
 * Only interior values of the inputs are read. */
dn_status dn_projection(dn_handle *h, int step, const double *u_star, const double *v_star, const double *p,
                        const double *p_prev, double *u, double *v, double *p_new, double *p_prev_new,
                        int *iterations, double *relative_residual);
/* No counterpart in the reference (it has no adjoint).  Vector-Jacobian product of dn_projection with
 * rho_mid held fixed: cotangents gu, gv, gp, gpp of the interior values of u, v, p_new, p_prev_new in;
 * cotangents au, av, ap, app of the interior values of u_star, v_star, p, p_prev out (ghosts set to 0).  The
 * transposed pressure solve is the same PCG (the operator is symmetric), so it reports its iterations and
 * relative residual; the handle's rho_mid must be the one of the forward call.  DEVICE buffers. */
dn_status dn_projection_adjoint(dn_handle *h, int step, const double *gu, const double *gv, const double *gp,
                                const double *gpp, double *au, double *av, double *ap, double *app,
                                int *iterations, double *relative_residual);
/* dn_projection with rho_mid as an input (its scalar BC applied), and the vector-Jacobian product with the
 * cotangent of rho_mid as well (the forward's p, p_prev and p_new in; arho out).  No counterpart in the
 * reference.  DEVICE buffers. */
dn_status dn_projection_rho(dn_handle *h, int step, const double *u_star, const double *v_star, const double *p,
                            const double *p_prev, const double *rho_mid, double *u, double *v, double *p_new,
                            double *p_prev_new, int *iterations, double *relative_residual);
dn_status dn_projection_rho_adjoint(dn_handle *h, int step, const double *rho_mid, const double *p,
                                    const double *p_prev, const double *p_new, const double *gu, const double *gv,
                                    const double *gp, const double *gpp, double *au, double *av, double *ap,
                                    double *app, double *arho, int *iterations, double *relative_residual);
/* The momentum predictor as a map (compute_momentum_fluxes + solve_momentum_predictor, momentum.cpp:55-85,
 * 157-502): u, v (their BCs applied), H_prev (hu_prev, hv_prev), the face surface forces (fxu, fyv) and the
 * materials rho_mid, eta, eta_prev (scalar BCs applied) in; u_star, v_star and this step's convection H
 * (hu, hv: the next step's H_prev) out.  DEVICE Field2D buffers; uses the handle's fields as work space. */
dn_status dn_momentum_map(dn_handle *h, int step, const double *u, const double *v, const double *hu_prev,
                          const double *hv_prev, const double *fxu, const double *fyv, const double *rho_mid,
                          const double *eta, const double *eta_prev, double *u_star, double *v_star, double *hu,
                          double *hv, int *iterations, double *residual);
/* No counterpart in the reference.  Vector-Jacobian product of dn_momentum_map at its forward point (the same
 * u, v, hu_prev, hv_prev, rho_mid, eta, eta_prev, and the forward's u_star, v_star): cotangents of the
 * interior values of u_star, v_star, hu, hv in; cotangents of the interior values of u, v, hu_prev,
 * hv_prev, fxu, fyv, rho_mid, eta, eta_prev out (ghosts 0).  The transposed coupled system M^T is solved by
 * the same Jacobi-BiCGSTAB to a relative residual of 1e-14; its iterations and relative residual are
 * reported.  DEVICE buffers. */
dn_status dn_momentum_adjoint(dn_handle *h, int step, const double *u, const double *v, const double *hu_prev,
                              const double *hv_prev, const double *rho_mid, const double *eta, const double *eta_prev,
                              const double *u_star, const double *v_star, const double *gu_star,
                              const double *gv_star, const double *ghu, const double *ghv, double *au, double *av,
                              double *ahu, double *ahv, double *afu, double *afv, double *arho, double *aeta,
                              double *aeta_prev, int *iterations, double *residual);
/* The face surface forces as a map (update_surface_tension_force, phase_field.cpp:179-256): c_old, c_new
 * (scalar BCs applied) in; fxu, fyv out (face BCs and smoothing passes applied).  DEVICE buffers. */
dn_status dn_surface_force_map(dn_handle *h, const double *c_old, const double *c_new, double *fxu, double *fyv);
/* No counterpart in the reference.  Vector-Jacobian product of dn_surface_force_map at (c_old, c_new):
 * cotangents of the interior face forces in; cotangents of the interior values of c_old and c_new out.
 * DN_ERR_UNSUPPORTED with smoothing passes.  DEVICE buffers. */
dn_status dn_surface_force_adjoint(dn_handle *h, const double *c_old, const double *c_new, const double *gfxu,
                                   const double *gfyv, double *ac_old, double *ac_new);

/* The CH advective term -div(u c) with WENO5 face values, as build_phase_advection_fluxes
 * (phase_field.cpp:283-311) computes it, on caller DEVICE buffers: c (cell field), u, v (face fields) in,
 * rhs (cell field, ghosts filled) out.  Uses the handle's work fields. */
dn_status dn_advection(dn_handle *h, const double *c, const double *u, const double *v, double *rhs);
/* No counterpart in the reference.  Vector-Jacobian product of dn_advection at (c, u, v), the WENO5
 * nonlinear weights differentiated: cotangent g_rhs of the interior of rhs in; cotangents c_bar, u_bar,
 * v_bar of the interior values of c, u, v out (ghosts 0).  The upwind choice follows the sign of each face
 * velocity, so the map is not differentiable where a face velocity is exactly 0.  DEVICE buffers. */
dn_status dn_advection_adjoint(dn_handle *h, const double *c, const double *u, const double *v, const double *g_rhs,
                               double *c_bar, double *u_bar, double *v_bar);

/* The CH explicit operator E(c, u, v) of the phase step (build_phase_explicit_operator,
 * phase_field.cpp:354-396: diffusion of the chemical potential with the c(1-c) mobility, the linear
 * Laplacian terms and the WENO5 advective term) on caller DEVICE buffers: c (cell field), u, v (face fields)
 * in, E (cell field, ghosts filled) out.  Uses the handle's work fields. */
dn_status dn_explicit_operator(dn_handle *h, const double *c, const double *u, const double *v, double *E);
/* No counterpart in the reference.  Vector-Jacobian product of dn_explicit_operator at (c, u, v): cotangent
 * gE of the interior of E in; cotangents c_bar, u_bar, v_bar of the interior values of c, u, v out (ghosts
 * 0).  The mobility max(0, c(1-c)) and the upwind choice of the advective term are piecewise smooth; the
 * derivative is taken on the side the forward evaluation lies on.  DEVICE buffers. */
dn_status dn_explicit_operator_adjoint(dn_handle *h, const double *c, const double *u, const double *v,
                                       const double *gE, double *c_bar, double *u_bar, double *v_bar);

/* ---- pressure analysis ------------------------------------------------------------------------------------ */
/* Solver::run_pressure_analysis_from_snapshot (pressure_analysis.cpp:156-328) on the handle's current state,
 * whose step index is `step` (the files carry step + 1, as the reference's snapshot does): the pressure system
 * as the configured scheme assembles it, a PCG from x = 0 with ICC (ILDLT for the ILDLT schemes; the diagonal
 * when the factor fails), and under output_dir/name/pressure_analysis/ the per-iteration file
 * <name>_<source_mode>_step_NNNNNN_pcg.csv, the fields rhs, interface_mask, rho_mid, phi, residual_iter_NNNNNN
 * and residual_final in <stem>_fields/, and one appended row of summary.csv.  dn_step runs it itself at
 * analysis_trigger_step when analysis_enabled: "frozen" before the pressure solve, "online" after it (PCG
 * schemes only), as the reference's step does (solver.cpp:270, pressure.cpp:1078-1087). */
dn_status dn_pressure_analysis(dn_handle *h, int step, const char *source_mode);

/* ---- launch-shape autotuning ----------------------------------------------------------------------------- */
/* No counterpart in the reference.  Times one pressure solve of the handle's current state (u*, v*, rho_mid,
 * p, p_prev as a step leaves them) for each launch shape -- rows per CTA of the PCG's SpMV / update phases
 * in {256 .. 4096} x sweep warps per CTA of the staged wavefront -- twice, and keeps the fastest of the
 * second pass on the handle.  Outputs (each may be NULL): the chosen shape and its pressure-solve time. */
dn_status dn_autotune_pressure(dn_handle *h, int *rows_per_cta, int *sweep_warps_per_cta, double *best_ms);

/* ---- CG monitor ---------------------------------------------------------------------------------------- */
/* The per-iteration record of the pressure solve that the reference's CG monitor receives
 * (ch_sparse_krylov.hpp:515-660; read by the pressure analysis, pressure.cpp / pressure_analysis.cpp:156-328).
 * dn_set_pressure_monitor keeps up to `capacity` iterations of every later FP64 pressure solve (0 turns it
 * off; allocates a device record).  dn_pressure_monitor copies the last solve's record into out,
 * [iteration][4] = absolute residual, relative residual, iterate residual, alpha, for up to `capacity`
 * iterations; *count receives how many the solve recorded.  The mixed form records nothing. */
dn_status dn_set_pressure_monitor(dn_handle *h, int capacity);
dn_status dn_pressure_monitor(dn_handle *h, double *out, int capacity, int *count);

/* ---- history.csv --------------------------------------------------------------------------------------- */
/* Solver::write_history_csv_header (io.cpp:179-185): the header line; returns its length (buf may be NULL). */
size_t dn_history_csv_header(char *buf, size_t len);
/* Solver::append_history_csv_entry (io.cpp:187-202): the history row of the step just taken (its report
 * `rep`, the device diagnostics, the solver names and the dt-limit source), doubles at 17 significant
 * digits, newline-terminated, into buf (len bytes); *written (may be NULL) receives its length. */
dn_status dn_history_csv_row(dn_handle *h, int step, double time, const dn_report *rep, char *buf, size_t len,
                             size_t *written);

/* ---- restart snapshots --------------------------------------------------------------------------------- */
/* Solver::write_restart_snapshot (io.cpp:271-343): the reference's v2 snapshot of the handle's state (the
 * restart fields, initial mass, grid, physics scalars and boundary specs) at `path`, written to path.tmp and
 * renamed.  `step` is the step index stored for the resumed run.  Mode is written as "coupled",
 * "single_phase" or "advection_only". */
dn_status dn_write_restart(dn_handle *h, int step, const char *path);
/* Solver::load_restart_snapshot (io.cpp:345-437): reads a v1 or v2 snapshot (the reference's or
 * dn_write_restart's), checks it against the handle's config with the reference's rules and messages
 * ("restart snapshot incompatible with config: ..." -> DN_ERR_CONFIG), uploads the fields and rebuilds the
 * derived ones as the reference does.  *step (may be NULL) receives the stored step. */
dn_status dn_load_restart(dn_handle *h, const char *path, int *step);

/* ---- diagnostics ------------------------------------------------------------------------------------ */
/* Solver::compute_diagnostics (diagnostics.cpp:114-167) on the device.  Returns DN_ERR_NONFINITE, with
 * `out` filled, when mass drift, divergence, max velocity or max |mu| is not finite (solver.cpp:355-364). */
dn_status dn_diagnostics(dn_handle *h, dn_diag *out);
/* The diagnostics dn_step computed at the end of the last step (advance_one_timestep ends with
 * compute_diagnostics, solver.cpp:276; dn_step returns DN_ERR_NONFINITE where the reference's run loop
 * aborts). */
dn_status dn_last_diagnostics(dn_handle *h, dn_diag *out);
/* Solver::compute_mass (diagnostics.cpp:24-32), FP64 on the device. */
dn_status dn_compute_mass(dn_handle *h, int field, double *mass);

/* ---- timing / introspection ---------------------------------------------------------------------------- */
/* Block until the handle's stream is idle. */
dn_status dn_synchronize(dn_handle *h);
/* The handle's CUDA stream (cudaStream_t) for event timing by the caller. */
void *dn_stream(dn_handle *h);
/* Device-side times (CUDA events) of the last dn_step, milliseconds: [0] CH phase, [1] momentum phase,
 * [2] pressure phase, [3] correction phase, [4] pressure PCG kernel, [5] CH PCG kernel(s), [6] momentum
 * BiCGSTAB kernel, [7] pressure PCG iterations, then the pressure PCG kernel's own split (device clock):
 * [8] SpMV + dot phases, [9] update phases, [10] preconditioner sweeps.  `out` holds 11 doubles. */
dn_status dn_last_phase_times(dn_handle *h, double *out);
/* Device-clock profiling counters of the last pressure solve's wavefront (ns), 4 per sweep warp k:
 * [4k] forward sweep, [4k+1] waits for the neighbouring warp, [4k+2] waits for staged inputs,
 * [4k+3] backward sweep.  `count` <= 64. */
dn_status dn_profile_counters(dn_handle *h, double *out, int count);
/* Number of this library's kernels launched since the handle was created. */
long long dn_kernel_launches(const dn_handle *h);

#ifdef __cplusplus
}
#endif
#endif
