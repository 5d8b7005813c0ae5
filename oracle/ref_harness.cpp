// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own coupled-solver sources (built by oracle/Makefile straight from the
// reference tree, output in oracle/_ref/) behind the same flat C API as oracle/dn_oracle.h, so the
// tests can run the reference itself on injected states.  White-box access follows the reference's
// own unit-test harness (src/tests/core_solver_unit_tests.cpp:7-9: `#define private public`).
// The product path never links or calls this code.
#include <chrono>
#include <cstring>
#include <exception>
#include <string>
// The standard headers the reference's headers pull in come first, so that the `private` redefinition below
// reaches only the reference's own classes: standard classes compiled with it would lay out differently
// from the same classes in the reference's translation units.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iomanip>
#include <map>
#include <set>
#include <sstream>
#include <stdexcept>
#include <vector>

#define private public
#include "core/coupled/solver.hpp"
#undef private

#include "dn_oracle.h"

namespace {

struct RefHandle {
  ding::Solver *solver = nullptr;
  std::string err;
};

ding::BoundaryConditionSpec to_spec(const orc_bc &b) {
  ding::BoundaryConditionSpec s;
  s.type = static_cast<ding::BoundaryConditionType>(b.type);
  s.value = b.value;
  return s;
}

ding::Config to_config(const orc_config &c) {
  ding::Config cfg;
  cfg.name = "oracle_ref";
  cfg.nx = c.nx;
  cfg.ny = c.ny;
  cfg.ghost = c.ghost;
  cfg.mode = c.mode == ORC_MODE_SINGLE_PHASE ? "single_phase"
             : c.mode == ORC_MODE_ADVECTION_ONLY ? "advection_only"
                                                 : "coupled";
  cfg.freeze_ch = c.freeze_ch != 0;
  switch (c.pressure_scheme) {
  case ORC_P_ICPCG: cfg.pressure_scheme = "icpcg"; break;
  case ORC_P_ILDLT_PCG: cfg.pressure_scheme = "ildlt_pcg"; break;
  case ORC_P_SPLIT_ICPCG: cfg.pressure_scheme = "split_icpcg"; break;
  case ORC_P_SPLIT_ILDLT_PCG: cfg.pressure_scheme = "split_ildlt_pcg"; break;
  case ORC_P_SPLIT_DCDM_ICPCG: cfg.pressure_scheme = "split_dcdm_icpcg"; break;
  default: cfg.pressure_scheme = "jacobi"; break;
  }
#ifdef DN_REF_CUDA_BACKEND
  // the patched reference: the pressure and CH solves go to libdn_cuda through the reference-side binding
  cfg.pressure_scheme = "cuda_" + cfg.pressure_scheme;
  cfg.ch_solver = "cuda_sparse_pcg";
#endif
  cfg.phase_initializer = c.phase_initializer == 1 ? "zalesak_disk" : "default";
  cfg.velocity_profile = c.velocity_profile == 1 ? "solid_body_rotation" : "default";
  cfg.invert_phase = c.invert_phase != 0;
  cfg.periodic_x = c.periodic_x != 0;
  cfg.periodic_y = c.periodic_y != 0;
  cfg.ch_inner_iterations = c.ch_inner_iterations;
  cfg.momentum_iterations = c.momentum_iterations;
  cfg.poisson_iterations = c.poisson_iterations;
  cfg.surface_tension_smoothing_passes = c.surface_tension_smoothing_passes;
  cfg.dt = c.dt;
  cfg.lx = c.lx;
  cfg.ly = c.ly;
  cfg.re = c.re;
  cfg.ca = c.ca;
  cfg.pe = c.pe;
  cfg.cn = c.cn;
  cfg.density_ratio = c.density_ratio;
  cfg.viscosity_ratio = c.viscosity_ratio;
  cfg.surface_tension_multiplier = c.surface_tension_multiplier;
  cfg.surface_tension_smoothing_weight = c.surface_tension_smoothing_weight;
  cfg.ch_tolerance = c.ch_tolerance;
  cfg.pressure_tolerance = c.pressure_tolerance;
  cfg.momentum_tolerance = c.momentum_tolerance;
  cfg.body_force_x = c.body_force_x;
  cfg.body_force_y = c.body_force_y;
  cfg.interface_center_x = c.interface_center_x;
  cfg.interface_center_y = c.interface_center_y;
  cfg.interface_radius = c.interface_radius;
  cfg.interface_amplitude = c.interface_amplitude;
  cfg.interface_wavenumber = c.interface_wavenumber;
  cfg.zalesak_slot_width = c.zalesak_slot_width;
  cfg.zalesak_slot_depth = c.zalesak_slot_depth;
  cfg.advect_u = c.advect_u;
  cfg.advect_v = c.advect_v;
  cfg.rotation_center_x = c.rotation_center_x;
  cfg.rotation_center_y = c.rotation_center_y;
  cfg.angular_velocity = c.angular_velocity;
  cfg.top_wall_velocity_x = c.top_wall_velocity_x;
  cfg.bottom_wall_velocity_x = c.bottom_wall_velocity_x;
  cfg.pressure_bc_left = to_spec(c.p_bc[ORC_LEFT]);
  cfg.pressure_bc_right = to_spec(c.p_bc[ORC_RIGHT]);
  cfg.pressure_bc_bottom = to_spec(c.p_bc[ORC_BOTTOM]);
  cfg.pressure_bc_top = to_spec(c.p_bc[ORC_TOP]);
  cfg.u_bc_left = to_spec(c.u_bc[ORC_LEFT]);
  cfg.u_bc_right = to_spec(c.u_bc[ORC_RIGHT]);
  cfg.u_bc_bottom = to_spec(c.u_bc[ORC_BOTTOM]);
  cfg.u_bc_top = to_spec(c.u_bc[ORC_TOP]);
  cfg.v_bc_left = to_spec(c.v_bc[ORC_LEFT]);
  cfg.v_bc_right = to_spec(c.v_bc[ORC_RIGHT]);
  cfg.v_bc_bottom = to_spec(c.v_bc[ORC_BOTTOM]);
  cfg.v_bc_top = to_spec(c.v_bc[ORC_TOP]);
  cfg.dcdm_direction_mode = c.dcdm_direction_mode == 1 ? "identity" : "icc_preconditioned";
  cfg.dcdm_history_size = c.dcdm_history_size;
  cfg.dcdm_max_stored_directions = c.dcdm_max_stored_directions;
  cfg.dcdm_restart_interval = c.dcdm_restart_interval;
  cfg.output_dir = "oracle/_ref/out";  // the dcdm backend creates its solver directory under the case output
  cfg.verbose = false;
  cfg.print_step_log = false;
  cfg.write_vtk = false;
  cfg.write_restart = false;
  return cfg;
}

ding::Field2D *field_of(ding::Solver &s, int id) {
  switch (id) {
  case ORC_F_C: return &s.c_;
  case ORC_F_C_PREV: return &s.c_previous_step_;
  case ORC_F_C_PREV2: return &s.c_two_steps_back_;
  case ORC_F_MU: return &s.mu_;
  case ORC_F_RHO: return &s.rho_;
  case ORC_F_ETA: return &s.eta_;
  case ORC_F_RHO_PREV: return &s.rho_previous_step_;
  case ORC_F_ETA_PREV: return &s.eta_previous_step_;
  case ORC_F_RHO_MID: return &s.rho_mid_;
  case ORC_F_ETA_MID: return &s.eta_mid_;
  case ORC_F_P: return &s.pressure_;
  case ORC_F_P_PREV: return &s.pressure_previous_step_;
  case ORC_F_P_CORR: return &s.pressure_correction_;
  case ORC_F_U: return &s.u_;
  case ORC_F_V: return &s.v_;
  case ORC_F_U_PREV: return &s.u_previous_step_;
  case ORC_F_V_PREV: return &s.v_previous_step_;
  case ORC_F_U_STAR: return &s.u_star_;
  case ORC_F_V_STAR: return &s.v_star_;
  case ORC_F_SFX_CELL: return &s.surface_fx_cell_;
  case ORC_F_SFY_CELL: return &s.surface_fy_cell_;
  case ORC_F_SFX_U: return &s.surface_fx_u_;
  case ORC_F_SFY_V: return &s.surface_fy_v_;
  case ORC_F_E_PREV: return &s.phase_explicit_operator_prev_;
  case ORC_F_HU_PREV: return &s.momentum_u_rhs_prev_;
  case ORC_F_HV_PREV: return &s.momentum_v_rhs_prev_;
  default: return nullptr;
  }
}

template <typename F>
int guarded(RefHandle *h, F &&fn) {
  try {
    h->err.clear();
    fn();
    return 0;
  } catch (const std::exception &ex) {
    h->err = ex.what();
    return 1;
  }
}

} // namespace

extern "C" {

void *ref_create(const orc_config *cfg) {
  auto *h = new RefHandle();
  h->solver = new ding::Solver(to_config(*cfg));
  return h;
}

void ref_destroy(void *hp) {
  auto *h = static_cast<RefHandle *>(hp);
  delete h->solver;
  delete h;
}

const char *ref_last_error(void *hp) { return static_cast<RefHandle *>(hp)->err.c_str(); }

double *ref_field(void *hp, int id, int *nx, int *ny, int *ghost) {
  auto *h = static_cast<RefHandle *>(hp);
  ding::Field2D *f = field_of(*h->solver, id);
  if (!f) return nullptr;
  if (nx) *nx = f->nx;
  if (ny) *ny = f->ny;
  if (ghost) *ghost = f->ghost;
  return f->data.data();
}

void ref_set_initial_mass(void *hp, double mass) { static_cast<RefHandle *>(hp)->solver->initial_mass_ = mass; }

int ref_initialize(void *hp) {
  auto *h = static_cast<RefHandle *>(hp);
  return guarded(h, [&] { h->solver->initialize(); });
}

int ref_step(void *hp, int step) {
  auto *h = static_cast<RefHandle *>(hp);
  return guarded(h, [&] { h->solver->advance_one_timestep(step); });
}

int ref_begin_step(void *hp, int step) {
  auto *h = static_cast<RefHandle *>(hp);
  ding::Solver &s = *h->solver;
  s.current_step_index_ = step;
  s.c_two_steps_back_ = s.c_previous_step_;
  s.c_previous_step_ = s.c_;
  s.rho_previous_step_ = s.rho_;
  s.eta_previous_step_ = s.eta_;
  s.u_previous_step_ = s.u_;
  s.v_previous_step_ = s.v_;
  return 0;
}

int ref_phase(void *hp, int step) {
  auto *h = static_cast<RefHandle *>(hp);
  return guarded(h, [&] {
    auto rep = h->solver->advance_phase_state(step);
    h->solver->last_coupling_iterations_ = rep.outer_iterations;
  });
}

int ref_momentum(void *hp, int step) {
  auto *h = static_cast<RefHandle *>(hp);
  return guarded(h, [&] {
    ding::Solver &s = *h->solver;
    ding::Field2D ua(s.u_.nx, s.u_.ny, s.u_.ghost, 0.0);
    ding::Field2D va(s.v_.nx, s.v_.ny, s.v_.ghost, 0.0);
    s.compute_momentum_fluxes(ua, va);
    s.solve_momentum_predictor(ua, va, step);
  });
}

int ref_pressure(void *hp) {
  auto *h = static_cast<RefHandle *>(hp);
  return guarded(h, [&] { h->solver->solve_pressure_correction(); });
}

int ref_correct(void *hp) {
  auto *h = static_cast<RefHandle *>(hp);
  return guarded(h, [&] { h->solver->apply_pressure_velocity_correction(); });
}

int ref_finish_step(void *hp) {
  auto *h = static_cast<RefHandle *>(hp);
  return guarded(h, [&] { h->solver->refresh_chemical_potential_for_current_phase(); });
}

int ref_refresh_derived(void *hp) {
  auto *h = static_cast<RefHandle *>(hp);
  return guarded(h, [&] {
    ding::Solver &s = *h->solver;
    s.apply_scalar_bc(s.c_);
    s.apply_scalar_bc(s.c_previous_step_);
    s.apply_scalar_bc(s.c_two_steps_back_);
    s.apply_pressure_bc(s.pressure_);
    s.apply_pressure_bc(s.pressure_previous_step_);
    s.apply_u_velocity_bc(s.u_);
    s.apply_v_bc(s.v_);
    s.apply_u_velocity_bc(s.u_previous_step_);
    s.apply_v_bc(s.v_previous_step_);
    s.update_materials();
    s.update_materials_from_phase(s.c_previous_step_, s.rho_previous_step_, s.eta_previous_step_);
    s.update_midpoint_materials();
    s.refresh_chemical_potential_for_current_phase();
  });
}

int ref_ch_linear_solve(void *hp, const double *rhs_field, double alpha0, double *c_state, double *iterate_residual,
                        double *equation_residual) {
  auto *h = static_cast<RefHandle *>(hp);
  return guarded(h, [&] {
    ding::Solver &s = *h->solver;
    ding::Field2D rhs(s.cfg_.nx, s.cfg_.ny, s.cfg_.ghost, 0.0);
    ding::Field2D cs(s.cfg_.nx, s.cfg_.ny, s.cfg_.ghost, 0.0);
    std::memcpy(rhs.data.data(), rhs_field, rhs.data.size() * sizeof(double));
    std::memcpy(cs.data.data(), c_state, cs.data.size() * sizeof(double));
    s.solve_phase_linear_system_eq25(rhs, alpha0, 0.0, cs, *iterate_residual, *equation_residual);
    std::memcpy(c_state, cs.data.data(), cs.data.size() * sizeof(double));
  });
}

// Solver::run_pressure_analysis_from_snapshot (pressure_analysis.cpp:156-328) on the current state, step index
// `step`, with the analysis settings that the config struct does not carry set here.
int ref_pressure_analysis(void *hp, int step, const char *source_mode, const char *output_dir, const char *name,
                          const char *case_group, const char *spectrum_iterations, double band) {
  auto *h = static_cast<RefHandle *>(hp);
  return guarded(h, [&] {
    ding::Solver &s = *h->solver;
    s.cfg_.output_dir = output_dir;
    s.cfg_.name = name;
    s.cfg_.analysis_case_group = case_group;
    s.cfg_.analysis_spectrum_iterations = spectrum_iterations;
    s.cfg_.analysis_interface_band_multiplier = band;
    s.current_step_index_ = step;
    s.run_pressure_analysis_from_snapshot(s.make_pressure_analysis_snapshot(source_mode));
  });
}

void ref_get_report(void *hp, orc_report *r) {
  ding::Solver &s = *static_cast<RefHandle *>(hp)->solver;
  std::memset(r, 0, sizeof(*r));
  r->ch_iterations = s.last_ch_iterations_;
  r->momentum_iterations = s.last_momentum_iterations_;
  r->pressure_iterations = s.last_pressure_iterations_;
  r->coupling_iterations = s.last_coupling_iterations_;
  const std::string &n = s.last_ch_solver_name_;
  r->ch_preconditioner = n == "SparsePCG[ILDLT]" ? 1 : n == "SparsePCG[DiagonalFallback]" ? 2
                         : n == "SparsePCG[Diagonal]"                                      ? 0
                                                                                           : -1;
  r->ch_residual = s.last_diag_.ch_inner_residual;
  r->ch_equation_residual = s.last_ch_equation_residual_;
  r->momentum_residual = s.last_diag_.momentum_residual;
  r->pressure_residual = s.last_diag_.pressure_correction_residual;
  r->boundary_speed_pre = s.last_boundary_speed_pre_correction_;
  r->boundary_speed_post = s.last_boundary_speed_post_correction_;
}

void ref_diagnostics(void *hp, orc_diag *d) {
  ding::Solver &s = *static_cast<RefHandle *>(hp)->solver;
  const ding::Diagnostics g = s.compute_diagnostics();
  d->mass = g.mass;
  d->mass_drift = g.mass_drift;
  d->divergence_l2 = g.divergence_l2;
  d->max_divergence = g.max_divergence_after_correction;
  d->max_abs_mu = g.max_abs_mu;
  d->max_velocity = g.max_velocity;
  d->kinetic_energy = g.kinetic_energy;
  d->total_free_energy = g.total_free_energy;
  d->rho_min = g.rho_min;
  d->rho_max = g.rho_max;
  d->eta_min = g.eta_min;
  d->eta_max = g.eta_max;
  d->dt_limit_advective = g.dt_limit_advective;
  d->dt_limit_capillary = g.dt_limit_capillary;
  d->dt_limit_ch_explicit = g.dt_limit_ch_explicit;
  d->dt_limit_active = g.dt_limit_active;
  d->dt_limit_ratio = g.dt_limit_ratio;
}

double ref_compute_mass(void *hp, int field_id) {
  ding::Solver &s = *static_cast<RefHandle *>(hp)->solver;
  return s.compute_mass(*field_of(s, field_id));
}

// Times `count` calls of advance_one_timestep (steps first_step .. first_step+count-1) with
// std::chrono::steady_clock; returns seconds, or a negative value on failure.
double ref_time_steps(void *hp, int first_step, int count) {
  auto *h = static_cast<RefHandle *>(hp);
  double seconds = -1.0;
  const int rc = guarded(h, [&] {
    const auto t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < count; ++k) h->solver->advance_one_timestep(first_step + k);
    const auto t1 = std::chrono::steady_clock::now();
    seconds = std::chrono::duration<double>(t1 - t0).count();
  });
  return rc == 0 ? seconds : -1.0;
}

} // extern "C"
