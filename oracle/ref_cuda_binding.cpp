// The reference-side binding of libdn_cuda, as a maintainer adds it to the reference:
// Solver::dn() creates one dn_handle lazily from the solver's own Config.  Compiled only into
// oracle/_ref/libdnref_cuda.so, together with the copy of the reference's coupled-solver sources that
// oracle/patch_reference.py patches (the solver.hpp members, the `cuda_` branches of the pressure and CH
// dispatchers, the split predicate) -- test infrastructure that checks the binding builds and runs.
#include <stdexcept>
#include <string>

#include "core/coupled/solver.hpp"
#include "dn_cuda.h"

namespace ding {
namespace {

// pressure_scheme strings (pressure.cpp:1031-1089, with an optional `cuda_` prefix) -> dn_pressure_scheme
int scheme_of(std::string s) {
  if (s.rfind("cuda_", 0) == 0) s = s.substr(5);
  if (s == "icpcg") return DN_P_ICPCG;
  if (s == "ildlt_pcg") return DN_P_ILDLT_PCG;
  if (s == "split_icpcg" || s == "liu_split_icpcg" || s == "paper_split_icpcg") return DN_P_SPLIT_ICPCG;
  if (s == "split_ildlt_pcg" || s == "liu_split_ildlt_pcg" || s == "paper_split_ildlt_pcg")
    return DN_P_SPLIT_ILDLT_PCG;
  if (s == "split_dcdm_icpcg" || s == "liu_split_dcdm_icpcg" || s == "paper_split_dcdm_icpcg")
    return DN_P_SPLIT_DCDM_ICPCG;
  if (s == "jacobi") return DN_P_JACOBI;
  throw std::runtime_error("unsupported pressure scheme: " + s);
}

dn_bc bc_of(const BoundaryConditionSpec &b) {
  dn_bc o;
  o.type = b.type == BoundaryConditionType::dirichlet ? DN_BC_DIRICHLET
           : b.type == BoundaryConditionType::neumann ? DN_BC_NEUMANN
                                                      : DN_BC_UNSET;
  o.value = b.value;
  return o;
}

}  // namespace

dn_handle *Solver::dn() const {
  if (dn_) return dn_;
  dn_config c;
  dn_config_default(&c);
  c.nx = cfg_.nx;
  c.ny = cfg_.ny;
  c.ghost = cfg_.ghost;
  c.mode = cfg_.mode == "single_phase" ? DN_MODE_SINGLE_PHASE
           : cfg_.mode == "advection_only" ? DN_MODE_ADVECTION_ONLY
                                           : DN_MODE_COUPLED;
  c.freeze_ch = cfg_.freeze_ch ? 1 : 0;
  c.pressure_scheme = scheme_of(cfg_.pressure_scheme);
  c.phase_initializer = cfg_.phase_initializer == "zalesak_disk" ? 1 : 0;
  c.velocity_profile = cfg_.velocity_profile == "solid_body_rotation" ? 1 : 0;
  c.invert_phase = cfg_.invert_phase ? 1 : 0;
  c.periodic_x = cfg_.periodic_x ? 1 : 0;
  c.periodic_y = cfg_.periodic_y ? 1 : 0;
  c.ch_inner_iterations = cfg_.ch_inner_iterations;
  c.momentum_iterations = cfg_.momentum_iterations;
  c.poisson_iterations = cfg_.poisson_iterations;
  c.surface_tension_smoothing_passes = cfg_.surface_tension_smoothing_passes;
  c.dt = cfg_.dt;
  c.lx = cfg_.lx;
  c.ly = cfg_.ly;
  c.re = cfg_.re;
  c.ca = cfg_.ca;
  c.pe = cfg_.pe;
  c.cn = cfg_.cn;
  c.density_ratio = cfg_.density_ratio;
  c.viscosity_ratio = cfg_.viscosity_ratio;
  c.surface_tension_multiplier = cfg_.surface_tension_multiplier;
  c.surface_tension_smoothing_weight = cfg_.surface_tension_smoothing_weight;
  c.ch_tolerance = cfg_.ch_tolerance;
  c.pressure_tolerance = cfg_.pressure_tolerance;
  c.momentum_tolerance = cfg_.momentum_tolerance;
  c.body_force_x = cfg_.body_force_x;
  c.body_force_y = cfg_.body_force_y;
  c.top_wall_velocity_x = cfg_.top_wall_velocity_x;
  c.bottom_wall_velocity_x = cfg_.bottom_wall_velocity_x;
  const BoundaryConditionSpec *p[4] = {&cfg_.pressure_bc_left, &cfg_.pressure_bc_right, &cfg_.pressure_bc_bottom,
                                       &cfg_.pressure_bc_top};
  const BoundaryConditionSpec *u[4] = {&cfg_.u_bc_left, &cfg_.u_bc_right, &cfg_.u_bc_bottom, &cfg_.u_bc_top};
  const BoundaryConditionSpec *v[4] = {&cfg_.v_bc_left, &cfg_.v_bc_right, &cfg_.v_bc_bottom, &cfg_.v_bc_top};
  for (int s = 0; s < 4; ++s) {
    c.p_bc[s] = bc_of(*p[s]);
    c.u_bc[s] = bc_of(*u[s]);
    c.v_bc[s] = bc_of(*v[s]);
  }
  c.dcdm_direction_mode = cfg_.dcdm_direction_mode == "identity" ? 1 : 0;
  c.dcdm_history_size = cfg_.dcdm_history_size;
  c.dcdm_max_stored_directions = cfg_.dcdm_max_stored_directions;
  c.dcdm_restart_interval = cfg_.dcdm_restart_interval;
  if (dn_create(&c, -1, &dn_) != DN_OK) {
    const std::string msg = dn_ ? dn_last_error(dn_) : "dn_create failed";
    throw std::runtime_error(msg);
  }
  return dn_;
}

}  // namespace ding
