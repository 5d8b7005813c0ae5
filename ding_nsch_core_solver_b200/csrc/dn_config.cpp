// dn_config.cpp -- case-file parsing for libdn_cuda: restates ding::load_config (src/core/base/config.cpp:49-208)
// and the Config defaults (src/core/base/config.hpp:35-136), filling the flat dn_config of the C-ABI.
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>

#include "dn_cuda.h"

namespace {

std::string trim(const std::string &text) {
  const auto first = text.find_first_not_of(" \t\r\n");
  if (first == std::string::npos) return "";
  const auto last = text.find_last_not_of(" \t\r\n");
  return text.substr(first, last - first + 1);
}

std::string lower(std::string s) {
  std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::tolower(c); });
  return s;
}

// parse_bool, config.cpp:22-28
bool parse_bool(const std::string &v) {
  const std::string l = lower(v);
  return l == "1" || l == "true" || l == "yes" || l == "on";
}

// parse_boundary_condition_type, config.cpp:30-45
int parse_bc_type(const std::string &v) {
  const std::string l = lower(v);
  if (l.empty() || l == "unset" || l == "default") return DN_BC_UNSET;
  if (l == "dirichlet") return DN_BC_DIRICHLET;
  if (l == "neumann") return DN_BC_NEUMANN;
  throw std::runtime_error("unsupported boundary condition type: " + v);
}

int parse_pressure_scheme(const std::string &v) {
  // pressure.cpp:1031-1071 spellings, plus the cuda_* values of this backend
  static const std::map<std::string, int> m = {
      {"jacobi", DN_P_JACOBI},
      {"icpcg", DN_P_ICPCG},
      {"cuda_icpcg", DN_P_ICPCG},
      {"ildlt_pcg", DN_P_ILDLT_PCG},
      {"cuda_ildlt_pcg", DN_P_ILDLT_PCG},
      {"split_icpcg", DN_P_SPLIT_ICPCG},
      {"liu_split_icpcg", DN_P_SPLIT_ICPCG},
      {"paper_split_icpcg", DN_P_SPLIT_ICPCG},
      {"cuda_split_icpcg", DN_P_SPLIT_ICPCG},
      {"split_ildlt_pcg", DN_P_SPLIT_ILDLT_PCG},
      {"liu_split_ildlt_pcg", DN_P_SPLIT_ILDLT_PCG},
      {"paper_split_ildlt_pcg", DN_P_SPLIT_ILDLT_PCG},
      {"cuda_split_ildlt_pcg", DN_P_SPLIT_ILDLT_PCG},
      {"split_dcdm_icpcg", DN_P_SPLIT_DCDM_ICPCG},
      {"liu_split_dcdm_icpcg", DN_P_SPLIT_DCDM_ICPCG},
      {"paper_split_dcdm_icpcg", DN_P_SPLIT_DCDM_ICPCG},
      {"cuda_split_dcdm_icpcg", DN_P_SPLIT_DCDM_ICPCG},
  };
  auto it = m.find(v);
  if (it == m.end()) throw std::runtime_error("unsupported pressure scheme: " + v);
  return it->second;
}

}  // namespace

extern "C" void dn_config_default(dn_config *c) {
  std::memset(c, 0, sizeof(*c));
  c->nx = 64;
  c->ny = 64;
  c->ghost = 3;
  c->mode = DN_MODE_COUPLED;
  c->pressure_scheme = DN_P_JACOBI;
  c->ch_inner_iterations = 30;
  c->momentum_iterations = 50;
  c->poisson_iterations = 400;
  c->dt = 1.0e-4;
  c->lx = 1.0;
  c->ly = 1.0;
  c->re = 100.0;
  c->ca = 1.0;
  c->pe = 100.0;
  c->cn = 0.02;
  c->density_ratio = 0.1;
  c->viscosity_ratio = 0.1;
  c->surface_tension_multiplier = 1.0;
  c->ch_tolerance = 1.0e-8;
  c->pressure_tolerance = 1.0e-8;
  c->momentum_tolerance = 1.0e-8;
  c->interface_center_x = 0.5;
  c->interface_center_y = 0.5;
  c->interface_radius = 0.18;
  c->interface_wavenumber = 1.0;
  c->zalesak_slot_width = 0.05;
  c->zalesak_slot_depth = 0.25;
  c->rotation_center_x = 0.5;
  c->rotation_center_y = 0.5;
  c->periodic_x = 1;
  c->periodic_y = 1;
  c->precision = DN_PRECISION_FP64;
  c->mixed_inner_tolerance = 1.0e-5;
  c->device_share = 1;
  c->dcdm_direction_mode = 0;  // icc_preconditioned
  c->dcdm_history_size = 2;
  c->dcdm_max_stored_directions = 8;
  c->dcdm_restart_interval = 0;
  c->pcg_rows_per_cta = 0;     // 512
  c->sweep_warps_per_cta = 0;  // as many as the shared memory holds, up to 4
  c->device_wait_limit = 0;    // kSpinLimit polls
  c->mg_cluster_cells = 0;     // off
  c->mixed_preconditioner = DN_MIXED_PREC_MULTIGRID;
  c->analysis_enabled = 0;     // config.hpp:53-133
  c->analysis_mode = DN_ANALYSIS_OFF;
  c->analysis_trigger_step = 1;
  c->analysis_interface_band_multiplier = 2.0;
  std::snprintf(c->name, sizeof c->name, "%s", "unnamed");
  std::snprintf(c->output_dir, sizeof c->output_dir, "%s", "output");
  c->analysis_case_group[0] = '\0';
  std::snprintf(c->analysis_initial_guess, sizeof c->analysis_initial_guess, "%s", "zero");
  std::snprintf(c->analysis_nullspace_treatment, sizeof c->analysis_nullspace_treatment, "%s", "zero_mean_projection");
  std::snprintf(c->analysis_spectrum_iterations, sizeof c->analysis_spectrum_iterations, "%s", "0,1,2,5,10,20,final");
}

extern "C" dn_status dn_config_parse(const char *text, dn_config *cfg, char *err, size_t err_len) {
  auto set_err = [&](const std::string &m) {
    if (err && err_len) std::snprintf(err, err_len, "%s", m.c_str());
  };
  if (!text || !cfg) {
    set_err("null argument");
    return DN_ERR_INVALID_ARGUMENT;
  }
  try {
    std::map<std::string, std::string> kv;
    std::istringstream in(text);
    std::string line;
    while (std::getline(in, line)) {
      const auto hash = line.find('#');
      if (hash != std::string::npos) line = line.substr(0, hash);
      line = trim(line);
      if (line.empty()) continue;
      const auto eq = line.find('=');
      if (eq == std::string::npos) continue;
      kv[trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
    }
    if (kv.count("stabilization_a1") || kv.count("stabilization_a2"))
      throw std::runtime_error("stabilization_a1/stabilization_a2 are derived from cn and must not be set in case files");
    dn_config_default(cfg);
    auto geti = [&](const char *k, int &v) {
      if (kv.count(k)) v = std::stoi(kv[k]);
    };
    auto getd = [&](const char *k, double &v) {
      if (kv.count(k)) v = std::stod(kv[k]);
    };
    auto getb = [&](const char *k, int &v) {
      if (kv.count(k)) v = parse_bool(kv[k]) ? 1 : 0;
    };
    auto getbc = [&](const char *tk, const char *vk, dn_bc &b) {
      if (kv.count(tk)) b.type = parse_bc_type(kv[tk]);
      if (kv.count(vk)) b.value = std::stod(kv[vk]);
    };
    if (kv.count("mode")) {
      const std::string m = kv["mode"];
      if (m == "single_phase")
        cfg->mode = DN_MODE_SINGLE_PHASE;
      else if (m == "advection_only")
        cfg->mode = DN_MODE_ADVECTION_ONLY;
      else
        cfg->mode = DN_MODE_COUPLED;
    }
    if (kv.count("pressure_scheme")) cfg->pressure_scheme = parse_pressure_scheme(kv["pressure_scheme"]);
    if (kv.count("ch_solver")) {
      const std::string v = kv["ch_solver"];
      if (v != "sparse_pcg" && v != "cuda_sparse_pcg")
        throw std::runtime_error("unsupported ch_solver for the CUDA backend: " + v);
    }
    if (kv.count("phase_initializer")) cfg->phase_initializer = kv["phase_initializer"] == "zalesak_disk" ? 1 : 0;
    if (kv.count("velocity_profile")) cfg->velocity_profile = kv["velocity_profile"] == "solid_body_rotation" ? 1 : 0;
    if (kv.count("precision")) {
      const std::string v = lower(kv["precision"]);
      if (v == "fp64" || v == "plain")
        cfg->precision = DN_PRECISION_FP64;
      else if (v == "mixed")
        cfg->precision = DN_PRECISION_MIXED;
      else
        throw std::runtime_error("unsupported precision: " + kv["precision"]);
    }
    if (kv.count("mixed_preconditioner")) {
      const std::string v = lower(kv["mixed_preconditioner"]);
      if (v == "multigrid")
        cfg->mixed_preconditioner = DN_MIXED_PREC_MULTIGRID;
      else if (v == "ic" || v == "icc" || v == "ildlt")
        cfg->mixed_preconditioner = DN_MIXED_PREC_IC;
      else
        throw std::runtime_error("unsupported mixed_preconditioner: " + kv["mixed_preconditioner"]);
    }
    geti("nx", cfg->nx);
    geti("ny", cfg->ny);
    geti("ghost", cfg->ghost);
    geti("ch_inner_iterations", cfg->ch_inner_iterations);
    geti("momentum_iterations", cfg->momentum_iterations);
    geti("poisson_iterations", cfg->poisson_iterations);
    geti("surface_tension_smoothing_passes", cfg->surface_tension_smoothing_passes);
    getd("dt", cfg->dt);
    getd("lx", cfg->lx);
    getd("ly", cfg->ly);
    getd("re", cfg->re);
    getd("ca", cfg->ca);
    getd("pe", cfg->pe);
    getd("cn", cfg->cn);
    getd("density_ratio", cfg->density_ratio);
    getd("viscosity_ratio", cfg->viscosity_ratio);
    getd("surface_tension_multiplier", cfg->surface_tension_multiplier);
    getd("surface_tension_smoothing_weight", cfg->surface_tension_smoothing_weight);
    getd("ch_tolerance", cfg->ch_tolerance);
    getd("pressure_tolerance", cfg->pressure_tolerance);
    getd("momentum_tolerance", cfg->momentum_tolerance);
    getd("body_force_x", cfg->body_force_x);
    getd("body_force_y", cfg->body_force_y);
    getd("interface_center_x", cfg->interface_center_x);
    getd("interface_center_y", cfg->interface_center_y);
    getd("interface_radius", cfg->interface_radius);
    getd("interface_amplitude", cfg->interface_amplitude);
    getd("interface_wavenumber", cfg->interface_wavenumber);
    getd("zalesak_slot_width", cfg->zalesak_slot_width);
    getd("zalesak_slot_depth", cfg->zalesak_slot_depth);
    getd("advect_u", cfg->advect_u);
    getd("advect_v", cfg->advect_v);
    getd("rotation_center_x", cfg->rotation_center_x);
    getd("rotation_center_y", cfg->rotation_center_y);
    getd("angular_velocity", cfg->angular_velocity);
    getd("top_wall_velocity_x", cfg->top_wall_velocity_x);
    getd("bottom_wall_velocity_x", cfg->bottom_wall_velocity_x);
    getd("mixed_inner_tolerance", cfg->mixed_inner_tolerance);
    geti("device_share", cfg->device_share);
    geti("dcdm_history_size", cfg->dcdm_history_size);
    geti("dcdm_max_stored_directions", cfg->dcdm_max_stored_directions);
    geti("dcdm_restart_interval", cfg->dcdm_restart_interval);
    auto gets = [&](const char *k, char *dst, size_t cap) {
      if (!kv.count(k)) return;
      if (kv[k].size() >= cap) throw std::runtime_error(std::string(k) + " is too long");
      std::snprintf(dst, cap, "%s", kv[k].c_str());
    };
    gets("name", cfg->name, sizeof cfg->name);
    gets("output_dir", cfg->output_dir, sizeof cfg->output_dir);
    gets("analysis_case_group", cfg->analysis_case_group, sizeof cfg->analysis_case_group);
    gets("analysis_initial_guess", cfg->analysis_initial_guess, sizeof cfg->analysis_initial_guess);
    gets("analysis_nullspace_treatment", cfg->analysis_nullspace_treatment, sizeof cfg->analysis_nullspace_treatment);
    gets("analysis_spectrum_iterations", cfg->analysis_spectrum_iterations, sizeof cfg->analysis_spectrum_iterations);
    getb("analysis_enabled", cfg->analysis_enabled);
    geti("analysis_trigger_step", cfg->analysis_trigger_step);
    getd("analysis_interface_band_multiplier", cfg->analysis_interface_band_multiplier);
    if (kv.count("analysis_mode")) {  // analysis_mode_enabled, pressure_analysis.cpp:126-137
      const std::string m = lower(kv["analysis_mode"]);
      cfg->analysis_mode = m == "both" ? DN_ANALYSIS_BOTH : m == "online" ? DN_ANALYSIS_ONLINE
                           : m == "frozen" ? DN_ANALYSIS_FROZEN : DN_ANALYSIS_OFF;
    }
    geti("pcg_rows_per_cta", cfg->pcg_rows_per_cta);
    geti("sweep_warps_per_cta", cfg->sweep_warps_per_cta);
    geti("device_wait_limit", cfg->device_wait_limit);
    geti("mg_cluster_cells", cfg->mg_cluster_cells);
    if (cfg->device_wait_limit < 0) throw std::runtime_error("device_wait_limit must be non-negative (0: the default)");
    if (kv.count("dcdm_direction_mode")) {  // pressure.cpp:383-395
      const std::string m = lower(kv["dcdm_direction_mode"]);
      if (m == "identity")
        cfg->dcdm_direction_mode = 1;
      else if (m == "icc" || m == "icc_preconditioned" || m == "pcg_preconditioned")
        cfg->dcdm_direction_mode = 0;
      else if (m == "neural" || m == "hydea_neural" || m == "ml")
        throw std::runtime_error("dcdm neural directions need the HyDEA worker, which the CUDA backend does not run");
      else
        throw std::runtime_error("unsupported dcdm_direction_mode: " + kv["dcdm_direction_mode"]);
    }
    if (cfg->device_share < 1) throw std::runtime_error("device_share must be at least 1");
    if (cfg->pcg_rows_per_cta < 0 || cfg->sweep_warps_per_cta < 0)
      throw std::runtime_error("pcg_rows_per_cta and sweep_warps_per_cta must be non-negative (0: the default)");
    static const char *sides[4] = {"left", "right", "bottom", "top"};
    for (int s = 0; s < 4; ++s) {
      char tk[64], vk[64];
      std::snprintf(tk, sizeof tk, "pressure_bc_%s_type", sides[s]);
      std::snprintf(vk, sizeof vk, "pressure_bc_%s_value", sides[s]);
      getbc(tk, vk, cfg->p_bc[s]);
      std::snprintf(tk, sizeof tk, "u_bc_%s_type", sides[s]);
      std::snprintf(vk, sizeof vk, "u_bc_%s_value", sides[s]);
      getbc(tk, vk, cfg->u_bc[s]);
      std::snprintf(tk, sizeof tk, "v_bc_%s_type", sides[s]);
      std::snprintf(vk, sizeof vk, "v_bc_%s_value", sides[s]);
      getbc(tk, vk, cfg->v_bc[s]);
    }
    getb("periodic_x", cfg->periodic_x);
    getb("periodic_y", cfg->periodic_y);
    getb("invert_phase", cfg->invert_phase);
    getb("freeze_ch", cfg->freeze_ch);
  } catch (const std::exception &ex) {
    set_err(ex.what());
    return DN_ERR_CONFIG;
  }
  return DN_OK;
}
