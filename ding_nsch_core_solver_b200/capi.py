"""ctypes binding of libdn_cuda.so (include/dn_cuda.h).

This module is the Python face of the C-ABI.  ``Solver`` mirrors the reference's ``ding::Solver`` for the
time-step path: ``initialize`` (solver.cpp:69-113), ``advance_one_timestep`` (solver.cpp:224-283) and its
phases, field access in Field2D layout, ``compute_diagnostics`` (diagnostics.cpp:114-167), and the two
backend entry points that replace ``solve_phase_linear_system_eq25`` (phase_field.cpp:437-503) and
``solve_pressure_correction_*`` (pressure.cpp:302-365).  Every call goes to the GPU; if the library or
the device is missing the calls raise, there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdn_cuda.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "dn_cuda.h")

FIELDS = ("c", "c_prev", "c_prev2", "mu", "rho", "eta", "rho_prev", "eta_prev", "rho_mid", "eta_mid", "p",
          "p_prev", "p_corr", "u", "v", "u_prev", "v_prev", "u_star", "v_star", "sfx_cell", "sfy_cell", "sfx_u",
          "sfy_v", "e_prev", "hu_prev", "hv_prev")
FIELD_ID = {n: k for k, n in enumerate(FIELDS)}
U_FIELDS = {"u", "u_prev", "u_star", "sfx_u", "hu_prev"}
V_FIELDS = {"v", "v_prev", "v_star", "sfy_v", "hv_prev"}

STATUS = {0: "ok", 1: "invalid argument", 2: "invalid configuration", 3: "CUDA error",
          4: "ICC preconditioner construction failed", 5: "ILDLT preconditioner construction failed",
          6: "pcg breakdown", 7: "bicgstab breakdown", 8: "device wait timed out",
          9: "non-finite diagnostic detected", 10: "unsupported configuration"}


class BC(C.Structure):
    _fields_ = [("type", C.c_int), ("value", C.c_double)]


class Config(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "nx", "ny", "ghost", "mode", "freeze_ch", "pressure_scheme", "phase_initializer", "velocity_profile",
        "invert_phase", "periodic_x", "periodic_y", "ch_inner_iterations", "momentum_iterations",
        "poisson_iterations", "surface_tension_smoothing_passes")] + [(n, C.c_double) for n in (
        "dt", "lx", "ly", "re", "ca", "pe", "cn", "density_ratio", "viscosity_ratio",
        "surface_tension_multiplier", "surface_tension_smoothing_weight", "ch_tolerance", "pressure_tolerance",
        "momentum_tolerance", "body_force_x", "body_force_y", "interface_center_x", "interface_center_y",
        "interface_radius", "interface_amplitude", "interface_wavenumber", "zalesak_slot_width",
        "zalesak_slot_depth", "advect_u", "advect_v", "rotation_center_x", "rotation_center_y",
        "angular_velocity", "top_wall_velocity_x", "bottom_wall_velocity_x")] + [
        ("p_bc", BC * 4), ("u_bc", BC * 4), ("v_bc", BC * 4), ("precision", C.c_int),
        ("mixed_inner_tolerance", C.c_double), ("device_share", C.c_int), ("dcdm_direction_mode", C.c_int),
        ("dcdm_history_size", C.c_int), ("dcdm_max_stored_directions", C.c_int), ("dcdm_restart_interval", C.c_int),
        ("pcg_rows_per_cta", C.c_int), ("sweep_warps_per_cta", C.c_int), ("device_wait_limit", C.c_int), ("mixed_preconditioner", C.c_int),
        ("mg_cluster_cells", C.c_int),
        ("analysis_enabled", C.c_int), ("analysis_mode", C.c_int), ("analysis_trigger_step", C.c_int),
        ("analysis_interface_band_multiplier", C.c_double), ("name", C.c_char * 128), ("output_dir", C.c_char * 512),
        ("analysis_case_group", C.c_char * 128), ("analysis_initial_guess", C.c_char * 64),
        ("analysis_nullspace_treatment", C.c_char * 64), ("analysis_spectrum_iterations", C.c_char * 256)]


class Report(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "ch_iterations", "momentum_iterations", "pressure_iterations", "coupling_iterations",
        "ch_preconditioner")] + [(n, C.c_double) for n in (
        "ch_residual", "ch_equation_residual", "momentum_residual", "pressure_residual",
        "boundary_speed_pre", "boundary_speed_post")] + [("refinement_cycles", C.c_int), ("mixed_inner_multigrid", C.c_int)]


class Diag(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "mass", "mass_drift", "divergence_l2", "max_divergence", "max_abs_mu", "max_velocity", "kinetic_energy",
        "total_free_energy", "rho_min", "rho_max", "eta_min", "eta_max", "dt_limit_advective",
        "dt_limit_capillary", "dt_limit_ch_explicit", "dt_limit_active", "dt_limit_ratio")]


class DnError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


_LIB = None


def header_symbols() -> list:
    """Every entry point declared in include/dn_cuda.h."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(dn_[a-z_0-9]+)\s*\(", text)))


def load():
    """Load libdn_cuda.so (raises when it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is missing: build it with `python -m ding_nsch_core_solver_b200.build`")
    lib = C.CDLL(LIB_PATH)
    H, I, D, DP, VP = C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_double), C.c_void_p
    sig = {
        "dn_config_default": (None, [C.POINTER(Config)]),
        "dn_config_parse": (I, [C.c_char_p, C.POINTER(Config), C.c_char_p, C.c_size_t]),
        "dn_create": (I, [C.POINTER(Config), I, C.POINTER(H)]),
        "dn_destroy": (I, [H]),
        "dn_status_string": (C.c_char_p, [I]),
        "dn_last_error": (C.c_char_p, [H]),
        "dn_initialize": (I, [H]),
        "dn_set_field": (I, [H, I, DP, C.c_size_t]),
        "dn_get_field": (I, [H, I, DP, C.c_size_t]),
        "dn_field_device_ptr": (I, [H, I, C.POINTER(DP), C.POINTER(C.c_size_t)]),
        "dn_set_initial_mass": (None, [H, D]),
        "dn_refresh_derived": (I, [H]),
        "dn_step": (I, [H, I, C.POINTER(Report)]),
        "dn_step_batch": (I, [C.POINTER(H), I, C.POINTER(C.c_int), C.POINTER(Report)]),
        "dn_begin_step": (I, [H, I]),
        "dn_phase": (I, [H, I, C.POINTER(Report)]),
        "dn_momentum": (I, [H, I, C.POINTER(Report)]),
        "dn_pressure": (I, [H, C.POINTER(Report)]),
        "dn_correct": (I, [H, C.POINTER(Report)]),
        "dn_ch_linear_solve": (I, [H, DP, D, DP, DP, DP, C.POINTER(C.c_int)]),
        "dn_pressure_solve": (I, [H, I, DP, DP, DP, DP, DP, DP, C.POINTER(C.c_int), DP]),
        "dn_projection": (I, [H, I, VP, VP, VP, VP, VP, VP, VP, VP, C.POINTER(C.c_int), DP]),
        "dn_projection_adjoint": (I, [H, I, VP, VP, VP, VP, VP, VP, VP, VP, C.POINTER(C.c_int), DP]),
        "dn_momentum_map": (I, [H, I] + [VP] * 13 + [C.POINTER(C.c_int), DP]),
        "dn_momentum_adjoint": (I, [H, I] + [VP] * 22 + [C.POINTER(C.c_int), DP]),
        "dn_projection_rho": (I, [H, I] + [VP] * 9 + [C.POINTER(C.c_int), DP]),
        "dn_projection_rho_adjoint": (I, [H, I] + [VP] * 13 + [C.POINTER(C.c_int), DP]),
        "dn_surface_force_map": (I, [H, VP, VP, VP, VP]),
        "dn_surface_force_adjoint": (I, [H, VP, VP, VP, VP, VP, VP]),
        "dn_advection": (I, [H, VP, VP, VP, VP]),
        "dn_advection_adjoint": (I, [H, VP, VP, VP, VP, VP, VP, VP]),
        "dn_set_pressure_monitor": (I, [H, I]),
        "dn_pressure_monitor": (I, [H, DP, I, C.POINTER(C.c_int)]),
        "dn_autotune_pressure": (I, [H, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]),
        "dn_set_step_graph": (I, [H, I]),
        "dn_pressure_analysis": (I, [H, I, C.c_char_p]),
        "dn_history_csv_header": (C.c_size_t, [C.c_char_p, C.c_size_t]),
        "dn_history_csv_row": (I, [H, I, D, C.POINTER(Report), C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
        "dn_write_restart": (I, [H, I, C.c_char_p]),
        "dn_load_restart": (I, [H, C.c_char_p, C.POINTER(C.c_int)]),
        "dn_explicit_operator": (I, [H, VP, VP, VP, VP]),
        "dn_explicit_operator_adjoint": (I, [H, VP, VP, VP, VP, VP, VP, VP]),
        "dn_diagnostics": (I, [H, C.POINTER(Diag)]),
        "dn_last_diagnostics": (I, [H, C.POINTER(Diag)]),
        "dn_compute_mass": (I, [H, I, DP]),
        "dn_synchronize": (I, [H]),
        "dn_stream": (VP, [H]),
        "dn_last_phase_times": (I, [H, DP]),
        "dn_kernel_launches": (C.c_longlong, [H]),
        "dn_profile_counters": (I, [H, DP, I]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def _dict_to_text(cfg: dict) -> str:
    lines = []
    for k, v in cfg.items():
        if isinstance(v, bool):
            v = "true" if v else "false"
        elif isinstance(v, float):
            v = repr(v)
        lines.append(f"{k} = {v}")
    return "\n".join(lines) + "\n"


def parse_config(cfg) -> Config:
    """A reference case file (text) or a dict of its keys -> dn_config, through dn_config_parse."""
    lib = load()
    text = cfg if isinstance(cfg, str) else _dict_to_text(cfg)
    c = Config()
    err = C.create_string_buffer(512)
    st = lib.dn_config_parse(text.encode(), C.byref(c), err, len(err))
    if st != 0:
        raise DnError(st, err.value.decode())
    return c


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Solver:
    """One device-resident CHNS solver (one handle, one CUDA stream)."""

    def __init__(self, cfg, device: int = 0):
        self._lib = load()
        self.config = parse_config(cfg)
        self.nx, self.ny, self.ghost = self.config.nx, self.config.ny, self.config.ghost
        h = C.c_void_p()
        st = self._lib.dn_create(C.byref(self.config), int(device), C.byref(h))
        self._h = h
        if st != 0:
            msg = self._lib.dn_last_error(h).decode() if h else ""
            self.close()
            raise DnError(st, msg)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.dn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != 0:
            raise DnError(st, self._lib.dn_last_error(self._h).decode())

    # ---- fields
    def field_shape(self, name: str):
        nx = self.nx + (1 if name in U_FIELDS else 0)
        ny = self.ny + (1 if name in V_FIELDS else 0)
        return nx + 2 * self.ghost, ny + 2 * self.ghost

    def get_field(self, name: str, out: np.ndarray = None) -> np.ndarray:
        """Copy a field to the host (into `out` when given: a C-contiguous float64 array of the field's shape)."""
        a = np.empty(self.field_shape(name), dtype=np.float64) if out is None else out
        if a.shape != self.field_shape(name) or a.dtype != np.float64 or not a.flags.c_contiguous:
            raise ValueError(f"{name}: out must be C-contiguous float64 of shape {self.field_shape(name)}")
        self._check(self._lib.dn_get_field(self._h, FIELD_ID[name], _dp(a), a.size))
        return a

    def set_field(self, name: str, values: np.ndarray) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64)
        if a.shape != self.field_shape(name):
            raise ValueError(f"{name}: expected shape {self.field_shape(name)}, got {a.shape}")
        self._check(self._lib.dn_set_field(self._h, FIELD_ID[name], _dp(a), a.size))

    def device_ptr(self, name: str) -> int:
        p = C.POINTER(C.c_double)()
        n = C.c_size_t()
        self._check(self._lib.dn_field_device_ptr(self._h, FIELD_ID[name], C.byref(p), C.byref(n)))
        return C.cast(p, C.c_void_p).value or 0

    def set_initial_mass(self, m: float) -> None:
        self._lib.dn_set_initial_mass(self._h, float(m))

    def refresh_derived(self) -> None:
        self._check(self._lib.dn_refresh_derived(self._h))

    # ---- the step
    def initialize(self) -> None:
        self._check(self._lib.dn_initialize(self._h))

    def advance_one_timestep(self, step: int) -> dict:
        r = Report()
        self._check(self._lib.dn_step(self._h, int(step), C.byref(r)))
        return {n: getattr(r, n) for n, _ in Report._fields_}

    step = advance_one_timestep

    def begin_step(self, step: int) -> None:
        self._check(self._lib.dn_begin_step(self._h, int(step)))

    def phase(self, step: int) -> dict:
        r = Report()
        self._check(self._lib.dn_phase(self._h, int(step), C.byref(r)))
        return {n: getattr(r, n) for n, _ in Report._fields_}

    def momentum(self, step: int) -> dict:
        r = Report()
        self._check(self._lib.dn_momentum(self._h, int(step), C.byref(r)))
        return {n: getattr(r, n) for n, _ in Report._fields_}

    def pressure(self) -> dict:
        r = Report()
        self._check(self._lib.dn_pressure(self._h, C.byref(r)))
        return {n: getattr(r, n) for n, _ in Report._fields_}

    def correct(self) -> dict:
        r = Report()
        self._check(self._lib.dn_correct(self._h, C.byref(r)))
        return {n: getattr(r, n) for n, _ in Report._fields_}

    # ---- backend entry points with host buffers
    def ch_linear_solve(self, rhs: np.ndarray, alpha0: float, c_state: np.ndarray):
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        cs = np.ascontiguousarray(c_state, dtype=np.float64).copy()
        it, eq, n = C.c_double(), C.c_double(), C.c_int()
        self._check(self._lib.dn_ch_linear_solve(self._h, _dp(rhs), float(alpha0), _dp(cs), C.byref(it), C.byref(eq),
                                                 C.byref(n)))
        return cs, it.value, eq.value, n.value

    def pressure_solve(self, step, u_star, v_star, rho_mid, p, p_prev):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (u_star, v_star, rho_mid, p, p_prev)]
        out = np.zeros(self.field_shape("p"), dtype=np.float64)
        its, rel = C.c_int(), C.c_double()
        self._check(self._lib.dn_pressure_solve(self._h, int(step), *[_dp(a) for a in arrs], _dp(out), C.byref(its),
                                                C.byref(rel)))
        return out, its.value, rel.value

    # ---- diagnostics / timing
    def set_pressure_monitor(self, capacity: int) -> None:
        """Record up to `capacity` iterations of every later FP64 pressure solve (the CG monitor)."""
        self._check(self._lib.dn_set_pressure_monitor(self._h, int(capacity)))

    def pressure_monitor(self, capacity: int = 100000) -> np.ndarray:
        """The last pressure solve's record, one row per iteration: abs, rel, iterate residual, alpha."""
        out = np.zeros((capacity, 4))
        cnt = C.c_int()
        self._check(self._lib.dn_pressure_monitor(self._h, _dp(out), capacity, C.byref(cnt)))
        return out[:min(cnt.value, capacity)].copy()

    def pressure_analysis(self, step: int, source_mode: str = "frozen") -> None:
        """Solver::run_pressure_analysis_from_snapshot on the current state (step index `step`): the analysis
        files under output_dir/name/pressure_analysis/."""
        self._check(self._lib.dn_pressure_analysis(self._h, int(step), source_mode.encode()))

    def set_step_graph(self, enable: bool = True) -> None:
        """Replay captured steps (dn_set_step_graph): from the second eager step of index >= 1 on, each step
        is one CUDA graph launch whose solves loop on the device; results equal the eager steps'."""
        self._check(self._lib.dn_set_step_graph(self._h, 1 if enable else 0))

    def autotune_pressure(self) -> dict:
        """Time the pressure solve of the current state over the launch shapes (rows per CTA x sweep warps
        per CTA) and keep the fastest; the solve's P_CORR is rewritten, nothing else of the state."""
        rows, sw, ms = C.c_int(), C.c_int(), C.c_double()
        self._check(self._lib.dn_autotune_pressure(self._h, C.byref(rows), C.byref(sw), C.byref(ms)))
        return {"pcg_rows_per_cta": rows.value, "sweep_warps_per_cta": sw.value, "pressure_ms": ms.value}

    def history_csv_row(self, step: int, time: float, report: dict) -> str:
        """Solver::append_history_csv_entry: the history.csv row of the step whose report is `report`."""
        r = Report(**{n: report[n] for n, _ in Report._fields_})
        buf = C.create_string_buffer(2048)
        self._check(self._lib.dn_history_csv_row(self._h, int(step), float(time), C.byref(r), buf, len(buf), None))
        return buf.value.decode()

    def write_restart(self, path: str, step: int) -> None:
        """Solver::write_restart_snapshot: the reference's v2 snapshot of this solver's state."""
        self._check(self._lib.dn_write_restart(self._h, int(step), str(path).encode()))

    def load_restart(self, path: str) -> int:
        """Solver::load_restart_snapshot: state from a v1/v2 snapshot; returns its step."""
        st = C.c_int()
        self._check(self._lib.dn_load_restart(self._h, str(path).encode(), C.byref(st)))
        return st.value

    def diagnostics(self) -> dict:
        d = Diag()
        self._check(self._lib.dn_diagnostics(self._h, C.byref(d)))
        return {n: getattr(d, n) for n, _ in Diag._fields_}

    def last_diagnostics(self) -> dict:
        """The diagnostics computed at the end of the last step (no device work)."""
        d = Diag()
        self._check(self._lib.dn_last_diagnostics(self._h, C.byref(d)))
        return {n: getattr(d, n) for n, _ in Diag._fields_}

    def compute_mass(self, field: str = "c") -> float:
        m = C.c_double()
        self._check(self._lib.dn_compute_mass(self._h, FIELD_ID[field], C.byref(m)))
        return m.value

    def synchronize(self) -> None:
        self._check(self._lib.dn_synchronize(self._h))

    def stream(self) -> int:
        return self._lib.dn_stream(self._h) or 0

    def phase_times_ms(self) -> list:
        """[ch, momentum, pressure, correction] phase ms, then [pressure PCG kernel, CH PCG kernel, BiCGSTAB kernel]
        ms, the pressure PCG iteration count, and the pressure PCG kernel's split [SpMV, update, sweeps] ms."""
        out = (C.c_double * 11)()
        self._check(self._lib.dn_last_phase_times(self._h, out))
        return list(out)

    def profile_counters(self, count: int = 64) -> list:
        out = (C.c_double * count)()
        self._check(self._lib.dn_profile_counters(self._h, out, count))
        return list(out)

    def kernel_launches(self) -> int:
        return int(self._lib.dn_kernel_launches(self._h))


def step_batch(solvers, steps) -> list:
    """One step of each solver, the solvers advanced concurrently on the device (dn_step_batch).  Returns one
    report dict per solver; each solver's result equals its own step()."""
    lib = load()
    n = len(solvers)
    hs = (C.c_void_p * n)(*[s._h.value for s in solvers])
    st = (C.c_int * n)(*[int(k) for k in steps])
    reps = (Report * n)()
    code = lib.dn_step_batch(hs, n, st, reps)
    if code != 0:
        msgs = [lib.dn_last_error(s._h).decode() for s in solvers]
        raise DnError(code, "; ".join(m for m in msgs if m))
    return [{f: getattr(r, f) for f, _ in Report._fields_} for r in reps]


def history_csv_header() -> str:
    """Solver::write_history_csv_header: the history.csv header line."""
    lib = load()
    buf = C.create_string_buffer(1024)
    lib.dn_history_csv_header(buf, len(buf))
    return buf.value.decode()

