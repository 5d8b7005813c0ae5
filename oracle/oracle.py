"""ctypes bindings for the CPU checkers (TEST INFRASTRUCTURE ONLY).

Two interchangeable back ends expose the same calls:

* ``impl="port"`` -- ``oracle/libdnoracle.so``, the plain-C restatement of the reference step
  (``oracle/dn_oracle.c``);
* ``impl="reference"`` -- ``oracle/_ref/libdnref.so``, the reference's own sources compiled by
  ``oracle/Makefile`` behind ``oracle/ref_harness.cpp``.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import this
module.  The CUDA product never does.

``parse_cfg`` restates the reference's ``load_config`` (src/core/base/config.cpp:49-208): ``key = value``
lines, ``#`` comments, and the defaults of ``struct Config`` (src/core/base/config.hpp:35-136).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "libdnoracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libdnref.so")
# the reference with its pressure and CH dispatchers patched to call libdn_cuda (patch_reference.py)
REF_CUDA_LIB = os.path.join(HERE, "_ref", "libdnref_cuda.so")

BC_UNSET, BC_DIRICHLET, BC_NEUMANN = 0, 1, 2
SIDES = ("left", "right", "bottom", "top")
MODE = {"coupled": 0, "equilibrium": 0, "ch_only": 0, "single_phase": 1, "advection_only": 2}
PRESSURE = {
    "jacobi": 0,
    "icpcg": 1,
    "ildlt_pcg": 2,
    "split_icpcg": 3, "liu_split_icpcg": 3, "paper_split_icpcg": 3,
    "split_ildlt_pcg": 4, "liu_split_ildlt_pcg": 4, "paper_split_ildlt_pcg": 4,
    "split_dcdm_icpcg": 5, "liu_split_dcdm_icpcg": 5, "paper_split_dcdm_icpcg": 5,
}
DCDM_DIRECTION = {"icc_preconditioned": 0, "icc": 0, "pcg_preconditioned": 0, "identity": 1}

# struct Config defaults, config.hpp:35-136 (keys read by the time step).
DEFAULTS = {
    "name": "unnamed", "mode": "coupled", "ch_solver": "sparse_pcg", "pressure_scheme": "jacobi",
    "phase_initializer": "default", "velocity_profile": "default", "momentum_advection_scheme": "centered",
    "nx": 64, "ny": 64, "ghost": 3, "steps": 1,
    "ch_inner_iterations": 30, "momentum_iterations": 50, "poisson_iterations": 400,
    "surface_tension_smoothing_passes": 0,
    "dt": 1.0e-4, "lx": 1.0, "ly": 1.0, "re": 100.0, "ca": 1.0, "pe": 100.0, "cn": 0.02,
    "density_ratio": 0.1, "viscosity_ratio": 0.1, "surface_tension_multiplier": 1.0,
    "surface_tension_smoothing_weight": 0.0,
    "ch_tolerance": 1.0e-8, "pressure_tolerance": 1.0e-8, "momentum_tolerance": 1.0e-8,
    "body_force_x": 0.0, "body_force_y": 0.0,
    "interface_center_x": 0.5, "interface_center_y": 0.5, "interface_radius": 0.18,
    "interface_amplitude": 0.0, "interface_wavenumber": 1.0,
    "zalesak_slot_width": 0.05, "zalesak_slot_depth": 0.25,
    "advect_u": 0.0, "advect_v": 0.0, "rotation_center_x": 0.5, "rotation_center_y": 0.5,
    "angular_velocity": 0.0, "top_wall_velocity_x": 0.0, "bottom_wall_velocity_x": 0.0,
    "periodic_x": True, "periodic_y": True, "invert_phase": False, "freeze_ch": False,
    "dcdm_direction_mode": "icc_preconditioned", "dcdm_history_size": 2, "dcdm_max_stored_directions": 8,
    "dcdm_restart_interval": 0,
}
for _f in ("pressure", "u", "v"):
    for _s in SIDES:
        DEFAULTS[f"{_f}_bc_{_s}_type"] = "unset"
        DEFAULTS[f"{_f}_bc_{_s}_value"] = 0.0

_INT_KEYS = {"nx", "ny", "ghost", "steps", "ch_inner_iterations", "momentum_iterations", "poisson_iterations",
             "surface_tension_smoothing_passes", "dcdm_history_size", "dcdm_max_stored_directions",
             "dcdm_restart_interval"}
_BOOL_KEYS = {"periodic_x", "periodic_y", "invert_phase", "freeze_ch"}
_STR_KEYS = {"name", "mode", "ch_solver", "pressure_scheme", "phase_initializer", "velocity_profile",
             "momentum_advection_scheme", "dcdm_direction_mode"}


def _parse_bool(v: str) -> bool:
    return v.strip().lower() in ("1", "true", "yes", "on")


def parse_cfg(text: str) -> dict:
    """Parse a reference case file into a dict of typed values (config.cpp:49-208)."""
    kv = {}
    for line in text.splitlines():
        line = line.split("#", 1)[0].strip()
        if not line or "=" not in line:
            continue
        k, v = line.split("=", 1)
        kv[k.strip()] = v.strip()
    if "stabilization_a1" in kv or "stabilization_a2" in kv:
        raise ValueError("stabilization_a1/stabilization_a2 are derived from cn and must not be set in case files")
    cfg = dict(DEFAULTS)
    for k, v in kv.items():
        if k not in cfg:
            continue
        if k in _INT_KEYS:
            cfg[k] = int(v)
        elif k in _BOOL_KEYS:
            cfg[k] = _parse_bool(v)
        elif k in _STR_KEYS or k.endswith("_type"):
            cfg[k] = v
        else:
            cfg[k] = float(v)
    return cfg


def with_defaults(overrides: dict) -> dict:
    cfg = dict(DEFAULTS)
    cfg.update(overrides)
    return cfg


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
        ("p_bc", BC * 4), ("u_bc", BC * 4), ("v_bc", BC * 4)] + [(n, C.c_int) for n in (
        "dcdm_direction_mode", "dcdm_history_size", "dcdm_max_stored_directions", "dcdm_restart_interval")]


class Report(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "ch_iterations", "momentum_iterations", "pressure_iterations", "coupling_iterations",
        "ch_preconditioner")] + [(n, C.c_double) for n in (
        "ch_residual", "ch_equation_residual", "momentum_residual", "pressure_residual",
        "boundary_speed_pre", "boundary_speed_post")]


class Diag(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "mass", "mass_drift", "divergence_l2", "max_divergence", "max_abs_mu", "max_velocity", "kinetic_energy",
        "total_free_energy", "rho_min", "rho_max", "eta_min", "eta_max", "dt_limit_advective",
        "dt_limit_capillary", "dt_limit_ch_explicit", "dt_limit_active", "dt_limit_ratio")]


FIELDS = ("c", "c_prev", "c_prev2", "mu", "rho", "eta", "rho_prev", "eta_prev", "rho_mid", "eta_mid", "p",
          "p_prev", "p_corr", "u", "v", "u_prev", "v_prev", "u_star", "v_star", "sfx_cell", "sfy_cell", "sfx_u",
          "sfy_v", "e_prev", "hu_prev", "hv_prev")
FIELD_ID = {n: k for k, n in enumerate(FIELDS)}


def _bc_type(name: str) -> int:
    s = str(name).strip().lower()
    return {"": BC_UNSET, "unset": BC_UNSET, "default": BC_UNSET, "dirichlet": BC_DIRICHLET, "neumann": BC_NEUMANN}[s]


def to_struct(cfg: dict) -> Config:
    c = Config()
    for n, t in Config._fields_:
        if n in ("p_bc", "u_bc", "v_bc"):
            continue
        if n == "mode":
            c.mode = MODE[cfg["mode"]]
        elif n == "pressure_scheme":
            if cfg["pressure_scheme"] not in PRESSURE:
                raise ValueError(f"unsupported pressure scheme: {cfg['pressure_scheme']}")
            c.pressure_scheme = PRESSURE[cfg["pressure_scheme"]]
        elif n == "phase_initializer":
            c.phase_initializer = 1 if cfg["phase_initializer"] == "zalesak_disk" else 0
        elif n == "velocity_profile":
            c.velocity_profile = 1 if cfg["velocity_profile"] == "solid_body_rotation" else 0
        elif n == "dcdm_direction_mode":
            mode = str(cfg["dcdm_direction_mode"]).lower()
            if mode not in DCDM_DIRECTION:
                raise ValueError(f"unsupported dcdm_direction_mode: {cfg['dcdm_direction_mode']}")
            c.dcdm_direction_mode = DCDM_DIRECTION[mode]
        else:
            setattr(c, n, t(cfg[n]).value if t is C.c_double else int(cfg[n]))
    for f, attr in (("pressure", "p_bc"), ("u", "u_bc"), ("v", "v_bc")):
        arr = getattr(c, attr)
        for k, side in enumerate(SIDES):
            arr[k].type = _bc_type(cfg[f"{f}_bc_{side}_type"])
            arr[k].value = float(cfg[f"{f}_bc_{side}_value"])
    return c


def build(force: bool = False) -> None:
    """Compile the checkers with oracle/Makefile (the reference harness only where the reference exists)."""
    targets = ["oracle"]
    ref = os.environ.get("DN_REFERENCE", "")
    if ref and os.path.isdir(ref):
        targets.append("ref")
        if os.path.exists(os.path.join(os.path.dirname(HERE), "ding_nsch_core_solver_b200", "libdn_cuda.so")):
            targets.append("refcuda")
    cmd = ["make", "-s", "-C", HERE] + (["-B"] if force else []) + targets + ([f"REFERENCE={ref}"] if ref else [])
    subprocess.run(cmd, check=True)


_LIBS: dict = {}


def _load(impl: str):
    if impl in _LIBS:
        return _LIBS[impl]
    path = {"port": PORT_LIB, "reference": REF_LIB, "reference_cuda": REF_CUDA_LIB}[impl]
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing; run `make -C oracle`")
    lib = C.CDLL(path)
    pre = "orc_" if impl == "port" else "ref_"
    vp = C.c_void_p
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    sig = {
        "create": (vp, [C.POINTER(Config)]), "destroy": (None, [vp]), "last_error": (C.c_char_p, [vp]),
        "field": (dp, [vp, C.c_int, ip, ip, ip]), "set_initial_mass": (None, [vp, C.c_double]),
        "initialize": (C.c_int, [vp]), "step": (C.c_int, [vp, C.c_int]), "begin_step": (C.c_int, [vp, C.c_int]),
        "phase": (C.c_int, [vp, C.c_int]), "momentum": (C.c_int, [vp, C.c_int]), "pressure": (C.c_int, [vp]),
        "correct": (C.c_int, [vp]), "finish_step": (C.c_int, [vp]), "refresh_derived": (C.c_int, [vp]),
        "ch_linear_solve": (C.c_int, [vp, dp, C.c_double, dp, dp, dp]),
        "get_report": (None, [vp, C.POINTER(Report)]), "diagnostics": (None, [vp, C.POINTER(Diag)]),
        "compute_mass": (C.c_double, [vp, C.c_int]),
    }
    if impl in ("reference", "reference_cuda"):
        sig["time_steps"] = (C.c_double, [vp, C.c_int, C.c_int])
        sig["pressure_analysis"] = (C.c_int, [vp, C.c_int, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p,
                                              C.c_char_p, C.c_double])
    else:
        sig["advection"] = (C.c_int, [vp, dp, dp, dp, dp])
        sig["explicit_operator"] = (C.c_int, [vp, dp, dp, dp, dp])
        sig["set_pressure_monitor"] = (None, [vp, C.c_int])
        sig["pressure_monitor"] = (C.c_int, [vp, dp, C.c_int])
    fns = {}
    for name, (res, args) in sig.items():
        fn = getattr(lib, pre + name)
        fn.restype = res
        fn.argtypes = args
        fns[name] = fn
    _LIBS[impl] = fns
    return fns


class OracleError(RuntimeError):
    pass


class OracleSolver:
    """One reference ``Solver`` instance on the CPU (restated port or the reference build)."""

    def __init__(self, cfg: dict, impl: str = "port"):
        self.cfg = dict(cfg)
        self.impl = impl
        self._f = _load(impl)
        self._cs = to_struct(self.cfg)
        self._h = self._f["create"](C.byref(self._cs))

    def close(self):
        if self._h:
            self._f["destroy"](self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise OracleError(self._f["last_error"](self._h).decode())

    def field(self, name: str) -> np.ndarray:
        """Writable numpy view of a ghosted field, shape (nx'+2g, ny'+2g), j contiguous."""
        nx, ny, g = C.c_int(), C.c_int(), C.c_int()
        ptr = self._f["field"](self._h, FIELD_ID[name], C.byref(nx), C.byref(ny), C.byref(g))
        shape = (nx.value + 2 * g.value, ny.value + 2 * g.value)
        return np.ctypeslib.as_array(ptr, shape=shape)

    def interior(self, name: str) -> np.ndarray:
        g = self.cfg["ghost"]
        a = self.field(name)
        return a[g:a.shape[0] - g, g:a.shape[1] - g]

    def set_field(self, name: str, values: np.ndarray) -> None:
        a = self.field(name)
        a[...] = values

    def set_initial_mass(self, m: float) -> None:
        self._f["set_initial_mass"](self._h, float(m))

    def initialize(self):
        self._check(self._f["initialize"](self._h))

    def step(self, k: int):
        self._check(self._f["step"](self._h, int(k)))

    def begin_step(self, k: int):
        self._check(self._f["begin_step"](self._h, int(k)))

    def phase(self, k: int):
        self._check(self._f["phase"](self._h, int(k)))

    def momentum(self, k: int):
        self._check(self._f["momentum"](self._h, int(k)))

    def pressure(self):
        self._check(self._f["pressure"](self._h))

    def correct(self):
        self._check(self._f["correct"](self._h))

    def finish_step(self):
        self._check(self._f["finish_step"](self._h))

    def refresh_derived(self):
        """Rebuild BC ghosts, materials and mu from the state fields, as a restart load does (io.cpp:412-436)."""
        self._check(self._f["refresh_derived"](self._h))

    def pressure_analysis(self, step: int, source_mode: str, output_dir: str, name: str, case_group: str = "",
                          spectrum_iterations: str = "0,1,2,5,10,20,final", band: float = 2.0):
        """The reference's pressure analysis files of the current state (reference build only)."""
        self._check(self._f["pressure_analysis"](self._h, int(step), source_mode.encode(), output_dir.encode(),
                                                 name.encode(), case_group.encode(), spectrum_iterations.encode(),
                                                 float(band)))

    def ch_linear_solve(self, rhs: np.ndarray, alpha0: float, c_state: np.ndarray):
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        cs = np.ascontiguousarray(c_state, dtype=np.float64).copy()
        it, eq = C.c_double(), C.c_double()
        dp = C.POINTER(C.c_double)
        self._check(self._f["ch_linear_solve"](self._h, rhs.ctypes.data_as(dp), float(alpha0), cs.ctypes.data_as(dp),
                                               C.byref(it), C.byref(eq)))
        return cs, it.value, eq.value

    def advection(self, c: np.ndarray, u: np.ndarray, v: np.ndarray) -> np.ndarray:
        """-div(u c) with WENO5 face values (port only); Field2D arrays in, the cell array out."""
        dp = C.POINTER(C.c_double)
        c, u, v = (np.ascontiguousarray(a, dtype=np.float64) for a in (c, u, v))
        out = np.zeros_like(self.field("c"))
        self._check(self._f["advection"](self._h, *(a.ctypes.data_as(dp) for a in (c, u, v, out))))
        return out

    def explicit_operator(self, c: np.ndarray, u: np.ndarray, v: np.ndarray) -> np.ndarray:
        """The CH explicit operator E(c, u, v) (port only); Field2D arrays in, the cell array out."""
        dp = C.POINTER(C.c_double)
        c, u, v = (np.ascontiguousarray(a, dtype=np.float64) for a in (c, u, v))
        out = np.zeros_like(self.field("c"))
        self._check(self._f["explicit_operator"](self._h, *(a.ctypes.data_as(dp) for a in (c, u, v, out))))
        return out

    def set_pressure_monitor(self, capacity: int) -> None:
        self._f["set_pressure_monitor"](self._h, int(capacity))

    def pressure_monitor(self, capacity: int = 100000) -> np.ndarray:
        """The last pressure solve's CG-monitor record (port only): abs, rel, iterate residual, alpha."""
        out = np.zeros((capacity, 4))
        cnt = self._f["pressure_monitor"](self._h, out.ctypes.data_as(C.POINTER(C.c_double)), capacity)
        return out[:min(cnt, capacity)].copy()

    def report(self) -> dict:
        r = Report()
        self._f["get_report"](self._h, C.byref(r))
        return {n: getattr(r, n) for n, _ in Report._fields_}

    def diagnostics(self) -> dict:
        d = Diag()
        self._f["diagnostics"](self._h, C.byref(d))
        return {n: getattr(d, n) for n, _ in Diag._fields_}

    def time_steps(self, first_step: int, count: int) -> float:
        """Wall seconds for ``count`` steps (steady clock inside the reference build)."""
        if self.impl != "reference":
            import time
            t0 = time.perf_counter()
            for k in range(count):
                self.step(first_step + k)
            return time.perf_counter() - t0
        sec = self._f["time_steps"](self._h, int(first_step), int(count))
        if sec < 0:
            raise OracleError(self._f["last_error"](self._h).decode())
        return sec


def available(impl: str) -> bool:
    return os.path.exists({"port": PORT_LIB, "reference": REF_LIB, "reference_cuda": REF_CUDA_LIB}[impl])
