"""Pins the CPU oracle (the C restatement of the reference step) to the reference itself.

* against the reference's published golden run (176Result case 92, reduced under tests/golden/);
* bit for bit against the reference sources compiled by oracle/Makefile (oracle/_ref), on seeded
  states over every periodicity / boundary-condition / pressure-scheme / mode combination;
* against the reference unit tests' own known answers (src/tests/core_solver_unit_tests.cpp).
"""
import csv
import math
import os

import numpy as np
import pytest

from oracle.oracle import OracleSolver, available, parse_cfg, with_defaults

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
STATE_FIELDS = ("c", "c_prev", "p", "p_prev", "u", "v", "e_prev", "hu_prev", "hv_prev")
OUT_FIELDS = ("c", "mu", "rho", "eta", "rho_mid", "u", "v", "p", "p_prev", "p_corr", "u_star", "v_star", "sfx_u",
              "sfy_v", "e_prev", "hu_prev", "hv_prev")


def unit_config(**kw):
    """Base configuration of the reference unit tests (core_solver_unit_tests.cpp:25-43)."""
    base = dict(nx=32, ny=32, ghost=3, dt=1.0e-3, periodic_x=True, periodic_y=True, poisson_iterations=5000,
                pressure_tolerance=1.0e-10, momentum_iterations=200, momentum_tolerance=1.0e-10,
                density_ratio=10.0, viscosity_ratio=5.0)
    base.update(kw)
    return with_defaults(base)


def seeded_state(solver, seed, amp=0.02):
    """Perturb c, u, v, p of an initialised solver with seeded noise and rebuild the derived fields the way a
    restart does (io.cpp:412-436): the same state is injected into every implementation under test."""
    rng = np.random.default_rng(seed)
    g = solver.cfg["ghost"]
    for name, a in (("c", amp), ("u", 0.05), ("v", 0.05), ("p", 0.1)):
        f = solver.field(name)
        f[g:-g, g:-g] += a * rng.standard_normal(f[g:-g, g:-g].shape)
    solver.refresh_derived()
    from oracle.oracle import FIELDS
    return {n: solver.field(n).copy() for n in FIELDS}


def inject(solver, state):
    for n, a in state.items():
        solver.set_field(n, a)


def test_parse_case92_cfg():
    cfg = parse_cfg(open(os.path.join(GOLDEN, "case92.cfg")).read())
    assert cfg["nx"] == 128 and cfg["ny"] == 128 and cfg["pressure_scheme"] == "icpcg"
    assert cfg["dt"] == 2e-7 and cfg["periodic_x"] and cfg["periodic_y"]
    assert cfg["steps"] == 5000 and cfg["pressure_tolerance"] == 1e-10
    with pytest.raises(ValueError):
        parse_cfg("stabilization_a1 = 1.0\n")


@pytest.mark.parametrize("impl", ["port", "reference"])
def test_golden_history_bitwise(impl):
    """The first 12 steps of case 92 reproduce the published history.csv bit for bit."""
    if not available(impl):
        pytest.skip(f"{impl} checker not built")
    cfg = parse_cfg(open(os.path.join(GOLDEN, "case92.cfg")).read())
    rows = list(csv.DictReader(open(os.path.join(GOLDEN, "case92_history.csv"))))
    s = OracleSolver(cfg, impl)
    s.initialize()
    assert s.diagnostics()["mass"] == float(rows[0]["mass"])
    for k in range(12):
        s.step(k)
        d, r, row = s.diagnostics(), s.report(), rows[k + 1]
        for col in ("mass", "mass_drift", "divergence_l2", "max_divergence", "max_abs_mu", "max_velocity",
                    "kinetic_energy", "total_free_energy"):
            assert d[col] == float(row[col]), (k, col)
        assert r["ch_residual"] == float(row["ch_inner_residual"])
        assert r["ch_equation_residual"] == float(row["ch_equation_residual"])
        assert r["pressure_residual"] == float(row["pressure_correction_residual"])
        assert r["momentum_residual"] == float(row["momentum_residual"])
        assert (r["ch_iterations"], r["pressure_iterations"], r["momentum_iterations"]) == (
            int(row["ch_iterations"]), int(row["pressure_iterations"]), int(row["momentum_iterations"]))


CASES = {
    "periodic_icpcg": unit_config(pressure_scheme="icpcg"),
    "periodic_split_icpcg": unit_config(pressure_scheme="split_icpcg"),
    "periodic_ildlt": unit_config(pressure_scheme="ildlt_pcg"),
    "walls_split_ildlt": unit_config(nx=20, ny=28, periodic_x=False, periodic_y=False,
                                     pressure_scheme="split_ildlt_pcg", body_force_y=-0.98, dt=1e-4),
    "channel_x_icpcg": unit_config(nx=24, ny=16, periodic_x=True, periodic_y=False, pressure_scheme="icpcg",
                                   top_wall_velocity_x=0.5, bottom_wall_velocity_x=-0.5, dt=1e-4),
    "channel_y_split": unit_config(nx=16, ny=24, periodic_x=False, periodic_y=True, pressure_scheme="split_icpcg",
                                   dt=1e-4),
    "mixed_bcs_icpcg": unit_config(
        nx=18, ny=22, periodic_x=False, periodic_y=False, pressure_scheme="icpcg", dt=1e-4,
        u_bc_left_type="dirichlet", u_bc_left_value=-0.1, u_bc_right_type="neumann", u_bc_right_value=0.05,
        v_bc_left_type="neumann", v_bc_right_type="neumann", v_bc_top_type="neumann", v_bc_top_value=0.02,
        pressure_bc_top_type="dirichlet", pressure_bc_top_value=0.3),
    "smoothing_split": unit_config(nx=20, ny=20, pressure_scheme="split_icpcg", surface_tension_smoothing_passes=2,
                                   surface_tension_smoothing_weight=0.1, dt=1e-4),
    "freeze_ch": unit_config(freeze_ch=True, pressure_scheme="icpcg", surface_tension_multiplier=0.0),
    "single_phase": unit_config(mode="single_phase", pressure_scheme="icpcg", density_ratio=3.0),
    "jacobi": unit_config(nx=12, ny=12, pressure_scheme="jacobi", poisson_iterations=300, dt=1e-4),
    "dcdm_walls": unit_config(nx=20, ny=28, periodic_x=False, periodic_y=False, pressure_scheme="split_dcdm_icpcg",
                              body_force_y=-0.98, dt=1e-4),
    "dcdm_periodic": unit_config(pressure_scheme="split_dcdm_icpcg"),
    "dcdm_identity_dirichlet": unit_config(nx=18, ny=22, periodic_x=False, periodic_y=False,
                                           pressure_scheme="split_dcdm_icpcg", dcdm_direction_mode="identity",
                                           dcdm_history_size=0, dcdm_max_stored_directions=4,
                                           pressure_bc_top_type="dirichlet", pressure_bc_top_value=0.3, dt=1e-4),
    "advection_only": unit_config(mode="advection_only", velocity_profile="solid_body_rotation",
                                  angular_velocity=2 * math.pi, phase_initializer="zalesak_disk",
                                  interface_radius=0.3),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_port_matches_reference_build_bitwise(name):
    if not available("reference"):
        pytest.skip("reference build absent")
    cfg = CASES[name]
    port, ref = OracleSolver(cfg, "port"), OracleSolver(cfg, "reference")
    port.initialize()
    ref.initialize()
    state = seeded_state(port, seed=hash(name) % 1000, amp=0.0 if cfg["mode"] != "coupled" else 0.02)
    inject(ref, state)
    for s in (port, ref):
        s.set_initial_mass(0.0)
    for k in range(3):
        port.step(k)
        ref.step(k)
        for f in OUT_FIELDS:
            np.testing.assert_array_equal(port.field(f), ref.field(f), err_msg=f"{name} step {k} field {f}")
        rp, rr = port.report(), ref.report()
        for key in ("ch_iterations", "momentum_iterations", "pressure_iterations", "ch_preconditioner"):
            assert rp[key] == rr[key], (name, k, key)
        dp, dr = port.diagnostics(), ref.diagnostics()
        for key in dp:
            assert dp[key] == dr[key] or (math.isinf(dp[key]) and math.isinf(dr[key])), (name, k, key)


def test_refresh_derived_matches_reference_build():
    """The restart-load rebuild (io.cpp:412-436) used to inject seeded states agrees bit for bit."""
    if not available("reference"):
        pytest.skip("reference build absent")
    cfg = CASES["mixed_bcs_icpcg"]
    port, ref = OracleSolver(cfg, "port"), OracleSolver(cfg, "reference")
    port.initialize()
    ref.initialize()
    rng = np.random.default_rng(1)
    for s in (port, ref):
        for name in ("c", "c_prev", "u", "v", "p", "p_prev"):
            s.field(name)[...] = np.random.default_rng(hash(name) % 97).standard_normal(s.field(name).shape)
        s.refresh_derived()
    from oracle.oracle import FIELDS
    for f in FIELDS:
        np.testing.assert_array_equal(port.field(f), ref.field(f), err_msg=f)


def test_port_phases_match_reference_build():
    """Phase-by-phase entry points (the per-backend boundary) agree with the reference build."""
    if not available("reference"):
        pytest.skip("reference build absent")
    cfg = CASES["walls_split_ildlt"]
    port, ref = OracleSolver(cfg, "port"), OracleSolver(cfg, "reference")
    port.initialize()
    ref.initialize()
    inject(ref, seeded_state(port, 7))
    for s in (port, ref):
        s.begin_step(1)
        s.phase(1)
        s.momentum(1)
        s.pressure()
        s.correct()
        s.finish_step()
    for f in OUT_FIELDS:
        np.testing.assert_array_equal(port.field(f), ref.field(f), err_msg=f)


def test_boundary_condition_known_answers():
    """Ghost/face rules pinned by test_configurable_boundary_conditions_apply_expected_values
    (core_solver_unit_tests.cpp:149-215), checked on the port."""
    cfg = unit_config(periodic_x=False, periodic_y=False,
                      u_bc_left_type="dirichlet", u_bc_left_value=-0.5, u_bc_right_type="neumann",
                      u_bc_right_value=0.25, u_bc_bottom_type="neumann", u_bc_bottom_value=0.1,
                      u_bc_top_type="dirichlet", u_bc_top_value=1.5, v_bc_left_type="neumann", v_bc_left_value=-0.2,
                      v_bc_right_type="dirichlet", v_bc_right_value=0.7, v_bc_bottom_type="dirichlet",
                      v_bc_bottom_value=-1.2, v_bc_top_type="neumann", v_bc_top_value=0.3,
                      pressure_bc_left_type="dirichlet", pressure_bc_left_value=2.0,
                      pressure_bc_right_type="neumann", pressure_bc_right_value=0.4,
                      pressure_bc_bottom_type="neumann", pressure_bc_bottom_value=-0.1,
                      pressure_bc_top_type="dirichlet", pressure_bc_top_value=-3.0, pressure_scheme="icpcg")
    s = OracleSolver(cfg, "port")
    s.initialize()
    g, nx, ny = 3, 32, 32
    dx = dy = 1.0 / 32
    # a pressure-correction solve exercises apply_pressure_bc on p_corr; check the ghost rules on it.
    s.begin_step(0)
    s.phase(0)
    s.momentum(0)
    s.pressure()
    P = s.field("p_corr")
    at = lambda f, i, j: f[i + g, j + g]
    assert abs(at(P, -1, 4) - (2 * 2.0 - at(P, 0, 4))) < 1e-12
    assert abs(at(P, nx, 4) - (at(P, nx - 1, 4) + 0.4 * dx)) < 1e-12
    assert abs(at(P, 6, -1) - (at(P, 6, 0) - 0.1 * dy)) < 1e-12
    assert abs(at(P, 6, ny) - (2 * -3.0 - at(P, 6, ny - 1))) < 1e-12
    U, V = s.field("u_star"), s.field("v_star")
    assert abs(at(U, 0, 5) - (-0.5)) < 1e-12
    assert abs(at(U, nx, 5) - (at(U, nx - 1, 5) + 0.25 * dx)) < 1e-12
    assert abs(at(U, 4, -1) - (at(U, 4, 0) + 0.1 * dy)) < 1e-12
    assert abs(at(U, 4, ny) - (2 * 1.5 - at(U, 4, ny - 1))) < 1e-12
    assert abs(at(V, 5, 0) - (-1.2)) < 1e-12
    assert abs(at(V, 5, ny) - (at(V, 5, ny - 1) + 0.3 * dy)) < 1e-12
    assert abs(at(V, -1, 6) - (at(V, 0, 6) - 0.2 * dx)) < 1e-12
    assert abs(at(V, nx, 6) - (2 * 0.7 - at(V, nx - 1, 6))) < 1e-12


def test_ch_solver_recovers_manufactured_state():
    """test_ch_sparse_krylov_solver_recovers_reference_state (core_solver_unit_tests.cpp:217-283) on the port."""
    cfg = unit_config(ch_inner_iterations=200, ch_tolerance=1e-12)
    s = OracleSolver(cfg, "port")
    s.initialize()
    g, n = 3, 32
    dx = 1.0 / n
    x = (np.arange(n) + 0.5) * dx
    c_exact = 0.42 + 0.08 * np.sin(2 * np.pi * x)[:, None] * np.cos(2 * np.pi * x)[None, :]
    ext = np.pad(c_exact, g, mode="wrap")

    def lap(a):
        out = np.zeros_like(a)
        out[g:-g, g:-g] = ((a[g + 1:-g + 1 or None, g:-g] - 2 * a[g:-g, g:-g] + a[g - 1:-g - 1, g:-g]) / dx ** 2 +
                           (a[g:-g, g + 1:-g + 1 or None] - 2 * a[g:-g, g:-g] + a[g:-g, g - 1:-g - 1]) / dx ** 2)
        return np.pad(out[g:-g, g:-g], g, mode="wrap")

    L = lap(ext)
    B = lap(L)
    alpha0 = 3.0 / (2.0 * cfg["dt"])
    a1 = 3 * math.sqrt(2) / (16 * cfg["cn"])
    a2 = 3 * math.sqrt(2) * cfg["cn"] / 4
    rhs = alpha0 * ext - (a1 * L - a2 * B) / cfg["pe"]
    cs, it_res, eq_res = s.ch_linear_solve(rhs, alpha0, np.zeros_like(ext))
    err = np.sqrt(((cs[g:-g, g:-g] - c_exact) ** 2).sum() / (c_exact ** 2).sum())
    assert math.isfinite(it_res) and eq_res < 1e-10 and err < 1e-8


def test_ch_step0_preserves_constant_state():
    """test_ch_step0_preserves_constant_equilibrium_state (core_solver_unit_tests.cpp:285-319)."""
    cfg = unit_config(dt=1e-4, density_ratio=1.0, viscosity_ratio=1.0, pressure_scheme="icpcg")
    s = OracleSolver(cfg, "port")
    s.initialize()
    for n in ("c", "c_prev", "c_prev2"):
        s.field(n)[...] = 1.0
    s.field("u")[...] = 0.0
    s.field("v")[...] = 0.0
    s.begin_step(0)
    s.phase(0)
    assert np.max(np.abs(s.interior("c") - 1.0)) < 1e-10


def test_projection_reduces_divergence():
    """Variable-coefficient projection cuts the divergence of a manufactured u*, v* by more than 100x
    (core_solver_unit_tests.cpp:104-147, here with the icpcg backend)."""
    cfg = unit_config(pressure_scheme="icpcg")
    s = OracleSolver(cfg, "port")
    s.initialize()
    g, n = 3, 32
    dx = 1.0 / n
    xc = (np.arange(n) + 0.5) * dx
    xf = np.arange(n + 1) * dx
    s.field("c")[g:-g, g:-g] = 0.5 + 0.3 * np.sin(2 * np.pi * xc)[:, None] * np.cos(2 * np.pi * xc)[None, :]
    s.begin_step(0)
    s.phase(0)
    us, vs = s.field("u_star"), s.field("v_star")
    us[g:-g, g:-g] = np.sin(2 * np.pi * xf)[:, None] * np.cos(2 * np.pi * xc)[None, :]
    vs[g:-g, g:-g] = np.cos(2 * np.pi * xc)[:, None] * np.sin(2 * np.pi * xf)[None, :]

    def div_l2(u, v):
        d = (u[g + 1:g + n + 1, g:-g] - u[g:g + n, g:-g]) / dx + (v[g:-g, g + 1:g + n + 1] - v[g:-g, g:g + n]) / dx
        return np.sqrt((d ** 2).mean())

    before = div_l2(us, vs)
    s.pressure()
    s.correct()
    after = div_l2(s.field("u"), s.field("v"))
    assert after < before / 100.0


# ---- failure paths: the restatement fails where and how the reference fails --------------------------
def _failure_cases():
    cfg = unit_config(nx=40, ny=32, periodic_x=False, periodic_y=False, pressure_scheme="icpcg", dt=1e-4)
    return cfg


def _error_of(fn):
    from oracle.oracle import OracleError
    try:
        fn()
    except OracleError as e:
        return str(e)
    return None


@pytest.mark.skipif(not available("reference"), reason="reference build (oracle/_ref) not built")
def test_failure_paths_match_reference_build():
    """A NaN in c (the CH PCG breaks down, its diagonal retry too: phase_field.cpp:468-473,
    ch_sparse_krylov.hpp:566-568), a density field with negative values (the variable pressure operator is
    indefinite, ICC fails: ch_sparse_krylov.hpp:400-402, pressure.cpp:36-38) and an exhausted pressure
    iteration budget (no error, the unconverged residual is reported) give the same outcome on the port and
    on the reference build."""
    cfg = _failure_cases()
    g = cfg["ghost"]
    out = {}
    for impl in ("port", "reference"):
        nan = OracleSolver(cfg, impl)
        nan.initialize()
        nan.field("c")[g + 5, g + 5] = np.nan
        bad = OracleSolver(cfg, impl)
        bad.initialize()
        bad.field("rho_mid")[g + 10:g + 20, g + 8:g + 16] = -2.0
        bad.field("u_star")[g:-g, g:-g] = 0.01 * np.random.default_rng(0).standard_normal(
            bad.field("u_star")[g:-g, g:-g].shape)
        short = OracleSolver(dict(cfg, poisson_iterations=3), impl)
        short.initialize()
        short.step(0)
        rep = short.report()
        out[impl] = (_error_of(lambda: nan.step(0)), _error_of(bad.pressure), rep["pressure_iterations"],
                     rep["pressure_residual"])
    assert out["port"] == out["reference"], out
    assert out["reference"][0] == "pcg preconditioner breakdown: non-positive r^T M^{-1} r"
    assert out["reference"][1] == "ICC preconditioner construction failed"
    assert out["reference"][2] == 3


def test_patched_reference_build_binds_the_c_abi():
    """oracle/_ref/libdnref_cuda.so (the reference patched by oracle/patch_reference.py) loads, and every
    library symbol it needs is declared in include/dn_cuda.h (the CPU half of
    tests/test_gpu_reference_binding.py)."""
    import ctypes
    import re
    import subprocess

    from oracle.oracle import REF_CUDA_LIB, available

    if not available("reference_cuda"):
        pytest.skip("oracle/_ref/libdnref_cuda.so not built (make -C oracle refcuda with DN_REFERENCE set)")
    lib = ctypes.CDLL(REF_CUDA_LIB)
    assert hasattr(lib, "ref_create") and hasattr(lib, "ref_step")
    out = subprocess.run(["nm", "-D", "--undefined-only", REF_CUDA_LIB], capture_output=True, text=True,
                         check=True).stdout
    needed = sorted(set(re.findall(r"\bU (dn_\w+)", out)))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    header = open(os.path.join(root, "include", "dn_cuda.h")).read()
    assert {"dn_create", "dn_pressure_solve", "dn_ch_linear_solve"} <= set(needed), needed
    for name in needed:
        assert re.search(r"\b" + name + r"\s*\(", header), name


def test_oracle_ctypes_structs_match_its_header(tmp_path):
    """oracle.py's ctypes mirrors have oracle/dn_oracle.h's sizes and field offsets (a C program compiled
    against the header prints them), so the checker never reads a shifted struct."""
    import ctypes as C
    import subprocess

    from oracle import oracle as o

    mirrors = {"orc_bc": o.BC, "orc_config": o.Config, "orc_report": o.Report, "orc_diag": o.Diag}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "dn_oracle.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
        for n, _ in py._fields_:
            lines.append(f'  printf("{cname}.{n} %zu\\n", offsetof({cname}, {n}));')
    lines += ["  return 0;", "}"]
    src, exe = tmp_path / "layout.c", tmp_path / "layout"
    src.write_text("\n".join(lines) + "\n")
    here = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle")
    subprocess.run(["gcc", "-std=c99", "-I", here, "-o", str(exe), str(src)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                       check=True).stdout.splitlines())
    for cname, py in mirrors.items():
        assert int(got[cname]) == C.sizeof(py), (cname, got[cname], C.sizeof(py))
        for n, _ in py._fields_:
            assert int(got[f"{cname}.{n}"]) == getattr(py, n).offset, (cname, n)
