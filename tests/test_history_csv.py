"""history.csv rows (dn_history_csv_header / dn_history_csv_row; Solver::write_history_csv_header and
append_history_csv_entry, io.cpp:179-206): the reference's columns, 17 significant digits, its solver
names and dt-limit source."""
import math

import numpy as np
import pytest

from ding_nsch_core_solver_b200 import capi

# io.cpp:180-184
HEADER = ("step,time,mass,mass_drift,divergence_l2,max_divergence,max_abs_mu,max_velocity,kinetic_energy,"
          "total_free_energy,ch_inner_residual,ch_equation_residual,coupling_residual,pressure_correction_residual,"
          "momentum_residual,boundary_speed_pre_correction,boundary_speed_post_correction,rho_min,rho_max,eta_min,"
          "eta_max,dt_limit_advective,dt_limit_capillary,dt_limit_ch_explicit,dt_limit_active,dt_limit_ratio,"
          "ch_iterations,coupling_iterations,pressure_iterations,momentum_iterations,"
          "ch_solver_name,momentum_solver_name,pressure_solver_name,dt_limit_source\n")


def test_header_is_the_references():
    assert capi.history_csv_header() == HEADER


@pytest.mark.gpu
@pytest.mark.parametrize("name,pname", [("walls_split_ildlt", "SplitILDLTPCG"), ("channel_x_icpcg", "ICCPCG"),
                                        ("dcdm_walls", "SplitDCDMICC"), ("advection_only_zalesak", "NotUsed")])
def test_rows_carry_the_step(name, pname):
    from test_gpu_parity import CASES

    cfg = CASES[name]
    s = capi.Solver(cfg)
    try:
        s.initialize()
        cols = HEADER.strip().split(",")
        for k in range(2):
            rep = s.step(k)
            row = s.history_csv_row(k + 1, (k + 1) * cfg["dt"], rep)
            assert row.endswith("\n")
            vals = dict(zip(cols, row.strip().split(",")))
            assert len(vals) == len(cols) and int(vals["step"]) == k + 1
            d = s.diagnostics()
            for key in ("mass", "kinetic_energy", "rho_min", "eta_max", "dt_limit_active"):
                assert float(vals[key]) == d[key] or (math.isinf(d[key]) and math.isinf(float(vals[key])))
            assert int(vals["pressure_iterations"]) == rep["pressure_iterations"]
            assert float(vals["pressure_correction_residual"]) == (0.0 if pname == "NotUsed" else
                                                                   rep["pressure_residual"])
            assert vals["pressure_solver_name"] == pname
            expect_ch = {1: "SparsePCG[ILDLT]", 0: "SparsePCG[Diagonal]", 2: "SparsePCG[DiagonalFallback]",
                         -1: "NotUsed"}[rep["ch_preconditioner"]]
            if cfg["mode"] == "advection_only":
                expect_ch = "PureAdvectionSSPRK3[WENO5]"
            assert vals["ch_solver_name"] == expect_ch
            limits = [d["dt_limit_advective"], d["dt_limit_capillary"], d["dt_limit_ch_explicit"]]
            src = ["advective", "capillary", "ch_explicit"][int(np.argmin(limits))]
            if not math.isfinite(min(limits)):
                src = "unbounded"
            assert vals["dt_limit_source"] == src
    finally:
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["walls_split_icpcg_wide", "channel_x_icpcg", "dcdm_walls"])
def test_pressure_monitor_matches_oracle(name):
    """The CG monitor's per-iteration record of the pressure solve (abs, rel, iterate residual, alpha) against
    the oracle's, on the same seeded step."""
    import ding_nsch_core_solver_b200 as dn
    from test_gpu_parity import CASES, seeded_pair

    orc, gpu = seeded_pair(dn, CASES[name], seed=9)
    try:
        orc.set_pressure_monitor(5000)
        gpu.set_pressure_monitor(5000)
        orc.step(0)
        rep = gpu.step(0)
        a, b = gpu.pressure_monitor(), orc.pressure_monitor()
        assert len(a) == rep["pressure_iterations"] == len(b) > 0
        # residuals differ only by the reduction order: compare where they are well above round-off
        keep = b[:, 1] > 1e-8
        np.testing.assert_allclose(a[keep, 1], b[keep, 1], rtol=1e-6)
        np.testing.assert_allclose(a[keep, 3], b[keep, 3], rtol=1e-6)
        np.testing.assert_allclose(a[keep, 0], b[keep, 0], rtol=1e-6)
    finally:
        gpu.close()
        orc.close()
