"""Failure paths of the device step, tested without faulting, trapping or hanging a GPU.

* A device wait that runs out.  With device_wait_limit = 1 every bounded wait (grid barrier, wavefront
  hand-over) that is not satisfied at its first poll gives up: the kernel records a status word, every
  other wait sees it and ends, and the call returns DN_ERR_TIMEOUT.  The process's context stays usable: a
  new handle with the default limit steps the same state and matches the oracle.
* ICC construction failure.  A density field with negative values makes the variable pressure operator
  indefinite: the pressure backend returns DN_ERR_ICC_FAILED with the reference's message "ICC
  preconditioner construction failed" (try_build_incomplete_cholesky, ch_sparse_krylov.hpp:400-402;
  pressure.cpp:36-38), where the oracle fails with the same message.
* A non-finite state.  A NaN in c makes the CH PCG break down ("pcg preconditioner breakdown: non-positive
  r^T M^{-1} r", ch_sparse_krylov.hpp:566-568) after its diagonal retry (phase_field.cpp:468-473), as on the
  reference; and dn_diagnostics on that state reports DN_ERR_NONFINITE ("non-finite diagnostic detected",
  solver.cpp:355-364).
* Iteration exhaustion.  poisson_iterations = 3 stops the pressure PCG after 3 iterations without an
  error and reports the unconverged residual, as the reference does (ch_sparse_krylov.hpp:515-660).

The oracle here is the reference build (oracle/_ref) where it is present, else the C restatement, which
tests/test_oracle.py pins to the reference on these same failure paths.
"""
import numpy as np
import pytest

from ding_nsch_core_solver_b200 import capi
from oracle.oracle import FIELDS, OracleError, OracleSolver, available
from test_gpu_parity import COMPARE, assert_fields_close, seeded_pair, unit



DN_ERR_ICC_FAILED, DN_ERR_PCG_BREAKDOWN, DN_ERR_TIMEOUT, DN_ERR_NONFINITE = 4, 6, 8, 9
IMPL = "reference" if available("reference") else "port"


@pytest.fixture(scope="module")
def dn():
    import ding_nsch_core_solver_b200 as m

    m.load()
    return m


def walls(**kw):
    return unit(nx=96, ny=64, periodic_x=False, periodic_y=False, pressure_scheme="icpcg", dt=1e-4, **kw)


@pytest.mark.gpu
def test_device_wait_limit_times_out_and_context_survives(dn):
    cfg = walls()
    orc, gpu = seeded_pair(dn, cfg, seed=31)
    state = {n: gpu.get_field(n) for n in FIELDS}
    gpu.close()
    short = dn.Solver(dict(cfg, device_wait_limit=1))
    for n, a in state.items():
        short.set_field(n, a)
    with pytest.raises(capi.DnError) as e:
        short.step(0)
    assert e.value.status == DN_ERR_TIMEOUT, e.value
    short.close()
    # a fresh handle in the same process: the context still works and the step matches the oracle
    again = dn.Solver(cfg)
    for n, a in state.items():
        again.set_field(n, a)
    again.set_initial_mass(0.0)
    orc.step(0)
    rep = again.step(0)
    assert_fields_close(orc, again, COMPARE, "after a timed-out handle")
    assert rep["pressure_iterations"] == orc.report()["pressure_iterations"]
    again.close()


def _indefinite_inputs(cfg):
    nx, ny, g = cfg["nx"], cfg["ny"], cfg["ghost"]
    rng = np.random.default_rng(0)
    shp = lambda a, b: (a + 2 * g, b + 2 * g)
    rho_mid = np.ones(shp(nx, ny))
    rho_mid[g + 10:g + 20, g + 8:g + 16] = -2.0
    us = np.zeros(shp(nx + 1, ny))
    us[g:-g, g:-g] = 0.01 * rng.standard_normal(us[g:-g, g:-g].shape)
    vs = np.zeros(shp(nx, ny + 1))
    p = np.zeros(shp(nx, ny))
    return dict(u_star=us, v_star=vs, rho_mid=rho_mid, p=p, p_prev=p.copy())


@pytest.mark.gpu
def test_indefinite_pressure_operator_fails_icc_like_the_reference(dn):
    cfg = walls()
    arrs = _indefinite_inputs(cfg)
    orc = OracleSolver(cfg, IMPL)
    orc.initialize()
    for n, a in (("rho_mid", arrs["rho_mid"]), ("u_star", arrs["u_star"]), ("v_star", arrs["v_star"])):
        orc.set_field(n, a)
    with pytest.raises(OracleError) as oe:
        orc.pressure()
    gpu = dn.Solver(cfg)
    with pytest.raises(capi.DnError) as ge:
        gpu.pressure_solve(0, **arrs)
    assert ge.value.status == DN_ERR_ICC_FAILED, ge.value
    assert str(oe.value) in str(ge.value), (str(oe.value), str(ge.value))
    gpu.close()


@pytest.mark.gpu
def test_nan_state_breaks_down_like_the_reference_and_is_reported_nonfinite(dn):
    cfg = walls()
    g = cfg["ghost"]
    orc = OracleSolver(cfg, IMPL)
    orc.initialize()
    orc.field("c")[g + 5, g + 5] = np.nan
    gpu = dn.Solver(cfg)
    for n in FIELDS:
        gpu.set_field(n, orc.field(n))
    with pytest.raises(capi.DnError) as de:
        gpu.diagnostics()
    assert de.value.status == DN_ERR_NONFINITE and "non-finite diagnostic detected" in str(de.value)
    with pytest.raises(OracleError) as oe:
        orc.step(0)
    with pytest.raises(capi.DnError) as ge:
        gpu.step(0)
    assert ge.value.status == DN_ERR_PCG_BREAKDOWN, ge.value
    assert str(oe.value) in str(ge.value), (str(oe.value), str(ge.value))
    gpu.close()


@pytest.mark.gpu
def test_pressure_iteration_exhaustion_reports_like_the_reference(dn):
    cfg = walls(poisson_iterations=3)
    orc = OracleSolver(cfg, IMPL)
    orc.initialize()
    gpu = dn.Solver(cfg)
    for n in FIELDS:
        gpu.set_field(n, orc.field(n))
    gpu.set_initial_mass(0.0)
    orc.set_initial_mass(0.0)
    orc.step(0)
    rep = gpu.step(0)
    ro = orc.report()
    assert rep["pressure_iterations"] == ro["pressure_iterations"] == 3
    assert rep["pressure_residual"] > cfg["pressure_tolerance"]
    assert abs(rep["pressure_residual"] - ro["pressure_residual"]) <= 1e-9 * ro["pressure_residual"]
    assert_fields_close(orc, gpu, COMPARE, "3 pressure iterations")
    gpu.close()


def test_device_wait_limit_config_key():
    """Parsed on the host: no device needed."""
    assert capi.parse_config("device_wait_limit = 1000\n").device_wait_limit == 1000
    assert capi.parse_config("nx = 32\n").device_wait_limit == 0
    with pytest.raises(capi.DnError):
        capi.parse_config("device_wait_limit = -5\n")
