"""Launch shapes of the pressure PCG and their autotuner (dn_autotune_pressure).

A launch shape (rows per CTA of the SpMV / update phases, sweep warps per CTA of the staged wavefront)
changes only how the grid-wide sums are split over CTAs, so every shape must keep the step within the
plain-form parity bar of the oracle (relative L2 <= 1e-10).  The iteration counts may then differ by one
from the oracle's when the last residual lands next to the tolerance.  The autotuner must apply exactly the
shape it reports: a handle tuned to a shape and a handle created with that shape in its config step bitwise
alike from the same state.
"""
import numpy as np
import pytest

from ding_nsch_core_solver_b200 import capi
from test_gpu_parity import COMPARE, assert_fields_close, seeded_pair, unit

WALLS = unit(nx=96, ny=48, periodic_x=False, periodic_y=False, pressure_scheme="split_icpcg", body_force_y=-0.98,
             dt=1e-4)
CHANNEL_X = unit(nx=64, ny=32, periodic_x=True, periodic_y=False, pressure_scheme="icpcg", top_wall_velocity_x=0.5,
                 bottom_wall_velocity_x=-0.5, dt=1e-4)


@pytest.fixture(scope="module")
def dn():
    import ding_nsch_core_solver_b200 as m

    m.load()
    return m


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", [WALLS, CHANNEL_X], ids=["walls_split_icpcg", "channel_x_icpcg"])
@pytest.mark.parametrize("shape", [(256, 1), (4096, 2), (1024, 4)])
def test_launch_shape_keeps_parity(dn, cfg, shape):
    rows, sw = shape
    orc, gpu = seeded_pair(dn, dict(cfg, pcg_rows_per_cta=rows, sweep_warps_per_cta=sw), seed=23)
    try:
        for k in range(2):
            orc.step(k)
            rep = gpu.step(k)
            assert_fields_close(orc, gpu, COMPARE, f"shape {shape} step {k}")
            assert abs(rep["pressure_iterations"] - orc.report()["pressure_iterations"]) <= 1
    finally:
        gpu.close()
        orc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", [WALLS, CHANNEL_X], ids=["walls_split_icpcg", "channel_x_icpcg"])
def test_autotune_applies_the_reported_shape(dn, cfg):
    orc, tuned = seeded_pair(dn, cfg, seed=29)
    twin = None
    try:
        tuned.step(0)
        orc.step(0)
        shape = tuned.autotune_pressure()
        assert shape["pcg_rows_per_cta"] in (256, 512, 1024, 2048, 4096)
        assert 0 <= shape["sweep_warps_per_cta"] <= 4
        assert 0.0 < shape["pressure_ms"] < 1.0e4
        # the tuned handle keeps parity with the oracle
        tuned.step(1)
        orc.step(1)
        assert_fields_close(orc, tuned, COMPARE, "step after autotuning")
        # a handle created with the reported shape steps bitwise like the tuned one from the same state
        twin = dn.Solver(dict(cfg, pcg_rows_per_cta=shape["pcg_rows_per_cta"],
                              sweep_warps_per_cta=max(1, shape["sweep_warps_per_cta"])))
        for name in capi.FIELDS:
            twin.set_field(name, tuned.get_field(name))
        twin.set_initial_mass(0.0)
        for k in (2, 3):
            ra, rb = tuned.step(k), twin.step(k)
            assert ra["pressure_iterations"] == rb["pressure_iterations"]
            for name in capi.FIELDS:
                assert np.array_equal(tuned.get_field(name), twin.get_field(name), equal_nan=True), (k, name)
    finally:
        for s in (tuned, twin):
            if s is not None:
                s.close()
        orc.close()


def test_launch_shape_config_keys():
    """Parsed on the host: no device needed."""
    c = capi.parse_config("pcg_rows_per_cta = 2048\nsweep_warps_per_cta = 2\n")
    assert c.pcg_rows_per_cta == 2048 and c.sweep_warps_per_cta == 2
    d = capi.parse_config("nx = 32\n")
    assert d.pcg_rows_per_cta == 0 and d.sweep_warps_per_cta == 0
    with pytest.raises(capi.DnError):
        capi.parse_config("pcg_rows_per_cta = -1\n")
