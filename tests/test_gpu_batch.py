"""dn_step_batch: several handles advanced concurrently, each on its own stream from its own host worker.

Every handle must end bitwise-identical to a twin handle stepped alone with dn_step: the batch shares the
device, never data, and each solve is deterministic (fixed reduction order, fixed wavefront hand-over).
The instances differ in size, boundaries, pressure scheme and precision, so their kernels overlap with
different grid shapes.
"""
import ctypes as C

import numpy as np
import pytest

from ding_nsch_core_solver_b200 import capi
from test_gpu_parity import unit

ENSEMBLE = [
    unit(nx=96, ny=48, periodic_x=False, periodic_y=False, pressure_scheme="split_icpcg", body_force_y=-0.98,
         dt=1e-4),
    unit(nx=40, ny=56, periodic_x=False, periodic_y=False, pressure_scheme="ildlt_pcg", dt=1e-4,
         pressure_bc_top_type="dirichlet", pressure_bc_top_value=0.3),
    unit(nx=48, ny=32, periodic_x=True, periodic_y=False, pressure_scheme="icpcg", top_wall_velocity_x=0.5,
         bottom_wall_velocity_x=-0.5, dt=1e-4),
    unit(pressure_scheme="split_ildlt_pcg"),
    unit(nx=64, ny=64, periodic_x=False, periodic_y=False, pressure_scheme="split_icpcg", body_force_y=-0.98,
         dt=1e-4, precision="mixed"),
    unit(nx=32, ny=40, periodic_x=False, periodic_y=True, pressure_scheme="split_icpcg", dt=1e-4),
]


def _seeded(cfg, seed):
    """A solver at its initial state plus seeded noise on c, u, v and p (derived fields rebuilt).  Each
    handle's persistent launches take 1/len(ENSEMBLE) of the SMs, so the instances fit side by side."""
    s = capi.Solver(dict(cfg, device_share=len(ENSEMBLE)))
    s.initialize()
    rng = np.random.default_rng(seed)
    g = cfg["ghost"]
    for name, a in (("c", 0.02), ("u", 0.05), ("v", 0.05), ("p", 0.1)):
        f = s.get_field(name)
        f[g:-g, g:-g] += a * rng.standard_normal(f[g:-g, g:-g].shape)
        s.set_field(name, f)
    s.set_initial_mass(0.0)
    s.refresh_derived()
    return s


@pytest.mark.gpu
def test_batch_equals_each_instance_alone():
    batch = [_seeded(cfg, 100 + k) for k, cfg in enumerate(ENSEMBLE)]
    alone = [_seeded(cfg, 100 + k) for k, cfg in enumerate(ENSEMBLE)]
    try:
        for step in range(3):
            reps = capi.step_batch(batch, [step] * len(batch))
            for k, s in enumerate(alone):
                rep = s.step(step)
                assert reps[k] == rep, (k, step, reps[k], rep)
            for k in range(len(batch)):
                for name in capi.FIELDS:
                    a, b = batch[k].get_field(name), alone[k].get_field(name)
                    assert np.array_equal(a, b, equal_nan=True), (k, step, name)
    finally:
        for s in batch + alone:
            s.close()


@pytest.mark.gpu
def test_batch_rejects_a_repeated_handle():
    s = _seeded(ENSEMBLE[3], 7)
    try:
        with pytest.raises(capi.DnError) as e:
            capi.step_batch([s, s], [0, 0])
        assert e.value.status == 1
    finally:
        s.close()


def test_batch_argument_checks_without_device():
    """Argument checks run before any CUDA call."""
    lib = capi.load()
    assert lib.dn_step_batch(None, 2, None, None) == 1
    hs = (C.c_void_p * 2)(None, None)
    assert lib.dn_step_batch(hs, 2, None, None) == 1
    assert lib.dn_step_batch(hs, -1, None, None) == 1
    assert lib.dn_step_batch(hs, 0, None, None) == 0
