"""Captured steps (dn_set_step_graph) and the one-launch batch against eager steps.

A captured step records dn_step's work once into a CUDA graph: the mixed-precision solves' defect-correction
and inner CG loops become conditional graph nodes whose conditions kernels set from the same residual
checks, and every result stays on the device until one read-back after the replay.  The eager step's mixed
solves run the same recorded loops, each as its own graph.  So a solver whose steps are replayed must end
bitwise-identical to a twin stepped eagerly:
  * every field after every step;
  * every report field (iteration counts, residuals, refinement cycles, the inner solver, boundary speeds,
    the CH preconditioner);
  * across the pressure schemes (split and variable-density, ICC and ILDLT), both precisions, walls and
    periodic sides, the multigrid and IC inner solvers of the mixed form, and a grid without a hierarchy.
A replayed step counts the eager step's kernel launches plus its few record copies.  dn_step_batch over handles that all
replay captured steps is one graph launch per call.  It must equal each handle stepped alone.
"""
import numpy as np
import pytest

from ding_nsch_core_solver_b200 import capi
from test_gpu_parity import unit

pytestmark = pytest.mark.gpu

CASES = {
    "mixed_split_walls_mg": unit(nx=96, ny=64, periodic_x=False, periodic_y=False, pressure_scheme="split_icpcg",
                                 body_force_y=-0.98, dt=1e-4, precision="mixed"),
    "mixed_variable_periodic_x_mg": unit(nx=64, ny=48, periodic_x=True, periodic_y=False, pressure_scheme="icpcg",
                                         top_wall_velocity_x=0.5, bottom_wall_velocity_x=-0.5, dt=1e-4,
                                         precision="mixed"),
    "mixed_split_ic_inner": unit(nx=64, ny=64, periodic_x=False, periodic_y=False, pressure_scheme="split_icpcg",
                                 body_force_y=-0.98, dt=1e-4, precision="mixed", mixed_preconditioner="ic"),
    "mixed_no_hierarchy": unit(nx=130, ny=24, periodic_x=False, periodic_y=False, pressure_scheme="split_ildlt_pcg",
                               body_force_y=-0.98, dt=1e-4, precision="mixed"),
    "mixed_dirichlet_top": unit(nx=48, ny=64, periodic_x=False, periodic_y=False, pressure_scheme="icpcg", dt=1e-4,
                                pressure_bc_top_type="dirichlet", pressure_bc_top_value=0.3, precision="mixed"),
    "plain_split_walls": unit(nx=96, ny=48, periodic_x=False, periodic_y=False, pressure_scheme="split_icpcg",
                              body_force_y=-0.98, dt=1e-4),
    "plain_variable_ildlt": unit(nx=40, ny=56, periodic_x=False, periodic_y=False, pressure_scheme="ildlt_pcg",
                                 dt=1e-4, pressure_bc_top_type="dirichlet", pressure_bc_top_value=0.3),
    "plain_periodic_icpcg": unit(pressure_scheme="icpcg"),
}
STEPS = 6


def _seeded(cfg, seed, share=1):
    s = capi.Solver(dict(cfg, device_share=share))
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


def _assert_same(a, b, where):
    for name in capi.FIELDS:
        x, y = a.get_field(name), b.get_field(name)
        assert np.array_equal(x, y, equal_nan=True), (where, name, float(np.nanmax(np.abs(x - y))))


@pytest.mark.parametrize("name", sorted(CASES))
def test_replayed_steps_equal_eager_steps(name):
    cfg = CASES[name]
    eager, graph = _seeded(cfg, 7), _seeded(cfg, 7)
    graph.set_step_graph(True)
    try:
        for step in range(STEPS):
            le, lg = eager.kernel_launches(), graph.kernel_launches()
            re, rg = eager.step(step), graph.step(step)
            assert re == rg, (name, step, re, rg)
            _assert_same(eager, graph, f"{name} step {step}")
            # a replay counts the kernels its graph ran (nodes outside the loops, loop bodies times the
            # iterations the record reports): the eager step's kernels, plus from step 2 on the graph's record
            # kernels (one copy per persistent solve, the pressure factor's status, the CH breakdown check)
            extra = (graph.kernel_launches() - lg) - (eager.kernel_launches() - le)
            assert (extra == 0) if step < 2 else (1 <= extra <= 5), (name, step, extra)
        # the replayed steps ran the device loops: mixed solves report their cycles and inner iterations
        if cfg.get("precision") == "mixed":
            assert rg["refinement_cycles"] >= 1 and rg["pressure_iterations"] >= 1
    finally:
        eager.close()
        graph.close()


BATCH = ["mixed_split_walls_mg", "mixed_variable_periodic_x_mg", "mixed_split_ic_inner", "plain_split_walls"]


def test_one_launch_batch_equals_each_instance_alone():
    batch = [_seeded(CASES[n], 40 + k, share=len(BATCH)) for k, n in enumerate(BATCH)]
    alone = [_seeded(CASES[n], 40 + k, share=len(BATCH)) for k, n in enumerate(BATCH)]
    for s in batch:
        s.set_step_graph(True)
    try:
        for step in range(STEPS):
            reps = capi.step_batch(batch, [step] * len(batch))
            for k, s in enumerate(alone):
                rep = s.step(step)
                assert reps[k] == rep, (BATCH[k], step, reps[k], rep)
                _assert_same(batch[k], s, f"{BATCH[k]} step {step}")
    finally:
        for s in batch + alone:
            s.close()


@pytest.mark.parametrize("name", ["plain_split_walls", "plain_variable_ildlt", "mixed_split_walls_mg"])
def test_replayed_step_fails_like_the_eager_step(name):
    """A NaN planted in c once the steps are replayed: the replayed step returns the eager step's status and
    message.  In the plain form that is the CH PCG's breakdown after its retry with the diagonal
    preconditioner (phase_field.cpp:468-473), which the graph runs as a conditional branch on the device
    status; in the mixed form the first failing solve or the non-finite diagnostics (solver.cpp:355-364).
    Every loop of the graph ends on its own on a NaN (breakdown checks, the decisions' std::max semantics,
    the cycle and iteration caps)."""
    cfg = CASES[name]
    eager, graph = _seeded(cfg, 7), _seeded(cfg, 7)
    graph.set_step_graph(True)
    g = cfg["ghost"]
    try:
        for step in range(3):
            assert eager.step(step) == graph.step(step)
        for s in (eager, graph):
            f = s.get_field("c")
            f[g + 5, g + 5] = np.nan
            s.set_field("c", f)
        errors = []
        for s in (eager, graph):
            with pytest.raises(capi.DnError) as e:
                s.step(3)
            errors.append(e.value)
        assert errors[0].status == errors[1].status, (str(errors[0]), str(errors[1]))
        assert str(errors[0]) == str(errors[1])
    finally:
        eager.close()
        graph.close()
