"""The reference-side binding, built and run: a copy of the reference patched as INTEGRATION.md §2 describes.

oracle/patch_reference.py adds to a copy of the reference's coupled-solver directory a first `cuda_*` branch in
the pressure dispatcher (pressure.cpp:1031-1089) and a `cuda_sparse_pcg` branch in the CH dispatcher
(phase_field.cpp:437-503) that call dn_pressure_solve / dn_ch_linear_solve on a handle that
oracle/ref_cuda_binding.cpp builds from the solver's own Config; oracle/Makefile (target refcuda) compiles
it into oracle/_ref/libdnref_cuda.so.  Here that patched reference runs whole steps with
pressure_scheme = cuda_<scheme> and ch_solver = cuda_sparse_pcg, and must agree with the unpatched
reference on the same state: every field to rel-L2 <= 1e-10, the same iteration counts.
"""
import numpy as np
import pytest

from oracle.oracle import FIELDS, OracleSolver, available
from test_gpu_parity import interior, rel_l2, unit

TOL = 1.0e-10

CASES = {
    "split_icpcg_walls": unit(nx=48, ny=96, lx=1.0, ly=2.0, periodic_x=False, periodic_y=False,
                              pressure_scheme="split_icpcg", body_force_y=-0.98, dt=1e-4),
    "icpcg_channel_x": unit(nx=64, ny=32, periodic_x=True, periodic_y=False, pressure_scheme="icpcg",
                            top_wall_velocity_x=0.5, bottom_wall_velocity_x=-0.5, dt=1e-4),
    "ildlt_periodic": unit(nx=40, ny=40, pressure_scheme="ildlt_pcg", dt=1e-4),
}


def _require_builds():
    for impl in ("reference", "reference_cuda"):
        if not available(impl):
            pytest.skip(f"oracle/_ref build of {impl} absent (make -C oracle ref refcuda with DN_REFERENCE set)")


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_patched_reference_steps_through_the_library(name):
    _require_builds()
    cfg = CASES[name]
    ref = OracleSolver(cfg, "reference")
    pat = OracleSolver(cfg, "reference_cuda")
    ref.initialize()
    pat.initialize()
    rng = np.random.default_rng(3)
    g = cfg["ghost"]
    f = ref.field("c")
    f[g:-g, g:-g] += 0.02 * rng.standard_normal(f[g:-g, g:-g].shape)
    for fname, a in (("u", 0.05), ("v", 0.05), ("p", 0.1)):
        f = ref.field(fname)
        f[g:-g, g:-g] += a * rng.standard_normal(f[g:-g, g:-g].shape)
    ref.refresh_derived()
    for fname in FIELDS:
        pat.field(fname)[...] = ref.field(fname)
    ref.set_initial_mass(0.0)
    pat.set_initial_mass(0.0)
    for k in range(3):
        ref.step(k)
        pat.step(k)
        rr, rp = ref.report(), pat.report()
        for key in ("pressure_iterations", "ch_iterations", "momentum_iterations"):
            assert rr[key] == rp[key], (name, k, key, rr[key], rp[key])
        for fname in ("c", "mu", "u", "v", "p"):
            err = rel_l2(interior(pat.field(fname), g), interior(ref.field(fname), g))
            assert err <= TOL, (name, k, fname, err)
    ref.close()
    pat.close()
