"""dn_pressure_solve_static: the allocation-free pressure solve against the handle's dn_pressure_solve.

The static entry point takes the caller's device buffers and stream and keeps its intermediates in a
fixed device array.  Each case runs two calls in a row on both entry points with different inputs (the
second call sees the array the first one left behind) and compares p_corr and the iteration count.  The
file is named to be collected last, so the check also runs after every other test has used the library.
"""
import ctypes as C

import numpy as np
import pytest

from ding_nsch_core_solver_b200 import capi

TOL = 1e-12  # relative L2: both entry points launch the same kernels with the same shapes

BASE = dict(nx=64, ny=128, lx=1.0, ly=2.0, dt=1e-3, density_ratio=10.0, viscosity_ratio=10.0,
            poisson_iterations=2000, pressure_tolerance=1e-10, periodic_x=False, periodic_y=False)
CASES = {
    # constant split operator, pure Neumann pressure (mean projection), staged wavefront
    "split_icpcg_walls": dict(BASE, pressure_scheme="split_icpcg"),
    # variable operator, a Dirichlet side (no projection), staged wavefront with ILDLT
    "ildlt_dirichlet_top": dict(BASE, nx=96, ny=64, pressure_scheme="ildlt_pcg",
                                pressure_bc_top_type="dirichlet", pressure_bc_top_value=0.25),
    # periodic x: the global-memory wavefront kernel
    "icpcg_periodic_x": dict(BASE, pressure_scheme="icpcg", periodic_x=True),
    # a handle sharing the device (device_share = 2) launches on half the SMs; so does the static call
    "split_icpcg_shared_device": dict(BASE, pressure_scheme="split_icpcg", device_share=2),
}


def _bind():
    lib = capi.load()
    fn = lib.dn_pressure_solve_static
    DP = C.c_void_p
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(capi.Config), C.c_int, DP, DP, DP, DP, DP, DP, C.c_void_p, C.POINTER(C.c_int),
                   C.POINTER(C.c_double), C.c_char_p, C.c_size_t]
    return fn


def _smooth(rng, shape, lo, hi):
    """A few random Fourier modes scaled into [lo, hi]."""
    i = np.arange(shape[0])[:, None] / shape[0]
    j = np.arange(shape[1])[None, :] / shape[1]
    f = np.zeros(shape)
    for _ in range(4):
        a, b = rng.integers(1, 5, size=2)
        f += rng.standard_normal() * np.sin(2 * np.pi * (a * i + rng.random())) * np.cos(2 * np.pi * (b * j + rng.random()))
    f = (f - f.min()) / max(f.max() - f.min(), 1e-300)
    return lo + (hi - lo) * f


def _inputs(cfg: capi.Config, seed: int):
    nx, ny, g = cfg.nx, cfg.ny, cfg.ghost
    rng = np.random.default_rng(seed)
    shp = lambda a, b: (a + 2 * g, b + 2 * g)
    return dict(u_star=_smooth(rng, shp(nx + 1, ny), -0.5, 0.5), v_star=_smooth(rng, shp(nx, ny + 1), -0.5, 0.5),
                rho_mid=_smooth(rng, shp(nx, ny), 1.0, 10.0), p=_smooth(rng, shp(nx, ny), -1.0, 1.0),
                p_prev=_smooth(rng, shp(nx, ny), -1.0, 1.0))


def _static_solve(fn, cfg, step, arrs, torch):
    dev = {k: torch.from_numpy(v).cuda() for k, v in arrs.items()}
    out = torch.full(arrs["p"].shape, float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    its, rel = C.c_int(), C.c_double()
    err = C.create_string_buffer(512)
    stream = torch.cuda.current_stream().cuda_stream
    st = fn(C.byref(cfg), int(step), *[dev[k].data_ptr() for k in ("u_star", "v_star", "rho_mid", "p", "p_prev")],
            out.data_ptr(), stream, C.byref(its), C.byref(rel), err, len(err))
    assert st == 0, (st, err.value.decode())
    return out.cpu().numpy(), its.value, rel.value


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_static_matches_handle_two_calls(name):
    import torch

    fn = _bind()
    solver = capi.Solver(CASES[name])
    cfg = solver.config
    try:
        for call, (step, seed) in enumerate(((0, 11), (1, 12))):
            arrs = _inputs(cfg, seed + 100 * len(name))
            ref, its_ref, rel_ref = solver.pressure_solve(step, **arrs)
            got, its, rel = _static_solve(fn, cfg, step, arrs, torch)
            assert np.all(np.isfinite(got)), (name, call)
            assert its == its_ref, (name, call, its, its_ref)
            assert _rel_l2(got, ref) < TOL, (name, call, _rel_l2(got, ref))
            assert abs(rel - rel_ref) <= 1e-12 * max(abs(rel_ref), 1e-300) + 1e-300
    finally:
        solver.close()


def test_static_rejects_grids_beyond_the_array():
    """The size check runs before any CUDA call, so it holds without a device too."""
    fn = _bind()
    cfg = capi.parse_config(dict(BASE, nx=512, ny=512, pressure_scheme="icpcg"))
    dummy = C.c_void_p(16)
    err = C.create_string_buffer(512)
    st = fn(C.byref(cfg), 0, dummy, dummy, dummy, dummy, dummy, dummy, None, None, None, err, len(err))
    assert st == 10, st
    msg = err.value.decode()
    assert "static scratch array holds" in msg and str(16 * 1024 * 1024) in msg, msg
