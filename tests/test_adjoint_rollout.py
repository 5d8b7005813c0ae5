"""Gradients of a droplet's Taylor deformation after a coupled rollout, against central finite differences.

An elliptical droplet (semi-axes 1.3 R and 0.77 R, the reference's tanh profile across an ellipse, so that
surface tension drives a real relaxation within the horizon) in a wall-driven shear channel (the
shear-droplet family: periodic x, walls moving at +-0.5) is rolled out by autograd.full_rollout -- whole coupled time steps (CH phase, materials, surface force,
momentum predictor, projection), each map with its hand-written adjoint -- with checkpointing every K
steps.  The loss is the second-moment Taylor deformation of c at the end (autograd.taylor_deformation,
python/postprocess_taylor_deformation.py:65-112), in its smooth variant (weights c, not c clamped to [0, 1]:
the clamp has a kink wherever c reaches 0 or 1, which the droplet's interior does to round-off, so finite
differences across it measure the kink, not the derivative).  Its gradients with respect to the surface-tension
multiplier sigma, the mobility 1/Pe (4-point differences, h = 1e-3) and a random direction of the initial c
(central, 1e-7 per cell) must match finite differences to 1e-6 relative, in the plain FP64 form and in the
mixed-precision form (whose solves, forward and transposed, end below the same tight tolerances).
"""
import numpy as np
import pytest
import torch

from test_adjoint_full_step import EPS_PARAM, TIGHT, _state, fd4
from test_gpu_parity import unit

pytestmark = pytest.mark.gpu

STEPS, K = 6, 2


def _cfg(precision):
    # re = 10, ca = 0.1, dt = 1e-3 (max |u| about 0.5): the ellipse relaxes by surface tension within the
    # horizon, dD/dsigma about 1.5e-4, far above the solves' noise on D (about 1e-15)
    return unit(nx=40, ny=32, lx=1.25, ly=1.0, periodic_x=True, periodic_y=False, pressure_scheme="icpcg",
                dt=1e-3, top_wall_velocity_x=0.5, bottom_wall_velocity_x=-0.5, density_ratio=2.0,
                viscosity_ratio=2.0, interface_radius=0.25, interface_center_x=0.625, interface_center_y=0.5,
                re=10.0, ca=0.1, cn=0.04, pe=25.0, precision=precision, **TIGHT)


def _ellipse_solver(dn, cfg, stretch=1.3):
    """A GPU solver holding the reference's tanh profile across an ellipse of area pi R^2, at rest."""
    from ding_nsch_core_solver_b200.capi import FIELDS
    from oracle.oracle import OracleSolver

    orc = OracleSolver(cfg, "port")
    orc.initialize()
    g, nx, ny = cfg["ghost"], cfg["nx"], cfg["ny"]
    dx, dy = cfg["lx"] / nx, cfg["ly"] / ny
    x = (np.arange(nx) + 0.5) * dx - cfg["interface_center_x"]
    y = (np.arange(ny) + 0.5) * dy - cfg["interface_center_y"]
    r = np.sqrt((x[:, None] / stretch) ** 2 + (y[None, :] * stretch) ** 2)
    c = 0.5 - 0.5 * np.tanh((r - cfg["interface_radius"]) / (2.0 * np.sqrt(2.0) * cfg["cn"]))
    for name in ("c", "c_prev"):
        orc.field(name)[g:-g, g:-g] = c
    orc.refresh_derived()
    gpu = dn.Solver(cfg)
    for name in FIELDS:
        gpu.set_field(name, orc.field(name))
    gpu.set_initial_mass(0.0)
    orc.close()
    return gpu


@pytest.fixture(scope="module")
def dn():
    import ding_nsch_core_solver_b200 as m

    m.load()
    return m


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_deformation_gradients_match_central_differences(dn, precision):
    from ding_nsch_core_solver_b200 import autograd as ag

    cfg = _cfg(precision)
    gpu = _ellipse_solver(dn, cfg)
    gpu.step(0)  # one step of history (BDF2 and AB2 from here on)
    st = _state(gpu, cfg)
    dx, dy = cfg["lx"] / cfg["nx"], cfg["ly"] / cfg["ny"]
    rng = np.random.default_rng(4)

    def loss(solver, state, sigma=None, mob=None, ckpt=K):
        out = ag.full_rollout(solver, state, 1, STEPS, checkpoint_every=ckpt, sigma_scale=sigma, inv_pe_scale=mob)
        return ag.taylor_deformation(out["c"], dx, dy, clamp=False)

    x = {k: a.clone().requires_grad_(k == "c") for k, a in st.items()}
    sig = torch.tensor(1.0, dtype=torch.float64, device="cuda", requires_grad=True)
    mob = torch.tensor(1.0, dtype=torch.float64, device="cuda", requires_grad=True)
    D = loss(gpu, x, sig, mob)
    g_c, g_s, g_m = torch.autograd.grad(D, [x["c"], sig, mob])
    # checkpointing recomputes the forward (its CH solves start from the handle's current iterate, so the
    # recomputed states agree to the solves' tolerance, not bitwise): the gradient equals the one kept in full
    x0 = {k: a.clone().requires_grad_(k == "c") for k, a in st.items()}
    g_full, = torch.autograd.grad(loss(gpu, x0, sig.detach(), mob.detach(), ckpt=0), [x0["c"]])
    assert float((g_full - g_c).norm()) <= 1e-12 * float(g_c.norm())
    d = torch.tensor(rng.standard_normal(tuple(st["c"].shape)) * 1e-2, device="cuda")
    # 1e-7 per cell: the central difference's O(eps^2) error, from WENO5's nonlinear weights, is 4e-9
    # relative here (7e-7 at 1e-6 per cell, 6e-5 at 1e-5), the solves' noise about 5e-8
    eps = 1e-5
    one = lambda v: torch.tensor(v, dtype=torch.float64, device="cuda")
    with torch.no_grad():
        fd_c = (float(loss(gpu, dict(st, c=st["c"] + eps * d), ckpt=0)) -
                float(loss(gpu, dict(st, c=st["c"] - eps * d), ckpt=0))) / (2 * eps)
        fd_s = fd4(lambda h: float(loss(gpu, st, sigma=one(1 + h), ckpt=0)), EPS_PARAM)

    def with_pe(h):
        s2 = dn.Solver(dict(cfg, pe=cfg["pe"] / (1.0 + h)))
        s2.set_initial_mass(0.0)
        with torch.no_grad():
            val = float(loss(s2, st, ckpt=0))
        s2.close()
        return val

    fd_m = fd4(with_pe, EPS_PARAM)
    res = {"c0": (fd_c, float((g_c * d).sum())), "sigma": (fd_s, float(g_s)), "mobility": (fd_m, float(g_m))}
    print(precision, f"D = {float(D):.6e}", {k: (f"{a:.10e}", f"{b:.10e}") for k, (a, b) in res.items()})
    for k, (a, b) in res.items():
        assert abs(a - b) <= 1e-6 * max(abs(a), 1e-12), (precision, k, a, b)
    gpu.close()
