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


def _cfg(precision, dt=1e-3):
    # re = 10, ca = 0.1, dt = 1e-3 (max |u| about 0.5): the ellipse relaxes by surface tension within the
    # 6-step horizon, dD/dsigma about 1.1e-4, far above the solves' noise on D (about 1e-15).  That step is
    # 4.3x the reference's explicit CH limit (2.3e-4 here, diagnostics.cpp:48-112): the state stays smooth
    # for these 6 steps (the reference itself departs after about 25), and a gradient check needs the
    # discrete map, not a long stable run.  The 500-step test runs at half the limit, dt = 1e-4.
    return unit(nx=40, ny=32, lx=1.25, ly=1.0, periodic_x=True, periodic_y=False, pressure_scheme="icpcg",
                dt=dt, top_wall_velocity_x=0.5, bottom_wall_velocity_x=-0.5, density_ratio=2.0,
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


# ---- the long horizon: 500 coupled steps, checkpoints every 50, 16 directions
LONG, K_LONG, NDIR = 500, 50, 16
# 4-point differences along d at 1e-6 per cell: O(eps^4) truncation, noise about 1e-8 relative; a larger
# step (1e-5 per cell) reaches across the mobility's kink at c = 0 for some directions (2.7e-6 off)
EPS_C = 1e-4


def _fd_rollouts(dn, cfg, base, steps):
    """D after `steps` dn_steps (captured steps, each one graph launch) from the ghosted fields `base`
    with c's interior replaced: the forward map full_rollout differentiates, solved to the same tight
    tolerances (the two agree to the solves' tolerance, test_composed_step_equals_dn_step)."""
    from ding_nsch_core_solver_b200.capi import FIELDS
    from ding_nsch_core_solver_b200 import autograd as ag

    g = cfg["ghost"]
    dx, dy = cfg["lx"] / cfg["nx"], cfg["ly"] / cfg["ny"]
    s = dn.Solver(cfg)
    s.set_step_graph(True)

    def run(c_interior):
        for n in FIELDS:
            s.set_field(n, base[n])
        f = base["c"].copy()
        f[g:-g, g:-g] = c_interior
        s.set_field("c", f)
        s.refresh_derived()
        s.set_initial_mass(0.0)
        for k in range(1, steps + 1):
            s.step(k)
        c = s.get_field("c")[g:-g, g:-g]
        return float(ag.taylor_deformation(torch.tensor(np.ascontiguousarray(c), device="cuda"), dx, dy, clamp=False))

    return s, run


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_long_horizon_gradients_match_finite_differences(dn, precision):
    """500 coupled steps at dt = 1e-5 (t = 5e-3), the adjoint through full_rollout with checkpoints every 50
    steps; 16 random directions of the initial c, and sigma and 1/Pe, each against 4-point finite differences
    of the rolled-out deformation, to 1e-6 relative.

    The step is a tenth of the one the 6-step test uses, for the discrete map's sake: at dt = 1e-4 (half the
    reference's explicit CH limit of 2.3e-4) the reference's map c0 -> D stops being smooth after 20-30
    steps.  Central differences no longer converge as eps shrinks (at 50 steps: 2.1, 12.6, 75, 485, 2303 for
    eps = 1e-4 .. 1e-8 per unit direction), with or without shear.  The explicit CH term then grows grid-scale
    perturbations by about 1.4-1.7 per step in the far field, where the degenerate mobility
    max(0, c (1 - c)) switches on and off as c crosses 0 (phase_field.cpp); the nonlinear map saturates
    them, so the forward stays bounded.  Where differences converge (20 steps at dt = 1e-4: 2.870843e-4 at
    eps = 1e-6 against the adjoint's 2.870839e-4; 500 steps at dt = 1e-5 or 4e-6 at every eps from 1e-3 to
    1e-8), they converge to the adjoint."""
    from ding_nsch_core_solver_b200.capi import FIELDS
    from ding_nsch_core_solver_b200 import autograd as ag

    cfg = _cfg(precision, dt=1e-5)
    gpu = _ellipse_solver(dn, cfg)
    gpu.step(0)
    base = {n: gpu.get_field(n) for n in FIELDS}
    st = _state(gpu, cfg)
    dx, dy = cfg["lx"] / cfg["nx"], cfg["ly"] / cfg["ny"]
    x = {k: a.clone().requires_grad_(k == "c") for k, a in st.items()}
    sig = torch.tensor(1.0, dtype=torch.float64, device="cuda", requires_grad=True)
    mob = torch.tensor(1.0, dtype=torch.float64, device="cuda", requires_grad=True)
    out = ag.full_rollout(gpu, x, 1, LONG, checkpoint_every=K_LONG, sigma_scale=sig, inv_pe_scale=mob)
    D = ag.taylor_deformation(out["c"], dx, dy, clamp=False)
    g_c, g_s, g_m = torch.autograd.grad(D, [x["c"], sig, mob])
    gpu.close()

    fd_solver, run = _fd_rollouts(dn, cfg, base, LONG)
    c0 = st["c"].cpu().numpy()
    D0 = run(c0)
    # the two forwards agree to the solves' tolerance accumulated over the horizon
    assert abs(D0 - float(D)) <= 1e-7 * abs(D0), (D0, float(D))
    rng = np.random.default_rng(12)
    worst = 0.0
    for k in range(NDIR):
        d = rng.standard_normal(c0.shape) * 1e-2
        fd = fd4(lambda h: run(c0 + h * d), EPS_C)
        ad = float((g_c * torch.tensor(d, device="cuda")).sum())
        worst = max(worst, abs(fd - ad) / abs(fd))
        assert abs(fd - ad) <= 1e-6 * abs(fd), (precision, k, fd, ad)
    fd_solver.close()

    def with_cfg(c2):
        s2, run2 = _fd_rollouts(dn, c2, base, LONG)
        val = run2(c0)
        s2.close()
        return val

    fd_s = fd4(lambda h: with_cfg(dict(cfg, surface_tension_multiplier=cfg["surface_tension_multiplier"] * (1 + h))),
               EPS_PARAM)
    fd_m = fd4(lambda h: with_cfg(dict(cfg, pe=cfg["pe"] / (1 + h))), EPS_PARAM)
    print(precision, f"D = {D0:.6e}", f"c0 worst {worst:.2e} over {NDIR}",
          f"sigma fd {fd_s:.10e} adjoint {float(g_s):.10e}", f"mobility fd {fd_m:.10e} adjoint {float(g_m):.10e}")
    assert abs(fd_s - float(g_s)) <= 1e-6 * abs(fd_s), (precision, fd_s, float(g_s))
    assert abs(fd_m - float(g_m)) <= 1e-6 * abs(fd_m), (precision, fd_m, float(g_m))
