"""Gradients of a droplet's Taylor deformation after a coupled rollout, against central finite differences.

A droplet in a wall-driven shear channel (the shear-droplet family: periodic x, walls moving at +-0.5) is
rolled out by autograd.full_rollout -- whole coupled time steps (CH phase, materials, surface force,
momentum predictor, projection), each map with its hand-written adjoint -- with checkpointing every K
steps.  The loss is the second-moment Taylor deformation of c at the end (autograd.taylor_deformation,
python/postprocess_taylor_deformation.py:65-112), in its smooth variant (weights c, not c clamped to [0, 1]:
the clamp has a kink wherever c reaches 0 or 1, which the droplet's interior does to round-off, so finite
differences across it measure the kink, not the derivative).  Its gradients with respect to the surface-tension
multiplier sigma, the mobility 1/Pe (4-point differences, h = 1e-3) and a random direction of the initial c
(central, eps 1e-6) must match finite differences to 1e-6 relative, in the plain FP64 form and in the
mixed-precision form (whose solves, forward and transposed, end below the same tight tolerances).
"""
import numpy as np
import pytest
import torch

from test_adjoint_full_step import EPS_PARAM, TIGHT, _state, fd4
from test_gpu_parity import seeded_pair, unit

pytestmark = pytest.mark.gpu

STEPS, K = 6, 2


def _cfg(precision):
    # re = 10, ca = 0.1: surface tension strong enough that sigma moves the deformation within the horizon
    return unit(nx=40, ny=32, lx=1.25, ly=1.0, periodic_x=True, periodic_y=False, pressure_scheme="icpcg",
                dt=2e-4, top_wall_velocity_x=0.5, bottom_wall_velocity_x=-0.5, density_ratio=2.0,
                viscosity_ratio=2.0, interface_radius=0.25, interface_center_x=0.625, interface_center_y=0.5,
                re=10.0, ca=0.1, cn=0.04, pe=25.0, precision=precision, **TIGHT)


@pytest.fixture(scope="module")
def dn():
    import ding_nsch_core_solver_b200 as m

    m.load()
    return m


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_deformation_gradients_match_central_differences(dn, precision):
    from ding_nsch_core_solver_b200 import autograd as ag

    cfg = _cfg(precision)
    orc, gpu = seeded_pair(dn, cfg, seed=2, amp=0.0)
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
    d = torch.tensor(rng.standard_normal(tuple(st["c"].shape)) * 1e-2, device="cuda")
    eps = 1e-6
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
