"""The momentum predictor's hand-written adjoint (dn_momentum_adjoint) against central finite differences.

The map (u, v, H_prev, f, rho_mid, eta, eta_prev) -> (u*, v*, H) of the momentum predictor is quadratic in
(u, v) (centred convection) and linear in H_prev and f, so central differences in those are exact up to the
forward solve's tolerance (1e-14 absolute here); in the materials (which enter the solved operator) the
O(eps^2) term is below the bar at eps = 1e-4 with perturbations of relative size 1e-4.  For random directions d and cotangents w,
<w, J d> by central differences must equal <J^T w, d> from the adjoint to 1e-6 relative, on walls with
Dirichlet and Neumann velocity sides, a periodic-x shear channel and a doubly periodic box, on step 0 (the
convection term alone) and step 1 (AB2 with H_prev).  The composition with the projection
(autograd.velocity_step) is checked the same way, and the gradient with respect to the surface-tension
multiplier sigma through f = sigma * f_hat.
"""
import numpy as np
import pytest
import torch

from test_gpu_parity import seeded_pair, unit

pytestmark = pytest.mark.gpu

CASES = {
    "walls_bc_values": unit(nx=24, ny=20, periodic_x=False, periodic_y=False, pressure_scheme="icpcg", dt=1e-3,
                            u_bc_left_type="dirichlet", u_bc_left_value=0.1, u_bc_right_type="neumann",
                            u_bc_right_value=0.2, v_bc_bottom_type="dirichlet", v_bc_bottom_value=-0.1,
                            v_bc_top_type="neumann", v_bc_top_value=0.05),
    "shear_channel_x": unit(nx=28, ny=16, periodic_x=True, periodic_y=False, pressure_scheme="split_icpcg",
                            top_wall_velocity_x=0.5, bottom_wall_velocity_x=-0.5, dt=1e-3),
    "periodic_box": unit(nx=20, ny=24, pressure_scheme="icpcg", dt=1e-3),
}
TIGHT = dict(momentum_tolerance=1e-14, momentum_iterations=2000, pressure_tolerance=1e-12,
             poisson_iterations=20000)


@pytest.fixture(scope="module")
def dn():
    import ding_nsch_core_solver_b200 as m

    m.load()
    return m


def _setup(dn, name):
    cfg = dict(CASES[name], **TIGHT)
    orc, gpu = seeded_pair(dn, cfg, seed=21)
    g = cfg["ghost"]
    t = lambda a: torch.tensor(np.ascontiguousarray(a[g:a.shape[0] - g, g:a.shape[1] - g]), dtype=torch.float64,
                               device="cuda")
    rng = np.random.default_rng(5)
    state = {n: t(gpu.get_field(n)) for n in ("u", "v", "rho_mid", "eta", "eta_prev")}
    for n, like in (("hu_prev", "u"), ("hv_prev", "v"), ("fxu", "u"), ("fyv", "v")):
        state[n] = torch.tensor(0.3 * rng.standard_normal(tuple(state[like].shape)), device="cuda")
    return cfg, gpu, state, rng


def _dirs(state, rng):
    return {n: torch.tensor(rng.standard_normal(tuple(a.shape)), device="cuda") for n, a in state.items()}


ORDER = ("u", "v", "hu_prev", "hv_prev", "fxu", "fyv", "rho_mid", "eta", "eta_prev")
VEL = ORDER[:6]


@pytest.mark.parametrize("step", [0, 1])
@pytest.mark.parametrize("name", sorted(CASES))
def test_momentum_adjoint_matches_central_differences(dn, name, step):
    from ding_nsch_core_solver_b200 import autograd as ag

    cfg, gpu, state, rng = _setup(dn, name)
    w = {n: torch.tensor(rng.standard_normal(tuple(state[k].shape)), device="cuda")
         for n, k in (("u", "u"), ("v", "v"), ("hu", "u"), ("hv", "v"))}

    def loss(st):
        us, vs, hu, hv = ag.momentum_predictor(gpu, step, *(st[n] for n in ORDER))
        return (w["u"] * us).sum() + (w["v"] * vs).sum() + (w["hu"] * hu).sum() + (w["hv"] * hv).sum()

    x = {n: a.clone().requires_grad_(True) for n, a in state.items()}
    grads = torch.autograd.grad(loss(x), [x[n] for n in ORDER])
    for trial in range(3):
        d = _dirs(state, rng)
        adj = sum(float((gr * d[n]).sum()) for gr, n in zip(grads, ORDER))
        eps = 1e-4
        with torch.no_grad():
            lp = float(loss({n: state[n] + eps * d[n] for n in ORDER}))
            lm = float(loss({n: state[n] - eps * d[n] for n in ORDER}))
        fd = (lp - lm) / (2 * eps)
        print(name, step, trial, f"fd {fd:.12e} adjoint {adj:.12e}")
        assert abs(fd - adj) <= 1e-6 * max(abs(fd), 1e-3), (name, step, trial, fd, adj)
    gpu.close()


@pytest.mark.parametrize("name", ["walls_bc_values", "shear_channel_x"])
def test_velocity_step_and_sigma_gradient(dn, name):
    """The predictor composed with the projection (rho_mid fixed), and d/d sigma of the same loss through
    f = sigma * f_hat."""
    from ding_nsch_core_solver_b200 import autograd as ag

    cfg, gpu, state, rng = _setup(dn, name)
    g = cfg["ghost"]
    p = torch.tensor(np.ascontiguousarray(gpu.get_field("p")[g:-g, g:-g]), device="cuda")
    pp = p.clone()
    w = {n: torch.tensor(rng.standard_normal(tuple(state[k].shape)), device="cuda") for n, k in (("u", "u"), ("v", "v"))}

    def loss(st, sigma):
        args = [st["u"], st["v"], st["hu_prev"], st["hv_prev"], sigma * st["fxu"], sigma * st["fyv"], p, pp]
        un, vn, _, _ = ag.velocity_step(gpu, 1, *args)
        return (w["u"] * un).sum() + (w["v"] * vn).sum()

    x = {n: a.clone().requires_grad_(True) for n, a in state.items()}
    sigma = torch.tensor(1.3, dtype=torch.float64, device="cuda", requires_grad=True)
    out = loss(x, sigma)
    grads = torch.autograd.grad(out, [x[n] for n in VEL] + [sigma])
    d = _dirs(state, rng)
    adj = sum(float((gr * d[n]).sum()) for gr, n in zip(grads[:-1], VEL))
    eps = 1e-4
    with torch.no_grad():
        s0 = torch.tensor(1.3, dtype=torch.float64, device="cuda")
        fd = (float(loss({n: state[n] + eps * d[n] for n in VEL}, s0)) -
              float(loss({n: state[n] - eps * d[n] for n in VEL}, s0))) / (2 * eps)
        fd_s = (float(loss(state, s0 + eps)) - float(loss(state, s0 - eps))) / (2 * eps)
    print(name, f"state fd {fd:.12e} adjoint {adj:.12e}; sigma fd {fd_s:.12e} adjoint {float(grads[-1]):.12e}")
    assert abs(fd - adj) <= 1e-6 * max(abs(fd), 1e-3), (fd, adj)
    assert abs(fd_s - float(grads[-1])) <= 1e-6 * max(abs(fd_s), 1e-3), (fd_s, float(grads[-1]))
    gpu.close()
