"""The hand-written adjoint of the whole time step (autograd.full_step) against the step itself and against
central finite differences.

full_step composes the differentiable maps of one step -- CH explicit operator and implicit solve, materials
and rho_mid, surface force, momentum predictor, projection with rho_mid -- each with its hand-written
vector-Jacobian product (dn_explicit_operator_adjoint, the CH solve, dn_surface_force_adjoint,
dn_momentum_adjoint, dn_projection_rho_adjoint).  Checked here:

* forward: the composition equals dn_step from the same state (c, u, v, p to 1e-9; the only difference is
  the CH solve's starting iterate, both converged to 1e-13);
* backward: for a loss over the state after two steps, <grad, d> equals finite differences to 1e-6 relative
  for random directions in the initial c, u, v, p (central, eps 1e-6), in the surface-tension multiplier
  sigma and in the mobility 1/Pe (4-point, h = 1e-3; the mobility through solvers built with Pe / (1 + h)).
"""
import numpy as np
import pytest
import torch

from ding_nsch_core_solver_b200.capi import FIELDS
from test_gpu_parity import seeded_pair, unit

pytestmark = pytest.mark.gpu

TIGHT = dict(pressure_tolerance=1e-13, poisson_iterations=50000, ch_tolerance=1e-13, ch_inner_iterations=20000,
             momentum_tolerance=1e-14, momentum_iterations=2000)
CASES = {
    # a shear channel with moving walls (the shear-droplet family), variable-density icpcg
    "shear_icpcg": unit(nx=32, ny=24, periodic_x=True, periodic_y=False, pressure_scheme="icpcg", dt=2e-4,
                        top_wall_velocity_x=0.5, bottom_wall_velocity_x=-0.5, density_ratio=5.0,
                        viscosity_ratio=3.0, **TIGHT),
    # walls and the split scheme with its explicit rho_mid term
    "walls_split": unit(nx=24, ny=32, periodic_x=False, periodic_y=False, pressure_scheme="split_icpcg", dt=2e-4,
                        body_force_y=-0.98, **TIGHT),
}
STATE = ("c", "c_old", "e_prev", "u", "v", "p", "p_prev", "hu_prev", "hv_prev")
FIELD = {"c": "c", "c_old": "c_prev", "e_prev": "e_prev", "u": "u", "v": "v", "p": "p", "p_prev": "p_prev",
         "hu_prev": "hu_prev", "hv_prev": "hv_prev"}


@pytest.fixture(scope="module")
def dn():
    import ding_nsch_core_solver_b200 as m

    m.load()
    return m


def _state(gpu, cfg):
    g = cfg["ghost"]
    out = {}
    for k, n in FIELD.items():
        a = gpu.get_field(n)
        out[k] = torch.tensor(np.ascontiguousarray(a[g:a.shape[0] - g, g:a.shape[1] - g]), dtype=torch.float64,
                              device="cuda")
    return out


def _pair(dn, name):
    cfg = CASES[name]
    orc, gpu = seeded_pair(dn, cfg, seed=9, amp=0.01)
    # a history consistent with one step already taken: run one step, then read the state
    gpu.step(0)
    return cfg, gpu


@pytest.mark.parametrize("name", sorted(CASES))
def test_composed_step_equals_dn_step(dn, name):
    from ding_nsch_core_solver_b200 import autograd as ag

    cfg, gpu = _pair(dn, name)
    st = _state(gpu, cfg)
    ref = dn.Solver(cfg)  # the same state, stepped by dn_step (the maps below use gpu's fields as work space)
    for n in FIELDS:
        ref.set_field(n, gpu.get_field(n))
    ref.set_initial_mass(0.0)
    ref.step(1)
    comp = ag.full_step(gpu, 1, st)
    g = cfg["ghost"]
    for k in ("c", "u", "v", "p"):
        a = ref.get_field(FIELD[k])
        want = a[g:a.shape[0] - g, g:a.shape[1] - g]
        got = comp[k].cpu().numpy()
        err = np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-300)
        print(name, k, f"{err:.2e}")
        assert err <= 1e-9, (name, k, err)
    ref.close()
    gpu.close()


# The parameter directions move the loss by ~1e-7 per 1e-6 of parameter, the order of the solves' own noise
# (tolerance 1e-13 on terms of size ~1e3): their differences use a 4-point stencil, O(h^4), at h = 1e-3.
EPS_PARAM = 1e-3


def fd4(f, h):
    return (8.0 * (f(h) - f(-h)) - (f(2 * h) - f(-2 * h))) / (12.0 * h)


def _loss(ag, gpu, st, w, sigma=None, mob=None):
    s = dict(st)
    for k in (1, 2):
        s = ag.full_step(gpu, k, s, sigma_scale=sigma, inv_pe_scale=mob)
    return sum((w[k] * s[k]).sum() for k in w)


@pytest.mark.parametrize("name", sorted(CASES))
def test_two_step_gradient_matches_central_differences(dn, name):
    from ding_nsch_core_solver_b200 import autograd as ag

    cfg, gpu = _pair(dn, name)
    st = _state(gpu, cfg)
    rng = np.random.default_rng(17)
    w = {k: torch.tensor(rng.standard_normal(tuple(st[k].shape)), device="cuda") for k in ("c", "u", "v", "p")}
    x = {k: a.clone().requires_grad_(k in ("c", "u", "v", "p")) for k, a in st.items()}
    one = lambda: torch.tensor(1.0, dtype=torch.float64, device="cuda", requires_grad=True)
    sig, mob = one(), one()
    grads = torch.autograd.grad(_loss(ag, gpu, x, w, sig, mob), [x["c"], x["u"], x["v"], x["p"], sig, mob])
    # directions in the initial c, u, v, p
    d = {k: torch.tensor(rng.standard_normal(tuple(st[k].shape)), device="cuda") for k in ("c", "u", "v", "p")}
    adj = sum(float((gr * d[k]).sum()) for gr, k in zip(grads[:4], ("c", "u", "v", "p")))
    eps = 1e-6
    with torch.no_grad():
        plus = {k: st[k] + eps * d[k] if k in d else st[k] for k in st}
        minus = {k: st[k] - eps * d[k] if k in d else st[k] for k in st}
        fd = (float(_loss(ag, gpu, plus, w)) - float(_loss(ag, gpu, minus, w))) / (2 * eps)
        fd_s = fd4(lambda h: float(_loss(ag, gpu, st, w, sigma=torch.tensor(1 + h, device="cuda",
                                                                             dtype=torch.float64))), EPS_PARAM)
    # mobility: 1/Pe scaled by 1 + h is Pe / (1 + h), on solvers built with it
    def with_pe(h):
        s2 = dn.Solver(dict(cfg, pe=cfg["pe"] / (1.0 + h)))
        s2.set_initial_mass(0.0)
        with torch.no_grad():
            val = float(_loss(ag, s2, st, w))
        s2.close()
        return val

    fd_m = fd4(with_pe, EPS_PARAM)
    res = {"state": (fd, adj), "sigma": (fd_s, float(grads[4])), "mobility": (fd_m, float(grads[5]))}
    for k, (a, b) in res.items():
        print(name, k, f"fd {a:.10e} adjoint {b:.10e}")
    for k, (a, b) in res.items():
        assert abs(a - b) <= 1e-6 * max(abs(a), 1e-6), (name, k, a, b)
    gpu.close()
