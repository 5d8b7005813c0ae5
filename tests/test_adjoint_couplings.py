"""The coupling maps of the full-step adjoint, each against central finite differences on its own.

* surface_force: (c_old, c_new) -> (fxu, fyv), dn_surface_force_adjoint;
* projection_rho: (u*, v*, p, p_prev, rho_mid) -> (u, v, p_new, p_prev_new), dn_projection_rho_adjoint, on
  the variable-density operator (icpcg) and the split scheme (its explicit rho_mid term);
* full_step restricted to the direction of c alone (the path through the materials, the surface force and
  the CH phase), so that no other input's sensitivity can mask it.
For random directions d and cotangents w, <w, J d> by central differences (eps 1e-6) must equal <J^T w, d>
to 1e-6 relative.
"""
import numpy as np
import pytest
import torch

from test_adjoint_full_step import CASES as STEP_CASES
from test_adjoint_full_step import _pair, _state
from test_gpu_parity import seeded_pair, unit

pytestmark = pytest.mark.gpu

TIGHT = dict(pressure_tolerance=1e-13, poisson_iterations=50000, ch_tolerance=1e-13, ch_inner_iterations=20000,
             momentum_tolerance=1e-14, momentum_iterations=2000)
CASES = {
    "walls_icpcg": unit(nx=24, ny=20, periodic_x=False, periodic_y=False, pressure_scheme="icpcg", dt=2e-4,
                        density_ratio=5.0, pressure_bc_top_type="dirichlet", pressure_bc_top_value=0.2, **TIGHT),
    "channel_split": unit(nx=28, ny=16, periodic_x=True, periodic_y=False, pressure_scheme="split_icpcg", dt=2e-4,
                          density_ratio=4.0, top_wall_velocity_x=0.5, bottom_wall_velocity_x=-0.5, **TIGHT),
}


@pytest.fixture(scope="module")
def dn():
    import ding_nsch_core_solver_b200 as m

    m.load()
    return m


def _t(a, g):
    return torch.tensor(np.ascontiguousarray(a[g:a.shape[0] - g, g:a.shape[1] - g]), dtype=torch.float64,
                        device="cuda")


def _check(fn, inputs, rng, label, eps=1e-6):
    x = [a.clone().requires_grad_(True) for a in inputs]
    outs = fn(*x)
    w = [torch.tensor(rng.standard_normal(tuple(o.shape)), device="cuda") for o in outs]
    grads = torch.autograd.grad(sum((wi * o).sum() for wi, o in zip(w, outs)), x)
    d = [torch.tensor(rng.standard_normal(tuple(a.shape)), device="cuda") for a in inputs]
    adj = sum(float((g * di).sum()) for g, di in zip(grads, d))
    with torch.no_grad():
        lp = sum(float((wi * o).sum()) for wi, o in zip(w, fn(*[a + eps * di for a, di in zip(inputs, d)])))
        lm = sum(float((wi * o).sum()) for wi, o in zip(w, fn(*[a - eps * di for a, di in zip(inputs, d)])))
    fd = (lp - lm) / (2 * eps)
    print(label, f"fd {fd:.12e} adjoint {adj:.12e}")
    assert abs(fd - adj) <= 1e-6 * max(abs(fd), 1e-9), (label, fd, adj)


@pytest.mark.parametrize("name", sorted(CASES))
def test_surface_force_adjoint(dn, name):
    from ding_nsch_core_solver_b200 import autograd as ag

    cfg = CASES[name]
    orc, gpu = seeded_pair(dn, cfg, seed=3)
    g = cfg["ghost"]
    rng = np.random.default_rng(1)
    c = _t(gpu.get_field("c"), g)
    c_new = c + 0.01 * torch.tensor(rng.standard_normal(tuple(c.shape)), device="cuda")
    _check(lambda a, b: ag.surface_force(gpu, a, b), [c, c_new], rng, f"{name} surface_force")
    gpu.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_projection_rho_adjoint(dn, name):
    from ding_nsch_core_solver_b200 import autograd as ag

    cfg = CASES[name]
    orc, gpu = seeded_pair(dn, cfg, seed=5)
    g = cfg["ghost"]
    rng = np.random.default_rng(2)
    ins = [_t(gpu.get_field(n), g) for n in ("u", "v", "p", "p_prev", "rho_mid")]
    for step in (0, 1):
        _check(lambda us, vs, p, pp, rho: ag.projection_rho(gpu, step, us, vs, p, pp, rho), ins, rng,
               f"{name} projection_rho step {step}")
    gpu.close()


@pytest.mark.parametrize("name", sorted(STEP_CASES))
def test_full_step_in_c_alone(dn, name):
    from ding_nsch_core_solver_b200 import autograd as ag

    cfg, gpu = _pair(dn, name)
    st = _state(gpu, cfg)
    rng = np.random.default_rng(8)

    def fn(c):
        out = ag.full_step(gpu, 1, dict(st, c=c))
        return [out[k] for k in ("c", "u", "v", "p")]

    _check(fn, [st["c"]], rng, f"{name} full_step(c)")
    gpu.close()
