"""Adjoints of the CH phase: the advective term with WENO5 face values (dn_advection_adjoint), nonlinear
weights included; the whole explicit operator E (dn_explicit_operator_adjoint); and the phase composed from E
and the implicit solve (autograd.ch_phase).

- dn_advection against the oracle's build_phase_advection_fluxes restatement on the same inputs;
- the adjoint against the reference FP64 adjoint J^T, J assembled by central differences of the oracle's
  advective term (step 1e-6), which shares no derivation with the CUDA transpose;
- the autograd gradient against central finite differences of the CUDA forward (eps = 1e-6) on 16 seeded
  random directions, and torch.autograd.gradcheck on the smallest grid.
The face velocities are kept at least 0.05 away from 0 (the upwind switch is not differentiable there), and
c is rough enough that every WENO5 smoothness indicator stays far above its 1e-6 regularisation, where
central differences stay accurate.
"""
import numpy as np
import pytest

from oracle.oracle import OracleSolver
from test_gpu_parity import unit

TOL_FWD = 1e-13
TOL_REF = 1e-6
TOL_FD = 1e-6

CASES = {
    "periodic": unit(nx=10, ny=12),
    "walls": unit(nx=12, ny=10, periodic_x=False, periodic_y=False),
    "neumann_left_moving_top": unit(nx=10, ny=12, periodic_x=False, periodic_y=False, u_bc_left_type="neumann",
                                    u_bc_left_value=0.05, v_bc_top_type="neumann", top_wall_velocity_x=0.4),
    "channel_x": unit(nx=12, ny=10, periodic_x=True, periodic_y=False, top_wall_velocity_x=0.5,
                      bottom_wall_velocity_x=-0.5),
}


def _shapes(cfg):
    nx, ny = cfg["nx"], cfg["ny"]
    return [(nx, ny), (nx + 1, ny), (nx, ny + 1)]


def _point(cfg, seed):
    """Interior c, u, v: c rough O(1), face velocities of random sign with |u| >= 0.05."""
    rng = np.random.default_rng(seed)
    c = rng.standard_normal(_shapes(cfg)[0])
    vel = []
    for shp in _shapes(cfg)[1:]:
        vel.append(rng.choice([-1.0, 1.0], size=shp) * (0.05 + 0.5 * np.abs(rng.standard_normal(shp))))
    return [c] + vel


def _full(cfg, a):
    g = cfg["ghost"]
    f = np.zeros((a.shape[0] + 2 * g, a.shape[1] + 2 * g))
    f[g:g + a.shape[0], g:g + a.shape[1]] = a
    return f


def _oracle_term(orc, cfg, c, u, v):
    g = cfg["ghost"]
    out = orc.advection(_full(cfg, c), _full(cfg, u), _full(cfg, v))
    return out[g:out.shape[0] - g, g:out.shape[1] - g]


def _oracle_jacobian(orc, cfg, x, h=1e-6):
    cols = []
    for k in range(3):
        for idx in range(x[k].size):
            xp = [a.copy() for a in x]
            xm = [a.copy() for a in x]
            xp[k].flat[idx] += h
            xm[k].flat[idx] -= h
            cols.append(((_oracle_term(orc, cfg, *xp) - _oracle_term(orc, cfg, *xm)) / (2 * h)).ravel())
    return np.stack(cols, axis=1)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _cuda(arrs):
    import torch

    return [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrs]


def _oracle(cfg):
    o = OracleSolver(cfg, "port")
    o.initialize()
    return o


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_advection_forward_matches_oracle(name):
    from ding_nsch_core_solver_b200 import capi
    from ding_nsch_core_solver_b200.autograd import advection

    cfg = CASES[name]
    x = _point(cfg, 3)
    orc, s = _oracle(cfg), capi.Solver(cfg)
    try:
        ref = _oracle_term(orc, cfg, *x)
        got = advection(s, *_cuda(x)).cpu().numpy()
        assert _rel(got, ref) <= TOL_FWD, (name, _rel(got, ref))
    finally:
        s.close()
        orc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_advection_adjoint_matches_reference_transpose(name):
    from ding_nsch_core_solver_b200 import capi
    from ding_nsch_core_solver_b200.autograd import advection

    cfg = CASES[name]
    x = _point(cfg, 5)
    orc, s = _oracle(cfg), capi.Solver(cfg)
    try:
        J = _oracle_jacobian(orc, cfg, x)
        w = np.random.default_rng(9).standard_normal(_shapes(cfg)[0])
        ref = J.T @ w.ravel()
        xt = [t.requires_grad_() for t in _cuda(x)]
        advection(s, *xt).backward(_cuda([w])[0])
        got = np.concatenate([t.grad.cpu().numpy().ravel() for t in xt])
        assert _rel(got, ref) <= TOL_REF, (name, _rel(got, ref))
        # the velocity and phase parts separately, so neither hides behind the other's norm
        n0 = x[0].size
        assert _rel(got[:n0], ref[:n0]) <= TOL_REF, name
        assert _rel(got[n0:], ref[n0:]) <= TOL_REF, name
    finally:
        s.close()
        orc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_advection_gradient_central_fd(name):
    import torch

    from ding_nsch_core_solver_b200 import capi
    from ding_nsch_core_solver_b200.autograd import advection

    cfg = CASES[name]
    s = capi.Solver(cfg)
    try:
        x = [t.requires_grad_() for t in _cuda(_point(cfg, 17))]
        w = _cuda([np.random.default_rng(19).standard_normal(_shapes(cfg)[0])])[0]

        def loss(args):
            return (advection(s, *args) * w).sum()

        loss(x).backward()
        grads = [t.grad.detach() for t in x]
        eps = 1e-6
        for k in range(16):
            d = _cuda([np.random.default_rng(200 + k).standard_normal(sh) for sh in _shapes(cfg)])
            with torch.no_grad():
                lp = loss([a + eps * b for a, b in zip(x, d)]).item()
                lm = loss([a - eps * b for a, b in zip(x, d)]).item()
            fd = (lp - lm) / (2 * eps)
            an = sum((g_ * b).sum().item() for g_, b in zip(grads, d))
            assert abs(fd - an) <= TOL_FD * abs(an), (name, k, fd, an)
    finally:
        s.close()


@pytest.mark.gpu
def test_advection_gradcheck_smallest_grid():
    import torch

    from ding_nsch_core_solver_b200 import capi
    from ding_nsch_core_solver_b200.autograd import advection

    cfg = unit(nx=8, ny=8, periodic_x=False, periodic_y=True)
    s = capi.Solver(cfg)
    try:
        x = tuple(t.requires_grad_() for t in _cuda(_point(cfg, 23)))
        assert torch.autograd.gradcheck(lambda *a: advection(s, *a), x, eps=1e-6, atol=1e-6, rtol=1e-5)
    finally:
        s.close()


def test_oracle_advection_properties():
    """The oracle's advective term, which the reference adjoint is built from: on a doubly periodic grid it
    conserves mass (sum of -div(u c) is 0), and for uniform c it is exactly -c div(u) (WENO5 reproduces
    constants)."""
    cfg = CASES["periodic"]
    c, u, v = _point(cfg, 29)
    orc = _oracle(cfg)
    try:
        r = _oracle_term(orc, cfg, c, u, v)
        assert abs(r.sum()) <= 1e-12 * np.abs(r).sum()
        dx, dy = cfg["lx"] / cfg["nx"], cfg["ly"] / cfg["ny"]
        # periodic: face nx is face 0 after the BC, so take u with that identification
        u[-1, :] = u[0, :]
        v[:, -1] = v[:, 0]
        r = _oracle_term(orc, cfg, np.full_like(c, 0.7), u, v)
        div = (u[1:, :] - u[:-1, :]) / dx + (v[:, 1:] - v[:, :-1]) / dy
        assert _rel(r, -0.7 * div) <= 1e-13
    finally:
        orc.close()


# ------------------------------------------------------------------ explicit operator E and the CH phase
def _ch_cfg(cfg):
    return dict(cfg, ch_tolerance=1e-13, ch_inner_iterations=500)


def _point_e(cfg, seed):
    """c around 0.5 (mostly inside the mobility's (0, 1) branch), face velocities away from 0."""
    x = _point(cfg, seed)
    x[0] = 0.5 + 0.3 * x[0]
    return x


def _oracle_e(orc, cfg, c, u, v):
    g = cfg["ghost"]
    out = orc.explicit_operator(_full(cfg, c), _full(cfg, u), _full(cfg, v))
    return out[g:out.shape[0] - g, g:out.shape[1] - g]


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_explicit_operator_forward_and_adjoint(name):
    from ding_nsch_core_solver_b200 import capi
    from ding_nsch_core_solver_b200.autograd import explicit_operator

    cfg = CASES[name]
    x = _point_e(cfg, 7)
    orc, s = _oracle(cfg), capi.Solver(cfg)
    try:
        xt = [t.requires_grad_() for t in _cuda(x)]
        out = explicit_operator(s, *xt)
        assert _rel(out.detach().cpu().numpy(), _oracle_e(orc, cfg, *x)) <= TOL_FWD, name
        h = 1e-6
        cols = []
        for k in range(3):
            for idx in range(x[k].size):
                xp = [a.copy() for a in x]
                xm = [a.copy() for a in x]
                xp[k].flat[idx] += h
                xm[k].flat[idx] -= h
                cols.append(((_oracle_e(orc, cfg, *xp) - _oracle_e(orc, cfg, *xm)) / (2 * h)).ravel())
        J = np.stack(cols, axis=1)
        w = np.random.default_rng(11).standard_normal(_shapes(cfg)[0])
        out.backward(_cuda([w])[0])
        got = np.concatenate([t.grad.cpu().numpy().ravel() for t in xt])
        ref = J.T @ w.ravel()
        n0 = x[0].size
        assert _rel(got[:n0], ref[:n0]) <= TOL_REF and _rel(got[n0:], ref[n0:]) <= TOL_REF, (name, _rel(got, ref))
    finally:
        s.close()
        orc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("step", [0, 1])
@pytest.mark.parametrize("name", ["walls", "channel_x", "periodic"])
def test_ch_phase_forward_matches_oracle(name, step):
    """The composed phase reproduces the oracle's CH phase of the same state."""
    from ding_nsch_core_solver_b200 import capi
    from ding_nsch_core_solver_b200.autograd import ch_phase

    cfg = _ch_cfg(CASES[name])
    g = cfg["ghost"]
    c, u, v = _point_e(cfg, 13)
    rng = np.random.default_rng(17)
    c_prev2 = c + 0.01 * rng.standard_normal(c.shape)
    e_prev = rng.standard_normal(c.shape)
    orc, s = _oracle(cfg), capi.Solver(cfg)
    try:
        orc.set_field("c", _full(cfg, c))
        orc.set_field("c_prev", _full(cfg, c_prev2))  # the step's history copy moves it to c_prev2
        orc.set_field("u", _full(cfg, u))
        orc.set_field("v", _full(cfg, v))
        orc.set_field("e_prev", _full(cfg, e_prev))
        orc.refresh_derived()  # BC ghosts of the injected state, as a step leaves them
        orc.begin_step(step)
        orc.phase(step)
        ref = orc.field("c")[g:g + cfg["nx"], g:g + cfg["ny"]]
        got = ch_phase(s, step, *_cuda([c, u, v]), *_cuda([c_prev2, e_prev])).cpu().numpy()
        assert _rel(got, ref) <= 1e-9, (name, step, _rel(got, ref))
    finally:
        s.close()
        orc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["walls", "channel_x"])
def test_ch_phase_gradient_central_fd(name):
    import torch

    from ding_nsch_core_solver_b200 import capi
    from ding_nsch_core_solver_b200.autograd import ch_phase

    cfg = _ch_cfg(CASES[name])
    s = capi.Solver(cfg)
    try:
        c, u, v = _point_e(cfg, 19)
        rng = np.random.default_rng(23)
        extra = [c + 0.01 * rng.standard_normal(c.shape), rng.standard_normal(c.shape)]
        x = [t.requires_grad_() for t in _cuda([c, u, v] + extra)]
        w = _cuda([rng.standard_normal(c.shape)])[0]

        def loss(a):
            return (ch_phase(s, 1, *a) * w).sum()

        loss(x).backward()
        grads = [t.grad.detach() for t in x]
        shapes = _shapes(cfg) + [c.shape, c.shape]
        eps = 1e-6
        for k in range(16):
            d = _cuda([np.random.default_rng(400 + k).standard_normal(sh) for sh in shapes])
            with torch.no_grad():
                lp = loss([a + eps * b for a, b in zip(x, d)]).item()
                lm = loss([a - eps * b for a, b in zip(x, d)]).item()
            fd = (lp - lm) / (2 * eps)
            an = sum((g_ * b).sum().item() for g_, b in zip(grads, d))
            assert abs(fd - an) <= TOL_FD * abs(an), (name, k, fd, an)
    finally:
        s.close()


@pytest.mark.gpu
def test_ch_rollout_checkpointed_gradient():
    """Six CH phases at fixed velocity: the gradient of <w, c^6> in (c^0, u, v) with checkpoints every 2 steps
    equals the gradient that keeps every step, and matches central FD on 16 directions."""
    import torch

    from ding_nsch_core_solver_b200 import capi
    from ding_nsch_core_solver_b200.autograd import ch_rollout

    cfg = _ch_cfg(CASES["channel_x"])
    s = capi.Solver(cfg)
    try:
        c, u, v = _point_e(cfg, 29)
        w = _cuda([np.random.default_rng(31).standard_normal(c.shape)])[0]
        grads = []
        for every in (0, 2):
            x = [t.requires_grad_() for t in _cuda([c, u, v])]
            (ch_rollout(s, x[0], x[1], x[2], 6, checkpoint_every=every) * w).sum().backward()
            grads.append([t.grad.detach().clone() for t in x])
        for a, b in zip(*grads):
            assert torch.equal(a, b)
        base = [t.detach() for t in _cuda([c, u, v])]

        def loss(a):
            return (ch_rollout(s, a[0], a[1], a[2], 6) * w).sum().item()

        eps = 1e-6
        for k in range(16):
            d = _cuda([np.random.default_rng(500 + k).standard_normal(sh) for sh in _shapes(cfg)])
            with torch.no_grad():
                fd = (loss([a + eps * b for a, b in zip(base, d)]) - loss([a - eps * b for a, b in zip(base, d)])) / (2 * eps)
            an = sum((g_ * b).sum().item() for g_, b in zip(grads[1], d))
            assert abs(fd - an) <= TOL_FD * abs(an), (k, fd, an)
    finally:
        s.close()
