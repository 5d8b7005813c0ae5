"""Discrete adjoint of the pressure projection (dn_projection_adjoint, the backward of
ding_nsch_core_solver_b200.autograd.Projection).

Three checks, all in FP64 with the pressure solve at tolerance 1e-13:
- the forward dn_projection against the oracle's projection on the same inputs;
- the adjoint against the reference FP64 adjoint J^T, with J assembled column by column from the oracle's
  projection (an affine map at fixed rho_mid; the CPU test pins that premise);
- the autograd gradient against central finite differences (eps = 1e-6) on 16 seeded random directions,
  and torch.autograd.gradcheck on the smallest grid.
The grids are small so that J (about 500 x 500) is cheap; the cases cover walls (pure Neumann pressure,
mean projection), a Dirichlet pressure side, Neumann velocity sides, periodic x, periodic y and both, the
split and the variable-coefficient operators, and step 0 (p_ext = p) against a later step (2p - p_prev).
"""
import numpy as np
import pytest

from oracle.projection_adjoint import ProjectionOracle, flat_outputs, input_shapes, output_shapes, split_cotangent
from test_gpu_parity import unit

TOL_REF = 1e-9   # GPU adjoint vs J^T (both solves at relative tolerance 1e-13)
TOL_FD = 1e-6    # autograd gradient vs central differences
TOL_FWD = 1e-10  # dn_projection vs the oracle's projection


def _cfg(**kw):
    base = dict(pressure_tolerance=1e-13, poisson_iterations=5000, dt=1e-3, density_ratio=10.0)
    base.update(kw)
    return unit(**base)


CASES = {
    "split_icpcg_walls": _cfg(nx=12, ny=10, periodic_x=False, periodic_y=False, pressure_scheme="split_icpcg"),
    "split_ildlt_periodic": _cfg(nx=10, ny=12, pressure_scheme="split_ildlt_pcg"),
    "icpcg_channel_x": _cfg(nx=12, ny=10, periodic_x=True, periodic_y=False, pressure_scheme="icpcg",
                            top_wall_velocity_x=0.5, bottom_wall_velocity_x=-0.5),
    "ildlt_dirichlet_neumann_u": _cfg(nx=10, ny=12, periodic_x=False, periodic_y=False, pressure_scheme="ildlt_pcg",
                                      pressure_bc_top_type="dirichlet", pressure_bc_top_value=0.3,
                                      u_bc_left_type="neumann", u_bc_left_value=0.05, v_bc_top_type="neumann",
                                      v_bc_top_value=0.02),
    "split_channel_y_neumann_u": _cfg(nx=12, ny=10, periodic_x=False, periodic_y=True, pressure_scheme="split_icpcg",
                                      u_bc_right_type="neumann", u_bc_right_value=-0.1),
}


def _rho_mid(cfg, seed):
    """A smooth positive density in [1, 10] on the full Field2D array (only interior cells are read)."""
    rng = np.random.default_rng(seed)
    g = cfg["ghost"]
    sx, sy = cfg["nx"] + 2 * g, cfg["ny"] + 2 * g
    i = np.arange(sx)[:, None] / sx
    j = np.arange(sy)[None, :] / sy
    f = np.sin(2 * np.pi * (i + rng.random())) * np.cos(2 * np.pi * (2 * j + rng.random())) + 0.3 * rng.random((sx, sy))
    return 1.0 + 9.0 * (f - f.min()) / (f.max() - f.min())


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_reference_adjoint_premise_affine():
    """The oracle's projection at fixed rho_mid is affine: F(x) - F(0) = J x, and J^T passes the
    dot-product test <J x, w> = <x, J^T w>.  This pins the reference adjoint without a GPU."""
    for name in ("split_icpcg_walls", "icpcg_channel_x"):
        cfg = CASES[name]
        po = ProjectionOracle(cfg, _rho_mid(cfg, 1), 2)
        try:
            J = po.jacobian()
            rng = np.random.default_rng(5)
            x = [rng.standard_normal(s) for s in input_shapes(cfg)]
            zeros = [np.zeros(s) for s in input_shapes(cfg)]
            fx = flat_outputs(po(*x)[0]) - flat_outputs(po(*zeros)[0])
            xv = np.concatenate([a.ravel() for a in x])
            assert _rel(fx, J @ xv) < 1e-11, name
            w = rng.standard_normal(J.shape[0])
            assert abs(np.dot(J @ xv, w) - np.dot(xv, J.T @ w)) < 1e-10 * abs(np.dot(J @ xv, w)) + 1e-12
        finally:
            po.close()


# ------------------------------------------------------------------------------------------------ GPU
def _solver(cfg, rho):
    from ding_nsch_core_solver_b200 import capi

    s = capi.Solver(cfg)
    s.set_field("rho_mid", rho)
    return s


def _cuda(arrs):
    import torch

    return [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrs]


@pytest.mark.gpu
@pytest.mark.parametrize("step", [0, 3])
@pytest.mark.parametrize("name", sorted(CASES))
def test_projection_forward_matches_oracle(name, step):
    from ding_nsch_core_solver_b200.autograd import projection

    cfg = CASES[name]
    rho = _rho_mid(cfg, 7)
    rng = np.random.default_rng(11 + step)
    x = [rng.standard_normal(s) for s in input_shapes(cfg)]
    po = ProjectionOracle(cfg, rho, step)
    s = _solver(cfg, rho)
    try:
        ref, _ = po(*x)
        got = projection(s, step, *_cuda(x))
        for k, (a, b) in enumerate(zip(got, ref)):
            assert _rel(a.cpu().numpy(), b) < TOL_FWD, (name, step, k)
    finally:
        s.close()
        po.close()


@pytest.mark.gpu
@pytest.mark.parametrize("step", [0, 3])
@pytest.mark.parametrize("name", sorted(CASES))
def test_adjoint_matches_reference_transpose(name, step):
    from ding_nsch_core_solver_b200.autograd import projection_adjoint

    cfg = CASES[name]
    rho = _rho_mid(cfg, 7)
    po = ProjectionOracle(cfg, rho, step)
    s = _solver(cfg, rho)
    try:
        J = po.jacobian()
        rng = np.random.default_rng(23 + step)
        cot = [rng.standard_normal(sh) for sh in output_shapes(cfg)]
        ref = split_cotangent(cfg, J.T @ flat_outputs(cot))
        got, (its, rel) = projection_adjoint(s, step, *_cuda(cot))
        assert its > 0 and rel < 1e-13
        for k, (a, b) in enumerate(zip(got, ref)):
            assert _rel(a.cpu().numpy(), b) < TOL_REF, (name, step, k, _rel(a.cpu().numpy(), b))
    finally:
        s.close()
        po.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["split_icpcg_walls", "icpcg_channel_x", "ildlt_dirichlet_neumann_u"])
def test_autograd_gradient_central_fd(name):
    import torch

    from ding_nsch_core_solver_b200.autograd import projection

    cfg = CASES[name]
    step = 2
    s = _solver(cfg, _rho_mid(cfg, 3))
    try:
        rng = np.random.default_rng(31)
        x = [t.requires_grad_() for t in _cuda([rng.standard_normal(sh) for sh in input_shapes(cfg)])]
        w = _cuda([rng.standard_normal(sh) for sh in output_shapes(cfg)])

        def loss(args):
            return sum((o * wk).sum() for o, wk in zip(projection(s, step, *args), w))

        loss(x).backward()
        grads = [t.grad.detach() for t in x]
        eps = 1e-6
        for k in range(16):
            d = _cuda([np.random.default_rng(100 + k).standard_normal(sh) for sh in input_shapes(cfg)])
            with torch.no_grad():
                lp = loss([a + eps * b for a, b in zip(x, d)]).item()
                lm = loss([a - eps * b for a, b in zip(x, d)]).item()
            fd = (lp - lm) / (2 * eps)
            an = sum((g_ * b).sum().item() for g_, b in zip(grads, d))
            assert abs(fd - an) <= TOL_FD * abs(an), (name, k, fd, an)
    finally:
        s.close()


@pytest.mark.gpu
def test_autograd_gradcheck_smallest_grid():
    import torch

    from ding_nsch_core_solver_b200.autograd import projection

    cfg = _cfg(nx=8, ny=8, periodic_x=False, periodic_y=False, pressure_scheme="split_icpcg")
    s = _solver(cfg, _rho_mid(cfg, 4))
    try:
        rng = np.random.default_rng(41)
        x = tuple(t.requires_grad_() for t in _cuda([rng.standard_normal(sh) for sh in input_shapes(cfg)]))
        assert torch.autograd.gradcheck(lambda *a: projection(s, 1, *a), x, eps=1e-6, atol=1e-6, rtol=1e-5)
    finally:
        s.close()


# ------------------------------------------------------------------------------------- CH implicit solve
CH_CASES = {
    "ch_periodic": _cfg(nx=10, ny=12, ch_tolerance=1e-13, ch_inner_iterations=500),
    "ch_walls": _cfg(nx=12, ny=10, periodic_x=False, periodic_y=False, ch_tolerance=1e-13, ch_inner_iterations=500),
    "ch_channel_x": _cfg(nx=12, ny=10, periodic_x=True, periodic_y=False, ch_tolerance=1e-13,
                         ch_inner_iterations=500),
}


def _oracle_ch_jacobian(cfg, alpha0):
    """Columns A^-1 e_k from the oracle's CH solve (zero start, tolerance 1e-13)."""
    from oracle.oracle import OracleSolver

    o = OracleSolver(cfg, "port")
    o.initialize()
    g = cfg["ghost"]
    nx, ny = cfg["nx"], cfg["ny"]
    cols = []
    try:
        for k in range(nx * ny):
            full = np.zeros((nx + 2 * g, ny + 2 * g))
            full[g + k // ny, g + k % ny] = 1.0
            c = o.ch_linear_solve(full, alpha0, np.zeros_like(full))[0]
            cols.append(c[g:g + nx, g:g + ny].ravel())
    finally:
        o.close()
    return np.stack(cols, axis=1)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CH_CASES))
def test_ch_solve_adjoint_matches_reference_transpose(name):
    """The backward of the CH implicit solve (the same solve on the cotangent) against J^T from the oracle."""
    import torch

    from ding_nsch_core_solver_b200 import capi
    from ding_nsch_core_solver_b200.autograd import ch_solve

    cfg = CH_CASES[name]
    alpha0 = 1.5 / cfg["dt"]
    J = _oracle_ch_jacobian(cfg, alpha0)
    s = capi.Solver(cfg)
    try:
        rng = np.random.default_rng(43)
        rhs = torch.from_numpy(rng.standard_normal((cfg["nx"], cfg["ny"]))).cuda().requires_grad_()
        w = rng.standard_normal((cfg["nx"], cfg["ny"]))
        out = ch_solve(s, alpha0, rhs)
        assert _rel(out.detach().cpu().numpy().ravel(), J @ rhs.detach().cpu().numpy().ravel()) < TOL_REF
        out.backward(torch.from_numpy(w).cuda())
        assert _rel(rhs.grad.cpu().numpy().ravel(), J.T @ w.ravel()) < TOL_REF, name
    finally:
        s.close()


@pytest.mark.gpu
def test_ch_solve_gradient_central_fd():
    import torch

    from ding_nsch_core_solver_b200 import capi
    from ding_nsch_core_solver_b200.autograd import ch_solve

    cfg = CH_CASES["ch_walls"]
    alpha0 = 1.0 / cfg["dt"]
    s = capi.Solver(cfg)
    try:
        rng = np.random.default_rng(47)
        x = torch.from_numpy(rng.standard_normal((cfg["nx"], cfg["ny"]))).cuda().requires_grad_()
        w = torch.from_numpy(rng.standard_normal((cfg["nx"], cfg["ny"]))).cuda()
        (ch_solve(s, alpha0, x) * w).sum().backward()
        eps = 1e-6
        for k in range(16):
            d = torch.from_numpy(np.random.default_rng(300 + k).standard_normal((cfg["nx"], cfg["ny"]))).cuda()
            with torch.no_grad():
                lp = (ch_solve(s, alpha0, x + eps * d) * w).sum().item()
                lm = (ch_solve(s, alpha0, x - eps * d) * w).sum().item()
            fd = (lp - lm) / (2 * eps)
            an = (x.grad * d).sum().item()
            assert abs(fd - an) <= TOL_FD * abs(an), (k, fd, an)
    finally:
        s.close()


def test_ch_operator_inverse_is_symmetric():
    """The premise of using the CH solve as its own adjoint: the oracle's A^-1 (assembled column by column)
    is symmetric to round-off for periodic, wall and channel boundaries."""
    for name, cfg in CH_CASES.items():
        J = _oracle_ch_jacobian(cfg, 1.5 / cfg["dt"])
        assert np.linalg.norm(J - J.T) <= 1e-12 * np.linalg.norm(J), name
