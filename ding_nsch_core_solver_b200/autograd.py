"""torch.autograd.Functions over the differentiable pieces of the C-ABI: the pressure projection, the CH
advective term and the CH implicit solve.

`projection(solver, step, u_star, v_star, p, p_prev)` runs the pressure projection of one step --
pressure solve plus velocity correction (dn_projection) -- on interior-shaped float64 CUDA tensors and
returns (u, v, p_new, p_prev_new).  Its backward is the hand-written discrete adjoint dn_projection_adjoint,
whose transposed pressure solve is the same PCG.  rho_mid is a constant of the map: the solver's rho_mid at
the forward call is kept and put back before the backward runs.  The reference has no adjoint.

`advection(solver, c, u, v)` returns the CH advective term -div(u c) with WENO5 face values (dn_advection);
its backward (dn_advection_adjoint) differentiates the WENO5 nonlinear weights.  The upwind side follows the
sign of each face velocity, so the term is not differentiable where a face velocity is exactly 0.

`momentum_predictor(solver, step, u, v, hu_prev, hv_prev, fxu, fyv)` is the momentum predictor at fixed
materials (dn_momentum_map); its backward (dn_momentum_adjoint) solves the transposed coupled viscous system
with the same BiCGSTAB and transposes the centred convection (linearised at u, v) and the explicit viscous
term.  `velocity_step` composes it with the projection.

`ch_solve(solver, alpha0, rhs)` is the CH implicit solve (dn_ch_linear_solve); its operator is symmetric, so
its backward is the same solve.  `explicit_operator(solver, c, u, v)` is the CH explicit operator, and
`ch_phase` composes the two into the CH phase of a step, and `ch_rollout` chains phases over a horizon with
optional checkpointing every K steps.

Shapes (interior values only): u, u_star (nx+1, ny); v, v_star (nx, ny+1); c, p, p_prev, p_new, the
advective term (nx, ny).
"""
import ctypes as C

import torch

from . import capi


def _full(solver, t, kind):
    """Zero-ghosted Field2D buffer holding interior values t."""
    g = solver.ghost
    nx, ny = solver.nx, solver.ny
    shp = {"u": (nx + 1, ny), "v": (nx, ny + 1), "c": (nx, ny)}[kind]
    if tuple(t.shape) != shp:
        raise ValueError(f"expected interior shape {shp}, got {tuple(t.shape)}")
    buf = torch.zeros((shp[0] + 2 * g, shp[1] + 2 * g), dtype=torch.float64, device=t.device)
    buf[g:g + shp[0], g:g + shp[1]] = t
    return buf


def _interior(solver, buf):
    g = solver.ghost
    return buf[g:buf.shape[0] - g, g:buf.shape[1] - g].clone()


def _call(solver, fn, step, ins, outs):
    torch.cuda.current_stream().synchronize()  # the C-ABI runs on the solver's own stream
    its, rel = C.c_int(), C.c_double()
    solver._check(fn(solver._h, int(step), *[t.data_ptr() for t in ins], *[t.data_ptr() for t in outs],
                     C.byref(its), C.byref(rel)))
    return its.value, rel.value


class Projection(torch.autograd.Function):
    @staticmethod
    def forward(ctx, solver, step, u_star, v_star, p, p_prev):
        ins = [_full(solver, u_star, "u"), _full(solver, v_star, "v"), _full(solver, p, "c"),
               _full(solver, p_prev, "c")]
        outs = [torch.empty_like(b) for b in ins]
        its, rel = _call(solver, solver._lib.dn_projection, step, ins, outs)
        ctx.solver, ctx.step = solver, int(step)
        ctx.rho_mid = solver.get_field("rho_mid")
        ctx.forward_report = (its, rel)
        return tuple(_interior(solver, b) for b in outs)

    @staticmethod
    def backward(ctx, gu, gv, gp, gpp):
        solver = ctx.solver
        solver.set_field("rho_mid", ctx.rho_mid)
        zeros = {"u": (solver.nx + 1, solver.ny), "v": (solver.nx, solver.ny + 1), "c": (solver.nx, solver.ny)}
        cot = []
        for g_, kind in zip((gu, gv, gp, gpp), ("u", "v", "c", "c")):
            if g_ is None:
                g_ = torch.zeros(zeros[kind], dtype=torch.float64, device="cuda")
            cot.append(_full(solver, g_.to(torch.float64).contiguous(), kind))
        outs = [torch.empty_like(b) for b in cot]
        _call(solver, solver._lib.dn_projection_adjoint, ctx.step, cot, outs)
        return (None, None) + tuple(_interior(solver, b) for b in outs)


def projection(solver, step, u_star, v_star, p, p_prev):
    """(u, v, p_new, p_prev_new) of one projection; differentiable in u_star, v_star, p and p_prev."""
    return Projection.apply(solver, step, u_star, v_star, p, p_prev)


def projection_adjoint(solver, step, gu, gv, gp, gpp):
    """The vector-Jacobian product alone: cotangents of (u, v, p_new, p_prev_new) in, of (u_star, v_star, p,
    p_prev) out, with the solver's current rho_mid.  Returns the four arrays and (iterations, residual)."""
    cot = [_full(solver, gu, "u"), _full(solver, gv, "v"), _full(solver, gp, "c"), _full(solver, gpp, "c")]
    outs = [torch.empty_like(b) for b in cot]
    rep = _call(solver, solver._lib.dn_projection_adjoint, step, cot, outs)
    return tuple(_interior(solver, b) for b in outs), rep


class MomentumPredictor(torch.autograd.Function):
    """(u, v, hu_prev, hv_prev, fxu, fyv) -> (u_star, v_star) through dn_momentum_map, with the solver's rho_mid,
    eta and eta_prev held fixed (kept at the forward call, put back before the backward); backward is
    dn_momentum_adjoint, whose transposed coupled solve is the same Jacobi-BiCGSTAB on M^T."""

    @staticmethod
    def forward(ctx, solver, step, u, v, hu_prev, hv_prev, fxu, fyv):
        kinds = ("u", "v", "u", "v", "u", "v")
        ins = [_full(solver, t.to(torch.float64).contiguous(), k)
               for t, k in zip((u, v, hu_prev, hv_prev, fxu, fyv), kinds)]
        outs = [torch.empty_like(ins[0]), torch.empty_like(ins[1])]
        its, res = _call(solver, solver._lib.dn_momentum_map, step, ins, outs)
        ctx.solver, ctx.step = solver, int(step)
        ctx.materials = {n: solver.get_field(n) for n in ("rho_mid", "eta", "eta_prev")}
        ctx.save_for_backward(ins[0], ins[1])
        ctx.forward_report = (its, res)
        return tuple(_interior(solver, b) for b in outs)

    @staticmethod
    def backward(ctx, gus, gvs):
        solver = ctx.solver
        for n, a in ctx.materials.items():
            solver.set_field(n, a)
        u_full, v_full = ctx.saved_tensors
        shapes = {"u": (solver.nx + 1, solver.ny), "v": (solver.nx, solver.ny + 1)}
        cot = []
        for g_, kind in ((gus, "u"), (gvs, "v")):
            if g_ is None:
                g_ = torch.zeros(shapes[kind], dtype=torch.float64, device="cuda")
            cot.append(_full(solver, g_.to(torch.float64).contiguous(), kind))
        outs = [torch.empty_like(u_full), torch.empty_like(v_full), torch.empty_like(u_full),
                torch.empty_like(v_full), torch.empty_like(u_full), torch.empty_like(v_full)]
        _call(solver, solver._lib.dn_momentum_adjoint, ctx.step, [u_full, v_full] + cot, outs)
        return (None, None) + tuple(_interior(solver, b) for b in outs)


def momentum_predictor(solver, step, u, v, hu_prev, hv_prev, fxu, fyv):
    """(u_star, v_star) of the momentum predictor; differentiable in u, v, H_prev and the face surface forces
    (rho_mid, eta, eta_prev fixed).  Surface-tension parameters enter through fxu, fyv, which are linear in
    the surface_tension_multiplier sigma: pass sigma * f_hat to get d/d sigma."""
    return MomentumPredictor.apply(solver, step, u, v, hu_prev, hv_prev, fxu, fyv)


def velocity_step(solver, step, u, v, hu_prev, hv_prev, fxu, fyv, p, p_prev):
    """The velocity half of a step at fixed phase: the momentum predictor, then the projection.  Returns
    (u, v, p_new, p_prev_new); differentiable in all inputs (rho_mid, eta, eta_prev fixed)."""
    us, vs = momentum_predictor(solver, step, u, v, hu_prev, hv_prev, fxu, fyv)
    return projection(solver, step, us, vs, p, p_prev)


class Advection(torch.autograd.Function):
    @staticmethod
    def forward(ctx, solver, c, u, v):
        ins = [_full(solver, c, "c"), _full(solver, u, "u"), _full(solver, v, "v")]
        out = torch.empty_like(ins[0])
        torch.cuda.current_stream().synchronize()
        solver._check(solver._lib.dn_advection(solver._h, *[t.data_ptr() for t in ins], out.data_ptr()))
        ctx.solver = solver
        ctx.save_for_backward(*ins)
        return _interior(solver, out)

    @staticmethod
    def backward(ctx, g):
        solver = ctx.solver
        cf, uf, vf = ctx.saved_tensors
        gf = _full(solver, g.to(torch.float64).contiguous(), "c")
        outs = [torch.empty_like(cf), torch.empty_like(uf), torch.empty_like(vf)]
        torch.cuda.current_stream().synchronize()
        solver._check(solver._lib.dn_advection_adjoint(solver._h, cf.data_ptr(), uf.data_ptr(), vf.data_ptr(),
                                                       gf.data_ptr(), *[t.data_ptr() for t in outs]))
        return (None,) + tuple(_interior(solver, b) for b in outs)


def advection(solver, c, u, v):
    """-div(u c) with WENO5 face values; differentiable in c, u and v."""
    return Advection.apply(solver, c, u, v)



class CHSolve(torch.autograd.Function):
    """c = A^-1 rhs for the CH implicit operator A = alpha0 I - beta1 L + beta2 L^2 (dn_ch_linear_solve, the
    ch_solver backend: ILDLT-preconditioned CG from a zero start).  A is symmetric, so the backward is the same
    solve applied to the cotangent."""

    @staticmethod
    def forward(ctx, solver, alpha0, rhs):
        ctx.solver, ctx.alpha0 = solver, float(alpha0)
        return _ch_solve(solver, float(alpha0), rhs)

    @staticmethod
    def backward(ctx, g):
        return None, None, _ch_solve(ctx.solver, ctx.alpha0, g)


def _ch_solve(solver, alpha0, t):
    import numpy as np

    g = solver.ghost
    full = np.zeros((solver.nx + 2 * g, solver.ny + 2 * g))
    full[g:g + solver.nx, g:g + solver.ny] = t.detach().to(torch.float64).cpu().numpy()
    cs = solver.ch_linear_solve(full, alpha0, np.zeros_like(full))[0]
    return torch.from_numpy(np.ascontiguousarray(cs[g:g + solver.nx, g:g + solver.ny])).to(t.device)


def ch_solve(solver, alpha0, rhs):
    """The CH implicit solve on an interior-shaped (nx, ny) right-hand side; differentiable in rhs."""
    return CHSolve.apply(solver, alpha0, rhs)


class ExplicitOperator(torch.autograd.Function):
    """E(c, u, v), the CH explicit operator of the phase step (dn_explicit_operator); backward
    dn_explicit_operator_adjoint."""

    @staticmethod
    def forward(ctx, solver, c, u, v):
        ins = [_full(solver, c, "c"), _full(solver, u, "u"), _full(solver, v, "v")]
        out = torch.empty_like(ins[0])
        torch.cuda.current_stream().synchronize()
        solver._check(solver._lib.dn_explicit_operator(solver._h, *[t.data_ptr() for t in ins], out.data_ptr()))
        ctx.solver = solver
        ctx.save_for_backward(*ins)
        return _interior(solver, out)

    @staticmethod
    def backward(ctx, g):
        solver = ctx.solver
        cf, uf, vf = ctx.saved_tensors
        gf = _full(solver, g.to(torch.float64).contiguous(), "c")
        outs = [torch.empty_like(cf), torch.empty_like(uf), torch.empty_like(vf)]
        torch.cuda.current_stream().synchronize()
        solver._check(solver._lib.dn_explicit_operator_adjoint(solver._h, cf.data_ptr(), uf.data_ptr(),
                                                               vf.data_ptr(), gf.data_ptr(),
                                                               *[t.data_ptr() for t in outs]))
        return (None,) + tuple(_interior(solver, b) for b in outs)


def explicit_operator(solver, c, u, v):
    """The CH explicit operator E(c, u, v); differentiable in c, u and v."""
    return ExplicitOperator.apply(solver, c, u, v)


def ch_phase(solver, step, c, u, v, c_prev2=None, e_prev=None):
    """c at the end of the CH phase of step `step` (advance_phase_state, phase_field.cpp:258-281, with
    c_prev = c as the step's history copy leaves it): A^-1 (c / dt + E) on step 0 and
    A^-1 ((4 c - c_prev2) / (2 dt) + 2 E - E_prev) after, A = alpha0 I - beta1 L + beta2 L^2 with alpha0 = 1/dt
    or 3/(2 dt).  Composed from explicit_operator and ch_solve, so its gradient in c, u, v, c_prev2 and
    E_prev is the discrete adjoint of the phase."""
    dt = solver.config.dt
    e = explicit_operator(solver, c, u, v)
    if step == 0:
        return ch_solve(solver, 1.0 / dt, c / dt + e)
    return ch_solve(solver, 3.0 / (2.0 * dt), (4.0 * c - c_prev2) / (2.0 * dt) + 2.0 * e - e_prev)


def _ch_segment(solver, first_step, count, u, v, c, c_old, e_prev):
    """`count` CH phases from step `first_step` at fixed velocity; returns the state (c, c_old, e_prev)."""
    dt = solver.config.dt
    for k in range(first_step, first_step + count):
        e = explicit_operator(solver, c, u, v)
        if k == 0:
            c_new = ch_solve(solver, 1.0 / dt, c / dt + e)
        else:
            c_new = ch_solve(solver, 3.0 / (2.0 * dt), (4.0 * c - c_old) / (2.0 * dt) + 2.0 * e - e_prev)
        c, c_old, e_prev = c_new, c, e
    return c, c_old, e_prev


def ch_rollout(solver, c0, u, v, steps, checkpoint_every=0):
    """c after `steps` CH phases from c0 (step 0 onwards) with the velocity held at (u, v): the CH part of
    the time step (BDF1 then BDF2 with the AB2 explicit operator) rolled out over a horizon.  With
    checkpoint_every = K > 0 the backward keeps only every K-th state and recomputes each segment of K steps
    from it (torch.utils.checkpoint), so memory grows with steps / K + K rather than with steps."""
    from torch.utils.checkpoint import checkpoint

    state = (c0, torch.zeros_like(c0), torch.zeros_like(c0))
    k = 0
    while k < steps:
        n = min(checkpoint_every, steps - k) if checkpoint_every > 0 else steps - k
        if checkpoint_every > 0:
            state = checkpoint(lambda a, b, c_, d, e, k0=k, m=n: _ch_segment(solver, k0, m, a, b, c_, d, e),
                               u, v, *state, use_reentrant=False)
        else:
            state = _ch_segment(solver, k, n, u, v, *state)
        k += n
    return state[0]
