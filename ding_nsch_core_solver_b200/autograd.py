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
    """(u, v, hu_prev, hv_prev, fxu, fyv, rho_mid, eta, eta_prev) -> (u_star, v_star, hu, hv) through
    dn_momentum_map (hu, hv: this step's convection H, the next step's H_prev); backward is
    dn_momentum_adjoint, whose transposed coupled solve is the same Jacobi-BiCGSTAB on M^T."""

    KINDS = ("u", "v", "u", "v", "u", "v", "c", "c", "c")

    @staticmethod
    def forward(ctx, solver, step, *args):
        ins = [_full(solver, t.to(torch.float64).contiguous(), k) for t, k in zip(args, MomentumPredictor.KINDS)]
        outs = [torch.empty_like(ins[0]), torch.empty_like(ins[1]), torch.empty_like(ins[0]),
                torch.empty_like(ins[1])]
        its, res = _call(solver, solver._lib.dn_momentum_map, step, ins, outs)
        ctx.solver, ctx.step = solver, int(step)
        ctx.save_for_backward(*ins, outs[0], outs[1])
        ctx.forward_report = (its, res)
        return tuple(_interior(solver, b) for b in outs)

    @staticmethod
    def backward(ctx, gus, gvs, ghu, ghv):
        solver = ctx.solver
        saved = ctx.saved_tensors
        u, v, hup, hvp, _, _, rho, eta, etap, us, vs = saved
        shapes = {"u": (solver.nx + 1, solver.ny), "v": (solver.nx, solver.ny + 1)}
        cot = []
        for g_, kind in ((gus, "u"), (gvs, "v"), (ghu, "u"), (ghv, "v")):
            if g_ is None:
                g_ = torch.zeros(shapes[kind], dtype=torch.float64, device="cuda")
            cot.append(_full(solver, g_.to(torch.float64).contiguous(), kind))
        outs = [torch.empty_like(b) for b in (u, v, u, v, u, v, rho, rho, rho)]
        _call(solver, solver._lib.dn_momentum_adjoint, ctx.step, [u, v, hup, hvp, rho, eta, etap, us, vs] + cot, outs)
        grads = [_interior(solver, b) for b in outs]
        # order of the forward's inputs: u, v, hu_prev, hv_prev, fxu, fyv, rho_mid, eta, eta_prev
        return (None, None) + tuple(grads)


def momentum_predictor(solver, step, u, v, hu_prev, hv_prev, fxu, fyv, rho_mid=None, eta=None, eta_prev=None):
    """(u_star, v_star, hu, hv) of the momentum predictor; differentiable in every input.  The materials
    default to the solver's current rho_mid, eta, eta_prev (then constants).  Surface-tension parameters enter
    through fxu, fyv, which are linear in the surface_tension_multiplier sigma."""
    g = solver.ghost
    mats = []
    for t, name in ((rho_mid, "rho_mid"), (eta, "eta"), (eta_prev, "eta_prev")):
        if t is None:
            a = solver.get_field(name)
            t = torch.tensor(a[g:a.shape[0] - g, g:a.shape[1] - g].copy(), dtype=torch.float64, device="cuda")
        mats.append(t)
    return MomentumPredictor.apply(solver, step, u, v, hu_prev, hv_prev, fxu, fyv, *mats)


def velocity_step(solver, step, u, v, hu_prev, hv_prev, fxu, fyv, p, p_prev):
    """The velocity half of a step at fixed phase: the momentum predictor, then the projection.  Returns
    (u, v, p_new, p_prev_new); differentiable in all inputs (rho_mid, eta, eta_prev fixed)."""
    us, vs, _, _ = momentum_predictor(solver, step, u, v, hu_prev, hv_prev, fxu, fyv)
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


class SurfaceForce(torch.autograd.Function):
    """(c_old, c_new) -> (fxu, fyv), the face surface forces (dn_surface_force_map); backward is
    dn_surface_force_adjoint (c_mid, its chemical potential and the face stencils, transposed)."""

    @staticmethod
    def forward(ctx, solver, c_old, c_new):
        ins = [_full(solver, c_old.to(torch.float64).contiguous(), "c"),
               _full(solver, c_new.to(torch.float64).contiguous(), "c")]
        nx, ny, g = solver.nx, solver.ny, solver.ghost
        outs = [torch.empty((nx + 1 + 2 * g, ny + 2 * g), dtype=torch.float64, device=c_old.device),
                torch.empty((nx + 2 * g, ny + 1 + 2 * g), dtype=torch.float64, device=c_old.device)]
        torch.cuda.current_stream().synchronize()
        solver._check(solver._lib.dn_surface_force_map(solver._h, *[t.data_ptr() for t in ins + outs]))
        ctx.solver = solver
        ctx.save_for_backward(*ins)
        return tuple(_interior(solver, b) for b in outs)

    @staticmethod
    def backward(ctx, gfu, gfv):
        solver = ctx.solver
        co, cn = ctx.saved_tensors
        shapes = {"u": (solver.nx + 1, solver.ny), "v": (solver.nx, solver.ny + 1)}
        cot = []
        for g_, kind in ((gfu, "u"), (gfv, "v")):
            if g_ is None:
                g_ = torch.zeros(shapes[kind], dtype=torch.float64, device="cuda")
            cot.append(_full(solver, g_.to(torch.float64).contiguous(), kind))
        outs = [torch.empty_like(co), torch.empty_like(cn)]
        torch.cuda.current_stream().synchronize()
        solver._check(solver._lib.dn_surface_force_adjoint(solver._h, *[t.data_ptr() for t in [co, cn] + cot + outs]))
        return None, _interior(solver, outs[0]), _interior(solver, outs[1])


def surface_force(solver, c_old, c_new):
    """The face surface forces (fxu, fyv) of a step; differentiable in c_old and c_new."""
    return SurfaceForce.apply(solver, c_old, c_new)


def materials(solver, c):
    """(rho, eta) of c (update_materials_from_phase, phase_field.cpp:57-66): c + (1 - c) * ratio."""
    cfg = solver.config
    return c + (1.0 - c) * cfg.density_ratio, c + (1.0 - c) * cfg.viscosity_ratio


FULL_STATE = ("c", "c_old", "e_prev", "u", "v", "p", "p_prev", "hu_prev", "hv_prev")


def full_step(solver, step, st, sigma_scale=None, inv_pe_scale=None):
    """One whole time step (advance_one_timestep, solver.cpp:224-283, without the history copies' side
    effects) as a composition of the differentiable maps: the CH phase (explicit operator + implicit
    solve), the materials and rho_mid, the surface force, the momentum predictor and the projection.
    `st` maps FULL_STATE to interior tensors (c_old: c at the previous step's start; e_prev: the previous
    explicit operator); returns the next state.  Gradients flow to every state entry.

    sigma_scale (a 0-d tensor, value 1 at the solver's surface_tension_multiplier) scales the surface force,
    which is linear in sigma; inv_pe_scale (value 1 at the solver's 1/Pe) scales the mobility: the explicit
    operator's mobility part E - (-div(u c)) is linear in 1/Pe, and the CH matrix is alpha0 I + (1/Pe) K', so
    its solve's derivative follows from the same solve (ch_solve_mobility)."""
    dt = solver.config.dt
    c, u, v = st["c"], st["u"], st["v"]
    e = explicit_operator(solver, c, u, v)
    if inv_pe_scale is not None:
        adv = advection(solver, c, u, v)
        e = adv + inv_pe_scale * (e - adv)
    if step == 0:
        alpha0, rhs = 1.0 / dt, c / dt + e
    else:
        alpha0, rhs = 3.0 / (2.0 * dt), (4.0 * c - st["c_old"]) / (2.0 * dt) + 2.0 * e - st["e_prev"]
    c_new = ch_solve(solver, alpha0, rhs) if inv_pe_scale is None else ch_solve_mobility(solver, alpha0, rhs,
                                                                                          inv_pe_scale)
    rho_old, eta_old = materials(solver, c)
    rho_new, eta_new = materials(solver, c_new)
    rho_mid = 0.5 * (rho_old + rho_new)
    fxu, fyv = surface_force(solver, c, c_new)
    if sigma_scale is not None:
        fxu, fyv = sigma_scale * fxu, sigma_scale * fyv
    us, vs, hu, hv = momentum_predictor(solver, step, u, v, st["hu_prev"], st["hv_prev"], fxu, fyv, rho_mid,
                                        eta_new, eta_old)
    un, vn, pn, ppn = projection_rho(solver, step, us, vs, st["p"], st["p_prev"], rho_mid)
    return {"c": c_new, "c_old": c, "e_prev": e, "u": un, "v": vn, "p": pn, "p_prev": ppn, "hu_prev": hu,
            "hv_prev": hv}


class CHSolveMobility(torch.autograd.Function):
    """c = A(s)^-1 rhs with A(s) = alpha0 I + s (A - alpha0 I), evaluated at s = 1 (the solver's 1/Pe): the
    CH matrix alpha0 I - (a1/Pe) L + (a2/Pe) L^2 is alpha0 I plus 1/Pe times a fixed matrix, so s scales the
    mobility.  dc/ds = -A^-1 (A - alpha0 I) c, hence dL/ds = -(lam . rhs - alpha0 lam . c) with lam = A^-1 g:
    the same solve as the rhs cotangent, nothing more."""

    @staticmethod
    def forward(ctx, solver, alpha0, rhs, s):
        c = _ch_solve(solver, float(alpha0), rhs)
        ctx.solver, ctx.alpha0 = solver, float(alpha0)
        ctx.save_for_backward(rhs, c)
        return c

    @staticmethod
    def backward(ctx, g):
        rhs, c = ctx.saved_tensors
        lam = _ch_solve(ctx.solver, ctx.alpha0, g)
        gs = -((lam * rhs).sum() - ctx.alpha0 * (lam * c).sum())
        return None, None, lam, gs


def ch_solve_mobility(solver, alpha0, rhs, s):
    return CHSolveMobility.apply(solver, alpha0, rhs, s)


class ProjectionRho(torch.autograd.Function):
    """The projection (dn_projection_rho) with rho_mid as a differentiable input: (u_star, v_star, p, p_prev,
    rho_mid) -> (u, v, p_new, p_prev_new); backward dn_projection_rho_adjoint (the transposed pressure solve,
    plus the rho_mid terms of the operator, the split explicit divergence and the correction)."""

    @staticmethod
    def forward(ctx, solver, step, u_star, v_star, p, p_prev, rho_mid):
        ins = [_full(solver, t.to(torch.float64).contiguous(), k)
               for t, k in zip((u_star, v_star, p, p_prev, rho_mid), ("u", "v", "c", "c", "c"))]
        outs = [torch.empty_like(ins[0]), torch.empty_like(ins[1]), torch.empty_like(ins[2]), torch.empty_like(ins[2])]
        _call(solver, solver._lib.dn_projection_rho, step, ins, outs)
        ctx.solver, ctx.step = solver, int(step)
        ctx.save_for_backward(ins[4], ins[2], ins[3], outs[2])
        return tuple(_interior(solver, b) for b in outs)

    @staticmethod
    def backward(ctx, gu, gv, gp, gpp):
        solver = ctx.solver
        rho, p, pp, pnew = ctx.saved_tensors
        shapes = {"u": (solver.nx + 1, solver.ny), "v": (solver.nx, solver.ny + 1), "c": (solver.nx, solver.ny)}
        cot = []
        for g_, kind in zip((gu, gv, gp, gpp), ("u", "v", "c", "c")):
            if g_ is None:
                g_ = torch.zeros(shapes[kind], dtype=torch.float64, device="cuda")
            cot.append(_full(solver, g_.to(torch.float64).contiguous(), kind))
        outs = [torch.empty_like(cot[0]), torch.empty_like(cot[1]), torch.empty_like(p), torch.empty_like(p),
                torch.empty_like(p)]
        _call(solver, solver._lib.dn_projection_rho_adjoint, ctx.step, [rho, p, pp, pnew] + cot, outs)
        return (None, None) + tuple(_interior(solver, b) for b in outs)


def projection_rho(solver, step, u_star, v_star, p, p_prev, rho_mid):
    return ProjectionRho.apply(solver, step, u_star, v_star, p, p_prev, rho_mid)


def taylor_deformation(c, dx, dy, clamp=True):
    """Taylor deformation D = (a - b) / (a + b) of the droplet c, from its second moments
    (compute_moment_taylor_ratio, python/postprocess_taylor_deformation.py:65-112): weights c clamped to
    [0, 1], centroid, covariance (mxx, myy, mxy), semi-axes 2 sqrt(eigenvalues).  Moments about the centroid
    do not depend on the grid's origin; cell (i, j) sits at (i dx, j dy).  Differentiable in c; the clamp is
    not differentiable where c touches 0 or 1 (a droplet's interior and exterior approach them to round-off),
    so clamp=False gives the smooth variant with weights c itself."""
    w = c.clamp(0.0, 1.0) if clamp else c
    nx, ny = c.shape
    x = (torch.arange(nx, dtype=c.dtype, device=c.device) * dx)[:, None]
    y = (torch.arange(ny, dtype=c.dtype, device=c.device) * dy)[None, :]
    mass = w.sum()
    xc, yc = (w * x).sum() / mass, (w * y).sum() / mass
    ddx, ddy = x - xc, y - yc
    mxx, myy, mxy = (w * ddx * ddx).sum() / mass, (w * ddy * ddy).sum() / mass, (w * ddx * ddy).sum() / mass
    tr, det = mxx + myy, mxx * myy - mxy * mxy
    disc = torch.sqrt(torch.clamp(0.25 * tr * tr - det, min=0.0))
    a = 2.0 * torch.sqrt(torch.clamp(0.5 * tr + disc, min=0.0))
    b = 2.0 * torch.sqrt(torch.clamp(0.5 * tr - disc, min=0.0))
    return (a - b) / (a + b)


def _full_segment(solver, first_step, count, sigma, mob, *state):
    st = dict(zip(FULL_STATE, state))
    for k in range(first_step, first_step + count):
        st = full_step(solver, k, st, sigma_scale=sigma, inv_pe_scale=mob)
    return tuple(st[n] for n in FULL_STATE)


def full_rollout(solver, state, first_step, steps, checkpoint_every=0, sigma_scale=None, inv_pe_scale=None):
    """`steps` whole time steps from `state` (a FULL_STATE dict) starting at step index `first_step`; returns
    the final state.  With checkpoint_every = K > 0 the backward keeps only every K-th state and recomputes
    each K-step segment from it (torch.utils.checkpoint), so memory grows with steps / K + K."""
    from torch.utils.checkpoint import checkpoint

    sig = sigma_scale if sigma_scale is not None else torch.tensor(1.0, dtype=torch.float64, device="cuda")
    mob = inv_pe_scale if inv_pe_scale is not None else torch.tensor(1.0, dtype=torch.float64, device="cuda")
    cur = tuple(state[n] for n in FULL_STATE)
    k = first_step
    end = first_step + steps
    while k < end:
        n = min(checkpoint_every, end - k) if checkpoint_every > 0 else end - k
        if checkpoint_every > 0:
            cur = checkpoint(lambda s_, m_, *a, k0=k, c0=n: _full_segment(solver, k0, c0, s_, m_, *a), sig, mob, *cur,
                             use_reentrant=False)
        else:
            cur = _full_segment(solver, k, n, sig, mob, *cur)
        k += n
    return dict(zip(FULL_STATE, cur))
