"""Reference FP64 adjoint of the pressure projection -- test infrastructure, never product code.

The reference has no adjoint.  Its projection -- the pressure solve and the velocity correction of one step
(solve_pressure_correction, pressure.cpp:1031-1089; apply_pressure_velocity_correction,
operators.cpp:480-534), restated in dn_oracle.c (pressure_solve, velocity_correction) -- is, at fixed rho_mid,
an affine map of the interior values

    (u*, v*, p, p_prev)  ->  (u, v, p_new, p_prev_new).

Its Jacobian is therefore J e_k = F(e_k) - F(0), column by column, exact up to the solver tolerance, and
J^T applied to a cotangent is the reference adjoint the CUDA transpose is checked against.  Nothing here
transposes anything by hand, so it shares no derivation with the CUDA kernels.
"""
import numpy as np

from .oracle import OracleSolver

INPUTS = ("u_star", "v_star", "p", "p_prev")
OUTPUTS = ("u", "v", "p", "p_prev")  # p_new, p_prev_new are the oracle's p, p_prev after the correction


def interior_shapes(cfg):
    nx, ny = cfg["nx"], cfg["ny"]
    return {"u": (nx + 1, ny), "v": (nx, ny + 1), "c": (nx, ny)}


def _in_shape(cfg, name):
    s = interior_shapes(cfg)
    return s["u"] if name == "u_star" else s["v"] if name == "v_star" else s["c"]


def _out_shape(cfg, name):
    s = interior_shapes(cfg)
    return s["u"] if name == "u" else s["v"] if name == "v" else s["c"]


class ProjectionOracle:
    """The oracle's projection on interior arrays, with rho_mid (a full Field2D array) held fixed."""

    def __init__(self, cfg, rho_mid_full, step):
        self.cfg, self.step = cfg, int(step)
        self.orc = OracleSolver(cfg, "port")
        self.orc.initialize()
        self.orc.begin_step(self.step)
        self.rho = np.array(rho_mid_full, dtype=np.float64)
        self.g = cfg["ghost"]

    def close(self):
        self.orc.close()

    def __call__(self, u_star, v_star, p, p_prev):
        g, o = self.g, self.orc
        o.set_field("rho_mid", self.rho)
        for name, a in zip(INPUTS, (u_star, v_star, p, p_prev)):
            f = np.zeros_like(o.field(name))
            f[g:f.shape[0] - g, g:f.shape[1] - g] = a
            o.set_field(name, f)
        o.pressure()
        o.correct()
        iters = o.report()["pressure_iterations"]
        return tuple(o.interior(n).copy() for n in OUTPUTS), iters

    def jacobian(self):
        """Dense J (rows: outputs u, v, p_new, p_prev_new flattened; columns: inputs u*, v*, p, p_prev)."""
        zeros = [np.zeros(_in_shape(self.cfg, n)) for n in INPUTS]
        base = np.concatenate([a.ravel() for a in self(*zeros)[0]])
        cols = []
        for k, name in enumerate(INPUTS):
            for idx in range(zeros[k].size):
                args = [z.copy() for z in zeros]
                args[k].flat[idx] = 1.0
                out = np.concatenate([a.ravel() for a in self(*args)[0]])
                cols.append(out - base)
        return np.stack(cols, axis=1)


def split_cotangent(cfg, vec):
    """Split a flat input-space vector into (u*, v*, p, p_prev) interior arrays."""
    out, k = [], 0
    for name in INPUTS:
        shp = _in_shape(cfg, name)
        n = shp[0] * shp[1]
        out.append(vec[k:k + n].reshape(shp))
        k += n
    return out


def flat_outputs(arrs):
    return np.concatenate([np.asarray(a).ravel() for a in arrs])


def output_shapes(cfg):
    return [_out_shape(cfg, n) for n in OUTPUTS]


def input_shapes(cfg):
    return [_in_shape(cfg, n) for n in INPUTS]
