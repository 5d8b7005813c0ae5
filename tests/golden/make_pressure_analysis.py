"""Golden pressure-analysis files written by the reference itself (oracle/_ref, the reference's own sources
compiled by oracle/Makefile; Solver::run_pressure_analysis_from_snapshot, pressure_analysis.cpp:156-328).

For each case below: a seeded state (initialize, then seeded noise on c, u, v, p, derived fields rebuilt)
is advanced by the reference through step 0 and through the phase and momentum parts of step 1; the frozen
analysis then runs on that state (step index 1, files tagged step 2), as solver.cpp:270 runs it.

Outputs, under pressure_analysis/<case>/:
  state.npz          -- the fields the analysis reads in the analysed state (c, rho_mid, u_star, v_star, p,
                        p_prev), and, for the first case, every field of the seeded initial state
                        ("init_<field>"), from which the CUDA step reaches the analysed state itself
  cfg.json           -- the case's config keys
  files/             -- the reference's pressure_analysis/ directory for that state, verbatim

Run in a container that has the reference mounted and `make -C oracle` done:
  python tests/golden/make_pressure_analysis.py
"""
import json
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import FIELDS, OracleSolver, with_defaults  # noqa: E402

OUT = os.path.join(HERE, "pressure_analysis")
SPECTRUM = "0,1,3,final"
ANALYSED = ("c", "rho_mid", "u_star", "v_star", "p", "p_prev")
BAND = 2.0


def base(**kw):
    cfg = dict(nx=16, ny=12, ghost=3, dt=1.0e-3, periodic_x=True, periodic_y=True, poisson_iterations=5000,
               pressure_tolerance=1.0e-10, momentum_iterations=200, momentum_tolerance=1.0e-10, density_ratio=10.0,
               viscosity_ratio=5.0, ch_inner_iterations=200, ch_tolerance=1e-10, interface_radius=0.3,
               cn=0.08)
    cfg.update(kw)
    return with_defaults(cfg)


CASES = {
    # doubly periodic: the zero-mean projection is active
    "periodic_icpcg": base(pressure_scheme="icpcg"),
    # walls, split operator (constant coefficients), gravity
    "walls_split_icpcg": base(nx=20, ny=16, periodic_x=False, periodic_y=False, pressure_scheme="split_icpcg",
                              body_force_y=-0.98, dt=1e-4),
    # a Dirichlet pressure side (no projection) and the ILDLT factor
    "dirichlet_top_ildlt": base(nx=16, ny=20, periodic_x=False, periodic_y=False, pressure_scheme="ildlt_pcg",
                                dt=1e-4, pressure_bc_top_type="dirichlet", pressure_bc_top_value=0.3),
}


def seeded(cfg, seed=5):
    s = OracleSolver(cfg, "reference")
    s.initialize()
    rng = np.random.default_rng(seed)
    g = cfg["ghost"]
    for name, a in (("c", 0.02), ("u", 0.05), ("v", 0.05), ("p", 0.1)):
        f = s.field(name)
        f[g:-g, g:-g] += a * rng.standard_normal(f[g:-g, g:-g].shape)
    s.refresh_derived()
    s.set_initial_mass(0.0)
    return s


def main():
    for case, cfg in CASES.items():
        dst = os.path.join(OUT, case)
        if os.path.isdir(dst):
            shutil.rmtree(dst)
        os.makedirs(dst)
        s = seeded(cfg)
        init = {f"init_{n}": s.field(n).copy() for n in FIELDS} if case == next(iter(CASES)) else {}
        s.step(0)
        s.begin_step(1)
        s.phase(1)
        s.momentum(1)
        state = {n: s.field(n).copy() for n in ANALYSED}
        with tempfile.TemporaryDirectory() as tmp:
            s.pressure_analysis(1, "frozen", tmp, case, "golden", SPECTRUM, BAND)
            shutil.copytree(os.path.join(tmp, case, "pressure_analysis"), os.path.join(dst, "files"))
        s.close()
        np.savez_compressed(os.path.join(dst, "state.npz"), **init, **state)
        with open(os.path.join(dst, "cfg.json"), "w") as f:
            json.dump(dict(cfg, name=case, analysis_case_group="golden", analysis_spectrum_iterations=SPECTRUM,
                           analysis_interface_band_multiplier=BAND), f, indent=1, sort_keys=True)
        print(case, sorted(os.listdir(os.path.join(dst, "files"))))


if __name__ == "__main__":
    main()
