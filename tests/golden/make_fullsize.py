"""Writes tests/golden/bubble_1024x2048_step0.npz: one time step of the 1024x2048 rising bubble on the CPU.

The workload is the bench's rising bubble (R0-unit parameters of the reference's testcase 26, split_icpcg,
seeded interface modes 2-8) refined to 1024 x 2048, from the seeded initial state that bench.py builds.  The
reference build (oracle/_ref, the reference's own sources) advances it by step 0 (about 5 minutes on one
core); the port is used when the reference build is absent.  A full field is 17 MB, so the fixture keeps, per
field, the values at 8192 seeded cells together with the field's full L2 norm, plus the step's iteration
counts.  The GPU test regenerates the same initial state, takes the same step and compares the sampled
cells (relative L2 over the sample) and the norms.

With --tight the same step is taken at ch/pressure tolerance 1e-13 and momentum tolerance 1e-14 (iteration
caps lifted) and written as bubble_<grid>_step0_tight.npz: the step solved well below the reference's own
solver error, which the mixed-precision form is compared against beside the reference's answer.

    python tests/golden/make_fullsize.py [--impl reference|port] [--grid 1024x2048] [--tight]
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

FIELDS = ("c", "mu", "u", "v", "p")
SAMPLES = 8192


def sample_index(shape, g, seed=7, count=SAMPLES):
    """Seeded interior cells (i, j) of a ghosted array of `shape` (ghost width g)."""
    rng = np.random.default_rng(seed)
    ni, nj = shape[0] - 2 * g, shape[1] - 2 * g
    return rng.integers(0, ni, count) + g, rng.integers(0, nj, count) + g


def main():
    import bench
    from oracle.oracle import OracleSolver, available, with_defaults

    ap = argparse.ArgumentParser()
    ap.add_argument("--impl", default="reference" if available("reference") else "port")
    ap.add_argument("--grid", default="1024x2048")
    ap.add_argument("--tight", action="store_true")
    args = ap.parse_args()
    grid = tuple(int(v) for v in args.grid.split("x"))
    cfg = bench.workload_cfg(grid)
    state = bench.initial_state(cfg)
    run_cfg = dict(cfg)
    if args.tight:
        run_cfg.update(ch_tolerance=1e-13, pressure_tolerance=1e-13, momentum_tolerance=1e-14,
                       ch_inner_iterations=100000, poisson_iterations=100000, momentum_iterations=10000)
    orc = OracleSolver(with_defaults(run_cfg), args.impl)
    orc.initialize()
    for n, a in state.items():
        orc.set_field(n, a)
    orc.refresh_derived()
    orc.set_initial_mass(0.0)
    t0 = time.time()
    orc.step(0)
    sec = time.time() - t0
    rep = orc.report()
    g = cfg["ghost"]
    out = {"grid": np.array(grid), "seconds": np.array(sec), "impl": np.array(args.impl)}
    for k in ("ch_iterations", "momentum_iterations", "pressure_iterations"):
        out[k] = np.array(rep[k])
    for name in FIELDS:
        a = orc.field(name)
        ii, jj = sample_index(a.shape, g)
        out[name + "_i"] = ii.astype(np.int32)
        out[name + "_j"] = jj.astype(np.int32)
        out[name + "_val"] = a[ii, jj].copy()
        out[name + "_norm"] = np.array(np.linalg.norm(a[g:a.shape[0] - g, g:a.shape[1] - g]))
    path = os.path.join(HERE, f"bubble_{grid[0]}x{grid[1]}_step0{'_tight' if args.tight else ''}.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {args.impl}, {sec:.1f} s, iterations ch {rep['ch_iterations']} "
          f"mom {rep['momentum_iterations']} p {rep['pressure_iterations']}")


if __name__ == "__main__":
    main()
