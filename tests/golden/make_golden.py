"""Reduce the reference's published golden run into small committed fixtures.

Source: the reference project's ``176Result/static_droplet_surface_tension_validation_128/`` (a 5000-step
run of case 92: 128x128, doubly periodic, icpcg, dt=2e-7) and the case file that produced it, which
ships inside ``ding_nsch_buildable_source_90c0805_2026-04-12.tar.gz`` as
``testcases/92_static_droplet_surface_tension_validation_128.cfg``.

Outputs (next to this script):
  case92.cfg           -- the case file, verbatim
  case92_history.csv   -- per-step diagnostics for steps 0..40 and every 50th step, 17 significant digits
  case92_final.npz     -- final cell fields (c, p, mu, cell-centred u, v) subsampled every 4th cell in i and j,
                          plus full-field sum / sum of squares / max-abs of each column

Run once in a container that has the reference mounted:
  python tests/golden/make_golden.py [/path/to/reference]
"""
import csv
import io
import os
import sys
import tarfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DN_REFERENCE", "")
if not REF or not os.path.isdir(REF):
    sys.exit("give the reference tree as the argument or in DN_REFERENCE")
RUN = os.path.join(REF, "176Result", "static_droplet_surface_tension_validation_128")
TARBALL = os.path.join(REF, "ding_nsch_buildable_source_90c0805_2026-04-12.tar.gz")
CFG_MEMBER = "testcases/92_static_droplet_surface_tension_validation_128.cfg"

HISTORY_COLUMNS = [
    "step", "mass", "mass_drift", "divergence_l2", "max_divergence", "max_abs_mu", "max_velocity",
    "kinetic_energy", "total_free_energy", "ch_inner_residual", "ch_equation_residual",
    "pressure_correction_residual", "momentum_residual", "ch_iterations", "pressure_iterations",
    "momentum_iterations",
]
FIELD_COLUMNS = ["c", "pressure", "chemical_potential", "u", "v"]


def main():
    with tarfile.open(TARBALL) as tf:
        member = [m for m in tf.getmembers() if m.name.endswith(CFG_MEMBER)][0]
        cfg_text = tf.extractfile(member).read().decode()
    with open(os.path.join(HERE, "case92.cfg"), "w") as f:
        f.write(cfg_text)

    with open(os.path.join(RUN, "history.csv")) as f:
        rows = list(csv.DictReader(f))
    keep = [r for r in rows if int(r["step"]) <= 40 or int(r["step"]) % 50 == 0]
    out = io.StringIO()
    w = csv.writer(out, lineterminator="\n")
    w.writerow(HISTORY_COLUMNS)
    for r in keep:
        w.writerow([r[c] for c in HISTORY_COLUMNS])
    with open(os.path.join(HERE, "case92_history.csv"), "w") as f:
        f.write(out.getvalue())

    with open(os.path.join(RUN, "final_cell_fields.csv")) as f:
        rows = list(csv.DictReader(f))
    nx = max(int(r["i"]) for r in rows) + 1
    ny = max(int(r["j"]) for r in rows) + 1
    arrays = {}
    for c in FIELD_COLUMNS:
        a = np.zeros((nx, ny))
        for r in rows:
            a[int(r["i"]), int(r["j"])] = float(r[c])
        arrays[c] = a
    payload = {"nx": nx, "ny": ny, "stride": 4}
    for c, a in arrays.items():
        payload[f"{c}_sub"] = a[::4, ::4].copy()
        payload[f"{c}_sum"] = float(a.sum())
        payload[f"{c}_sumsq"] = float((a * a).sum())
        payload[f"{c}_maxabs"] = float(np.abs(a).max())
    np.savez_compressed(os.path.join(HERE, "case92_final.npz"), **payload)
    print("wrote", len(keep), "history rows and", len(FIELD_COLUMNS), "final fields")

    # the reference's case files that the config-parser test reads (smoke, static droplets, shear droplets,
    # rising bubbles), copied as they are
    import glob
    import shutil

    dst = os.path.join(HERE, "testcases")
    os.makedirs(dst, exist_ok=True)
    names = sorted(glob.glob(os.path.join(REF, "testcases", "0[4-9]*.cfg")) +
                   glob.glob(os.path.join(REF, "testcases", "2[4-6]*.cfg")))
    for path in names:
        shutil.copyfile(path, os.path.join(dst, os.path.basename(path)))
    print("copied", len(names), "case files")


if __name__ == "__main__":
    main()
