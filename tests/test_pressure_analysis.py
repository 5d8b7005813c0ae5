"""The pressure analysis files (Solver::run_pressure_analysis_from_snapshot, pressure_analysis.cpp:156-328)
written by the CUDA path, against the files the reference itself wrote for the same state
(tests/golden/pressure_analysis/, made by make_pressure_analysis.py from oracle/_ref).

Bars: names, strings, integers, the config-derived numbers and the fields copied from the state (rho_mid,
phi, the interface mask) equal, character for character; the iteration count equal; the per-iteration
residuals, alpha, beta and q_k within 1e-6 relative (the CG trajectories of two summation orders); the
residual fields within 1e-6 of their largest entry.
"""
import csv
import glob
import json
import os

import numpy as np
import pytest

from ding_nsch_core_solver_b200 import capi

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "pressure_analysis")
CASES = sorted(os.listdir(GOLDEN)) if os.path.isdir(GOLDEN) else []
# columns of <stem>_pcg.csv compared as text (names, integers, config-derived numbers)
PCG_TEXT = set(range(0, 15))
SUMMARY_TEXT = set(range(0, 14)) | {18, 19}


def _case(case):
    d = os.path.join(GOLDEN, case)
    cfg = json.load(open(os.path.join(d, "cfg.json")))
    state = np.load(os.path.join(d, "state.npz"))
    return d, cfg, state


def _rows(path):
    with open(path, newline="") as f:
        return list(csv.reader(f))


def _close(got, ref, rtol, atol):
    g, r = float(got), float(ref)
    return abs(g - r) <= rtol * abs(r) + atol


def _rhs_scale(ref_dir):
    """max |rhs| x cells of the analysed system: the size of the rounding noise of its sums."""
    rhs = np.array(_rows(glob.glob(os.path.join(ref_dir, "*_fields", "rhs.csv"))[0]), dtype=float)
    return float(np.abs(rhs).max()) * rhs.size


def compare_dirs(got_dir, ref_dir, rtol=1e-6, exact_state=True):
    """Every file of `got_dir` against `ref_dir`.  `exact_state`: the analysed state was injected bit for bit,
    so the fields printed from it match as text; otherwise they match to 1e-8 of their largest entry."""
    ref_files = sorted(os.path.relpath(p, ref_dir) for p in glob.glob(os.path.join(ref_dir, "**", "*"), recursive=True)
                       if os.path.isfile(p))
    got_files = sorted(os.path.relpath(p, got_dir) for p in glob.glob(os.path.join(got_dir, "**", "*"), recursive=True)
                       if os.path.isfile(p))
    assert got_files == ref_files
    for rel in ref_files:
        g, r = _rows(os.path.join(got_dir, rel)), _rows(os.path.join(ref_dir, rel))
        assert len(g) == len(r), (rel, len(g), len(r))
        name = os.path.basename(rel)
        if name.endswith("_pcg.csv") or name == "summary.csv":
            assert g[0] == r[0], rel
            text = PCG_TEXT if name.endswith("_pcg.csv") else SUMMARY_TEXT
            cols = list(zip(*[[float(v) for k, v in enumerate(row) if k not in text] for row in r[1:]]))
            scale = [max(abs(v) for v in c) for c in cols]
            noise = 1e-12 * _rhs_scale(ref_dir)
            for gr, rr in zip(g[1:], r[1:]):
                assert [v for k, v in enumerate(gr) if k in text] == [v for k, v in enumerate(rr) if k in text], rel
                num = [(a, b) for k, (a, b) in enumerate(zip(gr, rr)) if k not in text]
                for q, (a, b) in enumerate(num):
                    # the summary's rhs and pressure means of a projected system are rounding noise: absolute
                    # against the size of that noise
                    atol = noise if name == "summary.csv" and q < 4 else 1e-12 * max(scale[q], 1e-300)
                    assert _close(a, b, rtol, atol), (rel, rr[14], q, a, b)
        elif name == "interface_mask.csv" or (exact_state and name in ("rho_mid.csv", "phi.csv")):
            assert g == r, rel
        else:  # rhs, residual_iter_*, residual_final
            ga = np.array(g, dtype=float)
            ra = np.array(r, dtype=float)
            assert ga.shape == ra.shape
            tol = (1e-9 if name == "rhs.csv" and exact_state else 1e-8 if name in ("rho_mid.csv", "phi.csv")
                   else 1e-6) * np.abs(ra).max() + 1e-300
            if name == "residual_final.csv":  # both at the solver tolerance: compare against the rhs scale
                rhs = np.array(_rows(os.path.join(ref_dir, os.path.dirname(rel), "rhs.csv")), dtype=float)
                tol = 1e-8 * np.abs(rhs).max()
            assert np.abs(ga - ra).max() <= tol, (rel, np.abs(ga - ra).max(), tol)


def test_golden_fixtures_present():
    assert CASES, "tests/golden/pressure_analysis is missing"
    for case in CASES:
        d, cfg, state = _case(case)
        files = os.path.join(d, "files")
        assert os.path.isfile(os.path.join(files, "summary.csv"))
        assert len(glob.glob(os.path.join(files, "*_pcg.csv"))) == 1
        for name in ("c", "rho_mid", "u_star", "v_star", "p", "p_prev"):
            assert name in state.files


def test_analysis_config_keys():
    c = capi.parse_config("name = bubble\noutput_dir = out/x\nanalysis_enabled = true\nanalysis_mode = Both\n"
                          "analysis_trigger_step = 7\nanalysis_spectrum_iterations = 0, 4 ,final\n"
                          "analysis_interface_band_multiplier = 3.5\nanalysis_case_group = g1\n")
    assert c.name == b"bubble" and c.output_dir == b"out/x" and c.analysis_enabled == 1
    assert c.analysis_mode == 3 and c.analysis_trigger_step == 7 and c.analysis_interface_band_multiplier == 3.5
    assert c.analysis_spectrum_iterations == b"0, 4 ,final" and c.analysis_case_group == b"g1"
    d = capi.parse_config("nx = 32\n")
    assert d.name == b"unnamed" and d.output_dir == b"output" and d.analysis_enabled == 0 and d.analysis_mode == 0
    assert d.analysis_initial_guess == b"zero" and d.analysis_nullspace_treatment == b"zero_mean_projection"
    assert capi.parse_config("analysis_mode = sometimes\n").analysis_mode == 0
    with pytest.raises(capi.DnError):
        capi.parse_config("name = " + "x" * 200 + "\n")


def test_reference_rewrites_the_fixtures(tmp_path):
    """The committed files are what the reference build writes for the committed state (pins the fixture)."""
    from oracle.oracle import OracleSolver, available

    if not available("reference"):
        pytest.skip("oracle/_ref is not built")
    case = CASES[0]
    d, cfg, state = _case(case)
    ref = OracleSolver({k: v for k, v in cfg.items() if not k.startswith("analysis_") and k != "name"}, "reference")
    try:
        ref.initialize()
        for n in state.files:
            if n.startswith("init_"):
                continue
            ref.set_field(n, state[n])
        ref.begin_step(1)
        ref.pressure_analysis(1, "frozen", str(tmp_path), case, cfg["analysis_case_group"],
                              cfg["analysis_spectrum_iterations"], cfg["analysis_interface_band_multiplier"])
    finally:
        ref.close()
    compare_dirs(str(tmp_path / case / "pressure_analysis"), os.path.join(d, "files"), rtol=0.0)


def _solver(cfg, tmp_path, **kw):
    return capi.Solver(dict(cfg, output_dir=str(tmp_path), **kw))


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_analysis_files_match_the_reference(case, tmp_path):
    d, cfg, state = _case(case)
    s = _solver(cfg, tmp_path)
    try:
        s.initialize()
        for n in ("c", "rho_mid", "u_star", "v_star", "p", "p_prev"):
            s.set_field(n, state[n])
        s.pressure_analysis(1, "frozen")
    finally:
        s.close()
    compare_dirs(str(tmp_path / case / "pressure_analysis"), os.path.join(d, "files"))


@pytest.mark.gpu
def test_step_runs_frozen_and_online_analysis_at_the_trigger_step(tmp_path):
    case = next(c for c in CASES if "init_c" in np.load(os.path.join(GOLDEN, c, "state.npz")).files)
    d, cfg, state = _case(case)
    s = _solver(cfg, tmp_path, analysis_enabled=True, analysis_mode="both", analysis_trigger_step=2)
    try:
        for n in capi.FIELDS:
            s.set_field(n, state["init_" + n])
        s.set_initial_mass(0.0)
        s.step(0)
        out = tmp_path / case / "pressure_analysis"
        assert not out.exists()  # step 1 (index 0) is not the trigger step
        s.step(1)
    finally:
        s.close()
    stems = sorted(p.name for p in out.iterdir())
    assert stems == [f"{case}_frozen_step_000002_fields", f"{case}_frozen_step_000002_pcg.csv",
                     f"{case}_online_step_000002_fields", f"{case}_online_step_000002_pcg.csv", "summary.csv"]
    frozen = _rows(out / f"{case}_frozen_step_000002_pcg.csv")
    online = _rows(out / f"{case}_online_step_000002_pcg.csv")
    # the online analysis sees the same system after the solve: the same numbers, another source_mode
    assert [r[:2] + r[3:] for r in frozen] == [r[:2] + r[3:] for r in online]
    assert [r[2] for r in online[1:]] == ["online"] * (len(online) - 1)
    summary = _rows(out / "summary.csv")
    assert len(summary) == 3 and [r[2] for r in summary[1:]] == ["frozen", "online"]
    # the state the CUDA step reached is the reference's to 1e-10, so the frozen files match the golden ones
    got = tmp_path / "frozen_only"
    os.makedirs(got)
    for p in out.iterdir():
        if "frozen" in p.name:
            os.rename(p, got / p.name)
    with open(got / "summary.csv", "w", newline="") as f:
        csv.writer(f, lineterminator="\n").writerows(summary[:2])
    compare_dirs(str(got), os.path.join(d, "files"), rtol=1e-5, exact_state=False)
