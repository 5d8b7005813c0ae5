"""Host-side checks of the C-ABI library (no GPU needed): it loads, exports every entry point that
include/dn_cuda.h declares, parses the reference's case files exactly like the reference's load_config,
and fails loudly (an error status, never a CPU fallback) when no device is present."""
import ctypes as C
import glob
import os
import subprocess

import pytest

from ding_nsch_core_solver_b200 import capi
from oracle.oracle import parse_cfg, PRESSURE, SIDES

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def lib():
    from ding_nsch_core_solver_b200 import build

    build.build()
    return capi.load()


def test_exports_every_declared_symbol(lib):
    declared = capi.header_symbols()
    assert len(declared) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in declared if s not in exported]
    assert not missing, missing


def test_status_strings(lib):
    assert lib.dn_status_string(4) == b"ICC preconditioner construction failed"
    assert lib.dn_status_string(5) == b"ILDLT preconditioner construction failed"
    assert lib.dn_status_string(9) == b"non-finite diagnostic detected"


def _struct_as_dict(c):
    d = {n: getattr(c, n) for n, t in capi.Config._fields_ if n not in ("p_bc", "u_bc", "v_bc")}
    for attr in ("p_bc", "u_bc", "v_bc"):
        arr = getattr(c, attr)
        for k in range(4):
            d[f"{attr}{k}"] = (arr[k].type, arr[k].value)
    return d


@pytest.mark.parametrize("path", [os.path.join(GOLDEN, "case92.cfg")] + sorted(
    glob.glob(os.path.join(GOLDEN, "testcases", "*.cfg"))))
def test_config_parse_matches_reference_parser(lib, path):
    text = open(path).read()
    ref = parse_cfg(text)  # restatement of config.cpp:49-208
    if ref["pressure_scheme"] not in PRESSURE:
        pytest.skip("pressure scheme outside the CUDA backend")
    c = capi.parse_config(text)
    for key in ("nx", "ny", "ghost", "ch_inner_iterations", "momentum_iterations", "poisson_iterations"):
        assert getattr(c, key) == ref[key], key
    for key in ("dt", "lx", "ly", "re", "ca", "pe", "cn", "density_ratio", "viscosity_ratio", "pressure_tolerance",
                "ch_tolerance", "momentum_tolerance", "body_force_x", "body_force_y", "interface_radius",
                "top_wall_velocity_x", "bottom_wall_velocity_x", "surface_tension_multiplier"):
        assert getattr(c, key) == ref[key], key
    assert bool(c.periodic_x) == ref["periodic_x"] and bool(c.periodic_y) == ref["periodic_y"]
    assert c.pressure_scheme == PRESSURE[ref["pressure_scheme"]]
    for f, attr in (("pressure", "p_bc"), ("u", "u_bc"), ("v", "v_bc")):
        for k, side in enumerate(SIDES):
            assert getattr(c, attr)[k].value == ref[f"{f}_bc_{side}_value"]


def test_config_errors(lib):
    with pytest.raises(capi.DnError):
        capi.parse_config("stabilization_a1 = 2\n")
    with pytest.raises(capi.DnError):
        capi.parse_config("pressure_scheme = hydea\n")
    with pytest.raises(capi.DnError):
        capi.parse_config("u_bc_left_type = robin\n")
    c = capi.parse_config("pressure_scheme = cuda_split_icpcg\nprecision = mixed\n")
    assert c.pressure_scheme == 3 and c.precision == 1
    assert capi.parse_config("nx = 32\n").device_share == 1
    assert capi.parse_config("device_share = 8\n").device_share == 8
    with pytest.raises(capi.DnError):
        capi.parse_config("device_share = 0\n")


def test_create_without_device_fails_loudly(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(capi.DnError) as ei:
        capi.Solver("nx = 32\nny = 32\npressure_scheme = icpcg\n")
    assert "no CUDA device" in str(ei.value)


def test_create_rejects_periodic_bc(lib):
    """validate_boundary_configuration (operators.cpp:11-34) runs before any device work."""
    with pytest.raises(capi.DnError) as ei:
        capi.Solver("nx = 32\nny = 32\nperiodic_x = true\nu_bc_left_type = dirichlet\n")
    assert "cannot be set when the direction is periodic" in str(ei.value)


def test_create_rejects_grids_below_eight_cells(lib):
    """The staged sweeps and the 13-point CH operator need at least 8 cells each way; smaller grids are
    refused before any device work (dn_create), with an UNSUPPORTED status, never run on the CPU."""
    with pytest.raises(capi.DnError) as ei:
        capi.Solver("nx = 6\nny = 6\nperiodic_x = false\nperiodic_y = false\n")
    assert ei.value.status == 10 and "nx, ny >= 8" in str(ei.value)


def test_ctypes_structs_match_the_c_header(tmp_path):
    """Every structure capi.py mirrors (dn_bc, dn_config, dn_report, dn_diag) has the C header's size and field
    offsets: a C program compiled against include/dn_cuda.h prints them.  A field added to the header but not
    to the mirror (or in another place) would hand the library a shifted struct."""
    mirrors = {"dn_bc": capi.BC, "dn_config": capi.Config, "dn_report": capi.Report, "dn_diag": capi.Diag}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "dn_cuda.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
        for n, _ in py._fields_:
            lines.append(f'  printf("{cname}.{n} %zu\\n", offsetof({cname}, {n}));')
    lines += ["  return 0;", "}"]
    src, exe = tmp_path / "layout.c", tmp_path / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                       check=True).stdout.splitlines())
    for cname, py in mirrors.items():
        assert int(got[cname]) == C.sizeof(py), (cname, got[cname], C.sizeof(py))
        for n, _ in py._fields_:
            assert int(got[f"{cname}.{n}"]) == getattr(py, n).offset, (cname, n)
