"""Restart snapshots v2 (dn_write_restart / dn_load_restart; Solver::write_restart_snapshot and
load_restart_snapshot, io.cpp:271-437).

- The written file is read back by an independent reader of the format as io.cpp lays it out, and its
  header and fields match the solver's state.
- A fresh solver loaded from the snapshot continues bit for bit like the solver that wrote it.
- The snapshot is a complete state for the reference algorithm: the oracle, given the fields and the
  restart rebuild (io.cpp:412-436), steps to the same fields as the loaded solver.
- A snapshot of another configuration is refused with the reference's message.
"""
import struct

import numpy as np
import pytest

from oracle.oracle import OracleSolver
from test_gpu_parity import CASES, assert_fields_close, seeded_pair

FIELDS = ("c", "c_prev", "c_prev2", "p", "p_prev", "u", "v", "u_prev", "v_prev", "e_prev", "hu_prev", "hv_prev")
SCALARS = ("dt", "lx", "ly", "re", "ca", "pe", "cn", "density_ratio", "viscosity_ratio", "body_force_x",
           "body_force_y", "top_wall_velocity_x", "bottom_wall_velocity_x")


def read_snapshot(path):
    """The v2 layout of io.cpp:282-333, read without the library."""
    data = open(path, "rb").read()
    pos = 0

    def take(fmt):
        nonlocal pos
        vals = struct.unpack_from("<" + fmt, data, pos)
        pos += struct.calcsize("<" + fmt)
        return vals if len(vals) > 1 else vals[0]

    def string():
        nonlocal pos
        n = take("Q")
        v = data[pos:pos + n].decode()
        pos += n
        return v

    out = {"magic": string(), "version": take("I"), "step": take("i"), "initial_mass": take("d"),
           "mode": string(), "grid": take("iii"), "scalars": dict(zip(SCALARS, take("13d"))),
           "periodic": take("ii"), "bcs": [take("id") for _ in range(12)], "fields": {}}
    for name in FIELDS:
        nx, ny, g, size = take("iiiQ")
        arr = np.frombuffer(data, dtype="<f8", count=size, offset=pos).reshape(nx + 2 * g, ny + 2 * g)
        pos += 8 * size
        out["fields"][name] = arr.copy()
    assert pos == len(data)
    return out


@pytest.fixture(scope="module")
def dn():
    import ding_nsch_core_solver_b200 as m

    m.load()
    return m


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["walls_split_ildlt", "channel_x_icpcg", "mixed_bcs_icpcg"])
def test_snapshot_roundtrip_and_continuation(dn, name, tmp_path):
    cfg = CASES[name]
    orc, gpu = seeded_pair(dn, cfg, seed=5)
    fresh = dn.Solver(cfg)
    try:
        for k in range(3):
            gpu.step(k)
        path = tmp_path / "restart_latest.bin"
        gpu.write_restart(path, 3)
        snap = read_snapshot(path)
        assert snap["magic"] == "ding_nsch_restart_v1" and snap["version"] == 2 and snap["step"] == 3
        assert snap["mode"] == "coupled" and snap["grid"] == (cfg["nx"], cfg["ny"], cfg["ghost"])
        assert snap["scalars"]["dt"] == cfg["dt"] and snap["periodic"] == (int(cfg["periodic_x"]), int(cfg["periodic_y"]))
        for f in FIELDS:
            assert np.array_equal(snap["fields"][f], gpu.get_field(f)), f
        assert fresh.load_restart(path) == 3
        for k in range(3, 5):
            gpu.step(k)
            fresh.step(k)
        for f in ("c", "mu", "u", "v", "p", "rho", "eta"):
            assert np.array_equal(fresh.get_field(f), gpu.get_field(f)), (name, f)
        # the oracle resumed from the same snapshot (its restart rebuild) steps to the same state
        o2 = OracleSolver(cfg, "port")
        o2.initialize()
        for f in FIELDS:
            o2.set_field(f, snap["fields"][f])
        o2.set_initial_mass(snap["initial_mass"])
        o2.refresh_derived()
        again = dn.Solver(cfg)
        try:
            again.load_restart(path)
            for k in range(3, 5):
                o2.step(k)
                again.step(k)
            assert_fields_close(o2, again, ("c", "mu", "u", "v"), f"{name} resumed")
        finally:
            again.close()
            o2.close()
    finally:
        fresh.close()
        gpu.close()
        orc.close()


@pytest.mark.gpu
def test_snapshot_of_another_config_is_refused(dn, tmp_path):
    import ding_nsch_core_solver_b200 as m

    a = dn.Solver(CASES["walls_split_ildlt"])
    b = dn.Solver(dict(CASES["walls_split_ildlt"], nx=CASES["walls_split_ildlt"]["nx"] + 2))
    c = dn.Solver(dict(CASES["walls_split_ildlt"], dt=2 * CASES["walls_split_ildlt"]["dt"]))
    try:
        a.initialize()
        path = tmp_path / "snap.bin"
        a.write_restart(path, 0)
        for other, what in ((b, "nx"), (c, "dt")):
            with pytest.raises(m.DnError) as e:
                other.load_restart(path)
            assert "restart snapshot incompatible with config: " + what in str(e.value)
        with pytest.raises(m.DnError):
            a.load_restart(tmp_path / "missing.bin")
    finally:
        for s in (a, b, c):
            s.close()
