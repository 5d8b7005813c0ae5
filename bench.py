"""Throughput of the CHNS time step on B200 (Mcell-steps/s), with roofline, CPU baseline and end-to-end legs.

Workload: the 192x384 rising bubble -- no-slip top/bottom, free-slip sides, density and viscosity ratio 10,
split_icpcg pressure (rho_ref = min density), WENO5 phase advection, seeded interface modes 2-8 -- run in the
reference's R0-unit parameterisation (testcase 26: lx=4, ly=8, R=1, Re=12.374, Ca=0.0202, Cn=0.04, Pe=150,
g=1, dt=5e-5).  The unit-square mapping of this bubble (lx=1, ly=2, R=0.25) diverges on the reference itself
after ~30 steps, so a bounded trajectory on the same grid is timed.  Inputs are synthetic (seeded numpy),
FP64 ("plain" form).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on stdout (rank 0).  Under torchrun (N > 1) every rank advances its own replica (the 2D step
does not shard without changing the preconditioner); value is the aggregate over ranks, timed as the max
over ranks.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# The ensemble arm runs one stream per instance; the CUDA runtime maps streams onto this many hardware work
# queues (8 by default), and streams sharing a queue serialise.  Read when the process creates its context.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
# Algorithmic bytes per cell per pressure-PCG iteration of the split scheme, FP64 (SpMV 16, x/r update 48,
# forward sweep 24, backward sweep 24, p update 24): every distinct array read once and written once.
PCG_BYTES_PER_CELL_IT = 136.0
METRIC = "Mcell-steps/s (plain FP64 step; the mixed-precision form in `mixed`)"
RESTART_FIELDS = ("c", "c_prev", "c_prev2", "p", "p_prev", "u", "v", "u_prev", "v_prev", "e_prev", "hu_prev",
                  "hv_prev")


def workload_cfg(grid=None) -> dict:
    """The rising bubble in R0 units (box 4 x 8); `grid` = (nx, ny) refines it (192 x 384 by default)."""
    cfg = dict(
        name="rising_bubble_192x384_split_icpcg", mode="coupled", nx=192, ny=384, ghost=3, lx=4.0, ly=8.0,
        periodic_x=False, periodic_y=False, v_bc_left_type="neumann", v_bc_left_value=0.0,
        v_bc_right_type="neumann", v_bc_right_value=0.0, interface_center_x=2.0, interface_center_y=2.0,
        interface_radius=1.0, re=12.374368670764582, ca=0.02020305007471719, cn=0.04, pe=150.0,
        density_ratio=10.0, viscosity_ratio=10.0, body_force_y=-1.0, dt=5e-5, pressure_scheme="split_icpcg",
        poisson_iterations=2000, pressure_tolerance=1e-10, ch_inner_iterations=500, ch_tolerance=1e-10,
        momentum_iterations=200, momentum_tolerance=1e-10, surface_tension_multiplier=1.0)
    if grid is not None:
        # finer grids need more CG iterations to reach the same tolerance: no cap in the way
        cfg.update(nx=int(grid[0]), ny=int(grid[1]), name=f"rising_bubble_{grid[0]}x{grid[1]}_split_icpcg",
                   poisson_iterations=50000, ch_inner_iterations=5000)
    return cfg


def initial_state(cfg: dict, seed: int = 2) -> dict:
    """Seeded perturbed bubble: R(theta) = R + sum_{k=2..8} a_k cos(k theta + phi_k), a_k = 0.02 U(-1,1)
    (0.005 in the unit-square units of config 2), c = 1/2 - 1/2 tanh((r - R(theta)) / (2 sqrt 2 Cn))."""
    rng = np.random.default_rng(seed)
    nx, ny, g = cfg["nx"], cfg["ny"], cfg["ghost"]
    dx, dy = cfg["lx"] / nx, cfg["ly"] / ny
    x = (np.arange(nx) + 0.5) * dx - cfg["interface_center_x"]
    y = (np.arange(ny) + 0.5) * dy - cfg["interface_center_y"]
    X, Y = np.meshgrid(x, y, indexing="ij")
    r, th = np.hypot(X, Y), np.arctan2(Y, X)
    R = np.full_like(r, cfg["interface_radius"])
    for k in range(2, 9):
        R += 0.02 * rng.uniform(-1, 1) * np.cos(k * th + rng.uniform(0, 2 * np.pi))
    c = 0.5 - 0.5 * np.tanh((r - R) / (2.0 * math.sqrt(2.0) * cfg["cn"]))
    cell = np.zeros((nx + 2 * g, ny + 2 * g))
    cell[g:-g, g:-g] = c
    state = {n: np.zeros((nx + 2 * g + (1 if n in ("u", "u_prev", "hu_prev") else 0),
                          ny + 2 * g + (1 if n in ("v", "v_prev", "hv_prev") else 0))) for n in RESTART_FIELDS}
    for n in ("c", "c_prev", "c_prev2"):
        state[n] = cell.copy()
    return state


PCG_PROFILE = os.path.join(ROOT, "profiles", "k_pcg_5_3_pressure_192x384.txt")


def pcg_traffic_per_launch():
    """DRAM bytes (read + write) of one pressure-PCG launch from the committed ncu summary, per iteration,
    or None when no summary is present."""
    try:
        for line in open(PCG_PROFILE):
            if line.startswith("dram_bytes_per_iteration:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def hbm_peak():
    try:
        with open(PEAKS_PATH) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.rows = []
        if self.proc is None:
            return False
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        for line in out.splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)
        return False

    def summary(self):
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return None, 0, 1, 0
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    return dist, rank, world, local


def reduce_max(dist, value: float) -> float:
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        import torch

        torch.cuda.synchronize()
        dist.barrier()


def cpu_reference_run(cfg, state, first_step, count, untimed=0):
    """Steps of the reference build (oracle/_ref, the reference's own C++ sources) on the host: seconds for
    `count` steps from step first_step + untimed, after `untimed` steps from `state` that are not timed."""
    from oracle.oracle import OracleSolver, available, with_defaults

    impl = "reference" if available("reference") else "port"
    s = OracleSolver(with_defaults(cfg), impl)
    s.initialize()
    for n, a in state.items():
        s.set_field(n, a)
    s.refresh_derived()
    for k in range(untimed):
        s.step(first_step + k)
    return s.time_steps(first_step + untimed, count), impl


def host_cpu():
    """The host's CPU model and hardware threads (the CPU baseline's machine)."""
    model = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"cpu_model": model, "host_threads": os.cpu_count()}


def first_timed_step(args) -> int:
    """Index of the first timed step: the warm-up steps, then one more after the untimed autotuning."""
    return args.warmup + (1 if args.autotune else 0)


def run_ours(args):
    import torch

    import ding_nsch_core_solver_b200 as dn
    from ding_nsch_core_solver_b200 import capi

    dist, rank, world, local = dist_setup(args.gpus)
    device = local if dist is not None else 0
    torch.cuda.set_device(device)
    cfg = workload_cfg(args.grid)
    state = initial_state(cfg)
    n_cells = cfg["nx"] * cfg["ny"]
    nxy = f"{cfg['nx']}x{cfg['ny']}"

    solver = dn.Solver(cfg, device=device)

    def inject(st):
        for n, a in st.items():
            solver.set_field(n, a)
        solver.refresh_derived()

    inject(state)
    solver.set_initial_mass(solver.compute_mass("c"))
    stream = torch.cuda.ExternalStream(solver.stream(), device=device)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=device)  # 512 MB > 126 MB L2

    step = 0
    for _ in range(args.warmup):
        solver.step(step)
        step += 1
    launch_shape = None
    if args.autotune:  # untimed: pick the pressure PCG's launch shape on the warmed-up state, then re-warm
        launch_shape = solver.autotune_pressure()
        solver.step(step)
        step += 1
    assert step == first_timed_step(args)
    timed_state = {n: solver.get_field(n) for n in RESTART_FIELDS}  # the CPU baseline starts from here
    barrier(dist)

    # ---- device-resident timed region: K steps, L2 flushed between steps (outside the timed windows)
    times, pcg_ms, pcg_its, reports, phases = [], [], [], [], []
    launches0 = solver.kernel_launches()
    with ClockSampler(device) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            torch.cuda.nvtx.range_push("plain_step")  # ncu --nvtx-include plain_step/ selects a timed step
            rep = solver.step(step)
            torch.cuda.nvtx.range_pop()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            ph = solver.phase_times_ms()
            phases.append(ph)
            pcg_ms.append(ph[4])
            pcg_its.append(ph[7])
            reports.append(rep)
            step += 1
    launches = solver.kernel_launches() - launches0
    plain_fields = {n: solver.get_field(n) for n in ("c", "mu", "u", "v", "p")}
    total_ms = sum(times)
    total_ms = reduce_max(dist, total_ms)
    value = n_cells * args.steps * world / (total_ms * 1e-3) / 1e6

    # ---- end-to-end through the C-ABI with host buffers: restart-field upload, step, download, per step
    host = {n: solver.get_field(n) for n in RESTART_FIELDS}
    pinned = {n: torch.from_numpy(a).pin_memory().numpy() for n, a in host.items()}
    h2d = sum(a.nbytes for a in pinned.values())
    barrier(dist)
    e2e_ms = 0.0
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        inject(pinned)
        solver.step(step)
        for n in RESTART_FIELDS:
            solver.get_field(n, out=pinned[n])
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
        step += 1
    e2e_ms = reduce_max(dist, e2e_ms)
    e2e_value = n_cells * args.steps * world / (e2e_ms * 1e-3) / 1e6

    # ---- the mixed-precision form: same state, same steps, timed the same way; fields compared with the
    # plain FP64 run after the same number of steps
    mixed = None
    if not args.no_mixed:
        msolver = dn.Solver(dict(cfg, precision="mixed"), device=device)
        for n, a in state.items():
            msolver.set_field(n, a)
        msolver.refresh_derived()
        msolver.set_initial_mass(msolver.compute_mass("c"))
        if args.step_graph:  # from the second step of index >= 1 on, each step is one graph launch
            msolver.set_step_graph(True)
        mstream = torch.cuda.ExternalStream(msolver.stream(), device=device)
        mstep = 0
        for _ in range(step - args.steps * 2):  # as many untimed steps as the plain run took
            msolver.step(mstep)
            mstep += 1
        mtimes, mreps, mphases = [], [], []
        mlaunch0 = msolver.kernel_launches()
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(mstream)
            torch.cuda.nvtx.range_push("mixed_step")
            mreps.append(msolver.step(mstep))
            torch.cuda.nvtx.range_pop()
            e1.record(mstream)
            e1.synchronize()
            mtimes.append(e0.elapsed_time(e1))
            mphases.append(msolver.phase_times_ms())
            mstep += 1
        g = cfg["ghost"]
        errs = {}
        for n, ref in plain_fields.items():
            got = msolver.get_field(n)[g:-g, g:-g]
            ref = ref[g:-g, g:-g]
            errs[n] = float(np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-300))
        mlaunches = msolver.kernel_launches() - mlaunch0
        mtotal = reduce_max(dist, sum(mtimes))
        mvalue = n_cells * args.steps * world / (mtotal * 1e-3) / 1e6
        phase_keys = ("ch", "momentum", "pressure", "correction") + (
            () if args.step_graph else ("pressure_inner_solves", "ch_inner_solves", "bicgstab_kernel"))
        mixed = {"value": round(mvalue, 4), "unit": "Mcell-steps/s", "ms_per_step": round(mtotal / args.steps, 4),
                 "vs_plain": round(mvalue / value, 4),
                 "pressure_iterations_mean": statistics.mean(r["pressure_iterations"] for r in mreps),
                 "refinement_cycles_mean": statistics.mean(r["refinement_cycles"] for r in mreps),
                 "inner_tolerance": 1e-5,
                 "inner_preconditioner": ("multigrid V-cycle" if all(r["mixed_inner_multigrid"] for r in mreps)
                                          else "IC(0)/ILDLT(0) wavefront"),
                 # the plain FP64 step is the oracle's to rel-L2 <= 1e-10 (tests/test_gpu_configs.py)
                 "rel_l2_vs_plain_fp64": {k: float(f"{v:.3e}") for k, v in errs.items()},
                 "ch_iterations_mean": statistics.mean(r["ch_iterations"] for r in mreps),
                 # with captured steps the phases are timed by the graph's event nodes
                 "phase_ms_mean": {k: round(statistics.mean(p[i] for p in mphases), 4)
                                   for i, k in enumerate(phase_keys)},
                 "step_graph": bool(args.step_graph),
                 "gpu_launches": mlaunches,
                 "ch_solver": ("FP32 CG, (K + s I)^-2 V-cycles, FP64 defect correction"
                               if all(r["ch_preconditioner"] == 3 for r in mreps) else "FP64 ILDLT-PCG"),
                 "compared_after_steps": mstep}
        msolver.close()

    # ---- batched ensemble: B instances of the workload (different seeded interfaces) advanced together by
    # dn_step_batch, each on its own stream and on 1/B of the SMs (device_share = B); one batch step = one
    # step of every instance.  Timed with events
    # on the default stream around the whole call (device idle before; the call returns when every instance
    # has finished), so host launch latency counts against it.
    batched = None
    if args.batch > 0:
        members = []
        for k in range(args.batch):
            s = dn.Solver(dict(cfg, device_share=args.batch), device=device)
            for n, a in initial_state(cfg, seed=40 + k).items():
                s.set_field(n, a)
            s.refresh_derived()
            s.set_initial_mass(s.compute_mass("c"))
            if args.step_graph:
                s.set_step_graph(True)
            members.append(s)
        bstep = 0
        for _ in range(args.warmup):
            capi.step_batch(members, [bstep] * len(members))
            bstep += 1
        blaunch0 = sum(s.kernel_launches() for s in members)
        btimes = []
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            capi.step_batch(members, [bstep] * len(members))
            e1.record()
            e1.synchronize()
            btimes.append(e0.elapsed_time(e1))
            bstep += 1
        blaunches = sum(s.kernel_launches() for s in members) - blaunch0
        btotal = reduce_max(dist, sum(btimes))
        bvalue = n_cells * len(members) * args.steps * world / (btotal * 1e-3) / 1e6
        batched = {"instances": len(members), "value": round(bvalue, 4), "unit": "Mcell-steps/s",
                   "ms_per_batch_step": round(btotal / args.steps, 4), "vs_single": round(bvalue / value, 4),
                   "gpu_launches": blaunches,
                   "entry_point": ("dn_step_batch: one CUDA graph launch per batch step, every instance's "
                                   "step a branch of it" if args.step_graph and args.warmup >= 2 else
                                   "dn_step_batch (one stream and host worker per instance)")}
        for s in members:
            s.close()

    # ---- ensemble of uneven droplet instances (periodic both ways, mixed precision): whole instances
    # sharded over the ranks by LPT on estimated cost, each rank's share stepped together by one
    # dn_step_batch call per batch step; one gather of per-instance records at the end
    ensemble = None
    if args.ensemble > 0:
        from ding_nsch_core_solver_b200.ensemble import ShardedEnsemble, droplet_cfgs, gather_records

        cfgs = droplet_cfgs(args.ensemble)
        cells = sum(c["nx"] * c["ny"] for c in cfgs)
        shard, err, etimes, ereps = None, "", [], []
        try:
            shard = ShardedEnsemble(cfgs, rank, world, device, proportional=not args.ensemble_equal,
                                    step_graph=args.step_graph)
            shard.initialize()
            estep = 0
            for _ in range(args.warmup):
                shard.step(estep)
                estep += 1
            for _ in range(args.steps):
                flush.zero_()
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                ereps.append(shard.step(estep))
                e1.record()
                e1.synchronize()
                etimes.append(e0.elapsed_time(e1))
                estep += 1
        except capi.DnError as e:
            err = str(e)
        # every rank reaches the same two collectives, an error on one rank included
        etotal = reduce_max(dist, sum(etimes) if not err else float("inf"))
        mine = shard.mine if shard is not None else []
        recs = []
        for k, i in enumerate(mine):
            d = shard.members[k].diagnostics() if not err else {}
            recs.append({"err": err, "pressure_iterations": [rs[k]["pressure_iterations"] for rs in ereps],
                         "ch_iterations": [rs[k]["ch_iterations"] for rs in ereps],
                         "max_velocity": d.get("max_velocity"), "mass_drift": d.get("mass_drift"),
                         "dt_limit_ratio": d.get("dt_limit_ratio")})
        if err and not mine:
            recs, mine = [{"err": err}], [-1 - rank]
        allrec = gather_records(dist, mine, recs)
        errors = sorted({r["err"] for r in allrec if r.get("err")})
        if errors:
            ensemble = {"instances": len(cfgs), "error": "; ".join(errors)}
        else:
            ensemble = {"instances": len(cfgs), "cells": cells,
                        "value": round(cells * args.steps / (etotal * 1e-3) / 1e6, 4), "unit": "Mcell-steps/s",
                        "ms_per_batch_step": round(etotal / args.steps, 3), "scaling": "strong",
                        "instances_per_rank": [len(p) for p in shard.parts],
                        "pressure_iterations_mean": round(statistics.mean(
                            x for r in allrec for x in r["pressure_iterations"]), 1),
                        "ch_iterations_mean": round(statistics.mean(x for r in allrec for x in r["ch_iterations"]), 1),
                        "max_velocity_max": max(r["max_velocity"] for r in allrec),
                        "dt_limit_ratio_max": max(r["dt_limit_ratio"] for r in allrec),
                        "mass_drift_max": max(r["mass_drift"] for r in allrec),
                        "workload": "uneven droplets: grids {64..256}^2, periodic both ways, split_icpcg, mixed, "
                                    "Pe = 1/Cn, each instance at half its tightest step limit (capillary, explicit "
                                    "CH, advective), seed 4; whole instances sharded over the ranks by LPT on cells x "
                                    "max(nx, ny), each rank's share stepped together by dn_step_batch" +
                                    (" as one CUDA graph launch per batch step" if args.step_graph else ""),
                        "cuda_device_max_connections": os.environ.get("CUDA_DEVICE_MAX_CONNECTIONS"),
                        "sm_share": "equal (1/instances)" if args.ensemble_equal else "in proportion to cells"}
        if shard is not None:
            shard.close()

    # ---- roofline of the dominant kernel (the pressure PCG), bytes per launch / launch time
    peak, peak_kind = hbm_peak()
    bytes_per_launch = PCG_BYTES_PER_CELL_IT * n_cells * statistics.mean(pcg_its)
    achieved = bytes_per_launch / (statistics.mean(pcg_ms) * 1e-3) / 1e9
    per_it = pcg_traffic_per_launch()
    roofline = {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 5),
                "traffic": None if per_it is None else round(per_it * statistics.mean(pcg_its)),
                "peak_source": peak_kind,
                "kernel": "k_pcg<5,3> (pressure ICC-PCG, persistent, staged wavefront, one launch per solve)",
                "algorithmic_bytes_per_launch": bytes_per_launch,
                "kernel_ms_mean": statistics.mean(pcg_ms)}
    # The sweeps are a dependency chain of nx + ny - 1 steps each way per iteration: time per dependent step
    # against the shuffle + FMA chain latency (61 cycles, about 31 ns at 1965 MHz, measured on B200).
    dep_steps = 2 * (cfg["nx"] + cfg["ny"] - 1) * statistics.mean(pcg_its)
    sweep_ms = statistics.mean(p[10] for p in phases)
    critical_path = {"dependent_sweep_steps_per_launch": round(dep_steps), "sweep_ms_per_launch": round(sweep_ms, 3),
                     "ns_per_dependent_step": round(sweep_ms * 1e6 / dep_steps, 1), "chain_floor_ns": 31.0}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        sample = max(1, args.cpu_sample_steps)
        first = first_timed_step(args)
        sec, impl = cpu_reference_run(cfg, timed_state, first, sample)
        cpu = {"value": round(n_cells * sample / sec / 1e6, 6), "unit": "Mcell-steps/s", "cores": 1,
               "kind": "reference" if impl == "reference" else "port",
               "sample": f"{sample} steps (steps {first}-{first + sample - 1}, the first timed steps of the GPU "
                         f"run, from the GPU's state before them) of the same {nxy} workload; the reference "
                         f"step is single-threaded",
               "seconds": round(sec, 3), **host_cpu()}

    if rank == 0:
        mean_rep = {k: statistics.mean(r[k] for r in reports) for k in ("pressure_iterations", "ch_iterations",
                                                                       "momentum_iterations")}
        line = {
            "metric": METRIC,
            "value": round(value, 4), "unit": "Mcell-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"rising bubble {nxy} split_icpcg, R0-unit parameters of testcase 26, seeded "
                                   "interface modes 2-8", "grid": [cfg["nx"], cfg["ny"]], "pressure_scheme": "split_icpcg",
                       "pressure_tolerance": 1e-10, "ch_tolerance": 1e-10, "precision": "fp64",
                       "l2": "flushed (512 MB write) between timed steps", "parallelism": f"replicas x{world}",
                       "launch_shape": launch_shape or "default (512 rows per CTA, sweep warps by shared memory)"},
            "iterations_mean": mean_rep,
            "phase_ms_mean": {k: round(statistics.mean(p[i] for p in phases), 4) for i, k in enumerate(
                ("ch", "momentum", "pressure", "correction", "pressure_pcg_kernel", "ch_pcg_kernel",
                 "bicgstab_kernel"))},
            "roofline": roofline,
            "critical_path": critical_path,
            "cpu_baseline": cpu,
            "mixed": mixed,
            "batched": batched,
            "ensemble": ensemble,
            "e2e": {"value": round(e2e_value, 4), "unit": "Mcell-steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": h2d},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    solver.close()
    if dist is not None:
        barrier(dist)
        dist.destroy_process_group()


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.oracle import available

    cfg = workload_cfg()
    state = initial_state(cfg)
    n_cells = cfg["nx"] * cfg["ny"]
    if not (available("reference") or available("port")):
        print(json.dumps({"impl": "reference", "unavailable": "CPU reference build missing (make -C oracle)"}))
        return
    # the same steps the GPU arm times: its warm-up (and autotuning) steps run first, untimed
    first = first_timed_step(args)
    sec, impl = cpu_reference_run(cfg, state, 0, args.steps, untimed=first)
    value = n_cells * args.steps / sec / 1e6
    cpu = {"value": round(value, 6), "unit": "Mcell-steps/s", "cores": 1, "kind": impl,
           "sample": f"steps {first}-{first + args.steps - 1} of the 192x384 workload (the steps the GPU arm "
                     f"times; steps 0-{first - 1} run untimed first); the reference step is single-threaded, so "
                     f"one host thread is all it can use", **host_cpu()}
    print(json.dumps({
        "impl": "reference", "metric": METRIC,
        "value": round(value, 6), "unit": "Mcell-steps/s", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(sec * 1e3 / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "rising bubble 192x384 split_icpcg, R0-unit parameters of testcase 26, seeded "
                               "interface modes 2-8", "grid": [192, 384]},
        "cpu_baseline": cpu,
        "e2e": {"value": round(value, 6), "unit": "Mcell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample-steps", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the default launch shape instead of picking the pressure PCG's with "
                         "dn_autotune_pressure before the timed steps")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision arm")
    ap.add_argument("--no-step-graph", dest="step_graph", action="store_false",
                    help="step the mixed, batched and ensemble arms eagerly instead of replaying captured steps")
    ap.add_argument("--batch", type=int, default=8, help="instances of the batched-ensemble arm (0 skips it)")
    ap.add_argument("--ensemble", type=int, default=64, help="uneven droplet instances of the ensemble arm (0 skips)")
    ap.add_argument("--ensemble-equal", action="store_true",
                    help="give every ensemble instance the same share of the SMs (default: in proportion to its cells)")
    ap.add_argument("--grid", type=lambda t: tuple(int(v) for v in t.lower().split("x")), default=None,
                    help="NXxNY: the rising bubble on another grid (default 192x384)")
    args = ap.parse_args()
    if args.warmup < 3:  # both arms: the reference arm times the same steps as this one
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
