"""A ragged batch of independent instances, sharded over the ranks of a job (one process per GPU).

The reference runs one instance per process; a batch of instances of uneven grids (droplets of nx, ny in
{64 .. 256}) has no exchange between instances, so it shards by whole instances: no collective inside a
step, each rank steps its share concurrently through dn_step_batch, and one gather of per-instance records
at the end.  Instances go to ranks by LPT greedy (longest estimated cost first, each to the least-loaded
rank), on cost = cells x estimated pressure iterations.

The partition is a pure function of the instance list and the world size, so every rank computes the same
one without communicating.
"""
from __future__ import annotations

import numpy as np

from . import capi

GRID_SIZES = (64, 96, 128, 192, 256)


def stable_dt(nx: int, ny: int, re: float, ca: float, pe: float, cn: float, density_ratio: float,
              speed: float, safety: float = 0.5) -> float:
    """`safety` x the tightest of the reference's step limits (populate_timestep_limits,
    diagnostics.cpp:48-112) for a droplet state: advective 0.5 / (|u|/dx + |v|/dy) at background speed
    `speed` in each direction, capillary 0.5 sqrt(Re Ca h^3 / rho_max), and the explicit CH limit
    0.25 h^2 / (6 sqrt 2 M W'' / (Pe Cn)) at its bounds M = 1/4, |W''| = 1/2 (h = min(dx, dy))."""
    dx, dy = 1.0 / nx, 1.0 / ny
    h = min(dx, dy)
    adv = 0.5 / max(speed / dx + speed / dy, 1e-30)
    cap = 0.5 * np.sqrt(re * ca * h ** 3 / max(1.0, density_ratio))
    chx = 0.25 * h * h / (6.0 * np.sqrt(2.0) * 0.25 * 0.5 / (pe * cn))
    return float(safety * min(adv, cap, chx))


def droplet_cfgs(count: int, seed: int = 4) -> list:
    """Droplet instances of uneven grids: nx, ny each from {64, 96, 128, 192, 256}; unit square, periodic
    both ways; radius U(0.15, 0.3) at a centre kept 0.05 inside the box; density and viscosity ratios
    log-uniform in [1, 100]; surface tension multiplier U(0.5, 2) with re = ca = 1; cn = 1.5 min(dx, dy),
    Pe = 1/Cn; uniform background velocity U(-0.1, 0.1)^2; split_icpcg in the mixed-precision form.  Each
    instance steps at half its tightest step limit (stable_dt), so every trajectory stays bounded: a common
    dt of 1e-5 lies above the explicit CH limit of the finer grids, whose chemical potential and then
    velocity blow up within 20 steps on the reference itself."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        nx, ny = (int(v) for v in rng.choice(GRID_SIZES, size=2))
        radius = rng.uniform(0.15, 0.3)
        cx, cy = rng.uniform(radius + 0.05, 1.0 - radius - 0.05, size=2)
        au, av = rng.uniform(-0.1, 0.1, size=2)
        dr, vr = float(10 ** rng.uniform(0, 2)), float(10 ** rng.uniform(0, 2))
        cn = 1.5 / max(nx, ny)
        out.append(dict(
            name=f"droplet_{nx}x{ny}", mode="coupled", nx=nx, ny=ny, ghost=3, lx=1.0, ly=1.0, periodic_x=True,
            periodic_y=True, interface_center_x=float(cx), interface_center_y=float(cy), interface_radius=float(radius),
            density_ratio=dr, viscosity_ratio=vr,
            surface_tension_multiplier=float(rng.uniform(0.5, 2.0)), re=1.0, ca=1.0, cn=cn, pe=1.0 / cn,
            advect_u=float(au), advect_v=float(av),
            dt=stable_dt(nx, ny, 1.0, 1.0, 1.0 / cn, cn, dr, max(abs(au), abs(av))),
            pressure_scheme="split_icpcg", precision="mixed",
            poisson_iterations=2000, pressure_tolerance=1e-10, ch_inner_iterations=500, ch_tolerance=1e-10,
            momentum_iterations=200, momentum_tolerance=1e-10))
    return out


def estimated_cost(cfg: dict) -> float:
    """Cells x estimated pressure iterations.  ICC-PCG on the 5-point operator needs O(1/h) iterations, so
    the estimate is max(nx, ny); each iteration touches every cell."""
    nx, ny = int(cfg["nx"]), int(cfg["ny"])
    return float(nx * ny * max(nx, ny))


def lpt_partition(costs, world: int) -> list:
    """Instance indices per rank: by cost descending (ties by index), each to the rank with the least load
    so far (ties to the lowest rank); each rank's list in ascending index order."""
    if world < 1:
        raise ValueError("world must be at least 1")
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def gather_records(dist, mine, records) -> list:
    """All ranks' per-instance records in global instance order: the job's one collective.  `mine` are this
    rank's instance indices, `records` one picklable record per instance.  Without a process group the
    records come back as they are."""
    pairs = list(zip(mine, records))
    if dist is None:
        chunks = [pairs]
    else:
        chunks = [None] * dist.get_world_size()
        dist.all_gather_object(chunks, pairs)
    merged = sorted((p for c in chunks for p in c), key=lambda p: p[0])
    idx = [p[0] for p in merged]
    if len(set(idx)) != len(idx):
        raise RuntimeError("an instance was stepped on more than one rank")
    return [p[1] for p in merged]


class ShardedEnsemble:
    """This rank's share of a ragged batch: one handle per instance, stepped together by dn_step_batch.
    Within the rank each handle's persistent grids take SMs in proportion to its cells (device_share =
    the rank's cells / its cells), or an equal share with `proportional=False`.  With `step_graph` every
    handle replays captured steps, so that from the second step of index >= 1 on a batch step is one CUDA
    graph launch holding every instance's step (dn_step_batch)."""

    def __init__(self, cfgs: list, rank: int = 0, world: int = 1, device: int = 0, proportional: bool = True,
                 step_graph: bool = False):
        self.cfgs = list(cfgs)
        self.parts = lpt_partition([estimated_cost(c) for c in self.cfgs], world)
        self.mine = self.parts[rank]
        cells = [self.cfgs[i]["nx"] * self.cfgs[i]["ny"] for i in self.mine]
        total = sum(cells)
        self.members = []
        try:
            for i, n in zip(self.mine, cells):
                share = max(1, round(total / n)) if proportional else max(1, len(self.mine))
                self.members.append(capi.Solver(dict(self.cfgs[i], device_share=share), device=device))
                if step_graph:
                    self.members[-1].set_step_graph(True)
        except Exception:
            self.close()
            raise

    def initialize(self) -> None:
        for m in self.members:
            m.initialize()
            m.set_initial_mass(m.compute_mass("c"))

    def step(self, step: int) -> list:
        """One step of every instance of this rank; their reports in the order of `mine`."""
        if not self.members:
            return []
        return capi.step_batch(self.members, [step] * len(self.members))

    def cells(self) -> int:
        return sum(self.cfgs[i]["nx"] * self.cfgs[i]["ny"] for i in self.mine)

    def close(self) -> None:
        for m in self.members:
            m.close()
        self.members = []
