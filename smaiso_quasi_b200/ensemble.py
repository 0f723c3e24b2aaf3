"""Batched stability analysis: an ensemble of independent quasi-stb instances.

quasi-stb.cpp runs ONE pure-smectic instance per MPI job and records the
growth rate of a perturbed mode (quasi-stb.cpp:2111-2159).  The ensemble runs
many such instances, each perturbed by an interface displacement
h(x) = eps cos(Q x), on uneven grids, concurrently on one GPU (one stream and
one step graph per instance, launched asynchronously), and shards the
instances over ranks by cell count when several GPUs are used.  Instances
never exchange data: the only collective is the final gather of results.

    python -m smaiso_quasi_b200.ensemble --members 48 --steps 2000
    torchrun --nproc-per-node N -m smaiso_quasi_b200.ensemble ...
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import os
import sys
import time

import numpy as np

GRIDS = [(64, 64, 128), (96, 96, 192), (128, 128, 256)]


@dataclasses.dataclass
class Member:
    index: int
    grid: tuple[int, int, int]
    eps_h: float     # interface displacement amplitude
    m: int           # Q = 2 pi m / Lx
    seed: int

    @property
    def cells(self) -> int:
        return self.grid[0] * self.grid[1] * self.grid[2]

    def q_h(self, nw: int = 8, q0: float = 1.0) -> float:
        lx = self.grid[0] * 2.0 * math.pi / (q0 * nw)
        return 2.0 * math.pi * self.m / lx


def make_members(n: int = 48, seed: int = 2024) -> list[Member]:
    """eps log-uniform in [0.01, 0.1], m uniform in 1..8, grid uniform over GRIDS."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        eps = float(10 ** rng.uniform(-2.0, -1.0))
        m = int(rng.integers(1, 9))
        grid = GRIDS[int(rng.integers(0, len(GRIDS)))]
        out.append(Member(i, grid, eps, m, int(rng.integers(0, 2**31))))
    return out


def partition(members: list[Member], world: int) -> list[list[int]]:
    """Longest-processing-time assignment by cell count: every rank gets a
    near-equal share of cells; deterministic for a given member list."""
    loads = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for mb in sorted(members, key=lambda x: (-x.cells, x.index)):
        r = min(range(world), key=lambda q: (loads[q], q))
        parts[r].append(mb.index)
        loads[r] += mb.cells
    return [sorted(p) for p in parts]


def run_members(members: list[Member], steps: int, precision: str = "fp32", device: int = 0,
                chunk: int = 50) -> dict:
    """Advance every member `steps` steps concurrently; returns growth rates
    (the quasi-stb probe at the perturbation's mode) and device-side timing."""
    from . import quasi as q
    cfgs = [q.default_config("stb", *mb.grid, precision=precision, device=device, q_pert=mb.q_h())
            for mb in members]
    ens = q.Ensemble(cfgs)   # quasi_ensemble_create
    for mb, cfg, s in zip(members, cfgs, ens.members):
        s.set_psi(q.initial_condition(cfg, "interface", seed=mb.seed, eps_h=mb.eps_h, q_h=mb.q_h()))
    ens.init()
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        n = min(chunk, steps - done)
        ens.step(n)   # every member enqueued before any is waited for
        done += n
    wall = time.perf_counter() - t0
    growth = [float(v) for v in ens.growth_rates()]
    cells = sum(mb.cells for mb in members)
    ens.close()
    return {"indices": [mb.index for mb in members], "growth": growth, "wall_s": wall,
            "instance_steps_per_s": len(members) * steps / wall if wall > 0 else 0.0,
            "cell_updates_per_s": cells * steps / wall if wall > 0 else 0.0}


def gather(local: dict, dist=None) -> list[dict]:
    """All ranks' result dicts (rank order); a single-process run returns [local]."""
    if dist is None or not dist.is_initialized():
        return [local]
    out: list = [None] * dist.get_world_size()
    dist.all_gather_object(out, local)
    return out


def merge(results: list[dict], n: int) -> dict:
    growth = [float("nan")] * n
    for r in results:
        for i, g in zip(r["indices"], r["growth"]):
            growth[i] = g
    wall = max(r["wall_s"] for r in results)
    return {"growth": growth, "max_wall_s": wall,
            "instance_steps_per_s": sum(r["instance_steps_per_s"] for r in results),
            "cell_updates_per_s": sum(r["cell_updates_per_s"] for r in results)}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m smaiso_quasi_b200.ensemble")
    ap.add_argument("--members", type=int, default=48)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64", "bf16x3"])
    ap.add_argument("--seed", type=int, default=2024)
    a = ap.parse_args(argv)
    dist = None
    rank, world, device = 0, 1, 0
    if "RANK" in os.environ and int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        rank, world = dist.get_rank(), dist.get_world_size()
        device = int(os.environ.get("LOCAL_RANK", rank))
    members = make_members(a.members, a.seed)
    mine = [members[i] for i in partition(members, world)[rank]]
    res = merge(gather(run_members(mine, a.steps, a.precision, device), dist), len(members))
    if rank == 0:
        print(json.dumps({"members": len(members), "steps": a.steps, "ranks": world, **res}))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
