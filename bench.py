"""Throughput of the quasi-incompressible smectic-isotropic step at 256^3.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload interface256|undulated256|droplet512]

Workload: the planar smectic-isotropic interface at 256x256x256 (seeded
+-1e-3 noise), the reference's quasi.cpp model at its default coefficients,
FP32 against FP64 after its 1000 steps; --workload undulated256: undulated
layers (delta = 0.5) at 256^3, 1000 steps; --workload droplet512: a smectic
droplet (r = 0.3 L) at 512x512x512, compared after its 200 steps.
One "step" is one time step of the whole model (24 r2r transforms plus the
pointwise stages).  The FP32 form (float fields and transforms; psi^, psi,
grad psi, the density chain, the update and the reductions in double) is the
headline when its error against the plain FP64 form after the workload's run
is within 1e-5 relative L2 in psi, rho and v; otherwise the FP64 step is.
Both forms are timed on the same GPU and reported, with the error.

Timing: W untimed warm-up steps, then windows of K steps between CUDA events
on the engine's stream, bracketed by a barrier and a device synchronise,
repeated for at least a second (the clock sampler runs meanwhile); the median
window, max over ranks.  Every step touches ~30 fields of 64-128 MiB: inputs
are far larger than the 126 MB L2, so no flush is needed between steps.

N > 1: the single instance does not shard (each transform is a global
transpose), so every rank runs an independent replica on its own GPU
("replicas only"); value is the aggregate steps/s over all ranks.

--impl reference: the reference's own quasi.cpp (built by oracle/build_ref.sh
against oracle/shim: FFTW's r2r kinds restated, MPI ranks as threads) on the
host cores, on the same workload size, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import re
import shutil
import subprocess
import sys
import tempfile
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

GRID = (256, 256, 256)
METRIC = "steps/s @256^3: plain FP64 vs FP32/split-BF16 TC; % HBM roofline; err vs FP64"
WORKLOAD = "planar smectic-isotropic interface 256x256x256, quasi.cpp model, seeded +-1e-3 noise"
IC_KIND = "planar"

# --workload: the headline case above, or the 512^3 droplet run (r = 0.3 L,
# 200 steps) the same line is measured on with --workload droplet512
WORKLOADS = {
    "interface256": ((256, 256, 256), "planar", METRIC, WORKLOAD, 1000),
    "undulated256": ((256, 256, 256), "undulated",
                     "steps/s @256^3 undulated layers: plain FP64 vs FP32; % HBM roofline; err vs FP64",
                     "undulated smectic layers A(z) cos(q0 z + 0.5 sin(2 pi x/Lx) sin(2 pi y/Ly)) 256x256x256, "
                     "quasi.cpp model, seeded +-1e-3 noise", 1000),
    "droplet512": ((512, 512, 512), "droplet",
                   "steps/s @512^3 droplet: plain FP64 vs FP32; % HBM roofline; err vs FP64",
                   "smectic droplet r = 0.3 L in the isotropic melt 512x512x512, quasi.cpp model, seeded", 200),
}


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        self.mark = 0
        if shutil.which("nvidia-smi"):
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.tmp, stderr=subprocess.DEVNULL)
            # the timed region starts once the sampler is running (first sample
            # written); only the samples after this point are summarised
            t_end = time.time() + 10
            while time.time() < t_end and os.path.getsize(self.tmp.name) == 0 and self.proc.poll() is None:
                time.sleep(0.02)
            self.mark = os.path.getsize(self.tmp.name)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        self.tmp.flush()
        rows = []
        with open(self.tmp.name) as f:
            f.seek(self.mark)
            lines = f.read().splitlines()
        for line in lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.tmp.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(rows)}


def dist_setup(n: int):
    """torch.distributed plumbing for N > 1 (barrier and max over ranks)."""
    if n <= 1 or "RANK" not in os.environ:
        return None
    import torch
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    import datetime
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return dist


def dist_max(dist, v: float) -> float:
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(dist):
    if dist is not None:
        dist.barrier()


def make_sim(q, prec: str, device: int):
    cfg = q.default_config("quasi", *GRID, precision=prec, device=device)
    return cfg, q.Simulation(cfg)


def run_profile_case(args) -> None:
    """One engine alone (FP32: about 2.3 GB on the device, FP64 about 4.6 GB):
    W + K steps, then 1 + 3 launches of the plain pass along --axis, the case
    the committed ncu summaries capture.  The autotuner is off (its timing
    under a profiler is not the live one): the default choices, which are the
    ones it makes live at 256^3 (double z passes as warp tiles, the rest as
    CTA tiles)."""
    import smaiso_quasi_b200 as q
    cfg = q.default_config("quasi", *GRID, precision=args.precision, device=0, autotune=0)
    sim = q.Simulation(cfg)
    sim.set_psi(q.initial_condition(cfg, IC_KIND, seed=1234))
    sim.init()
    sim.step(args.warmup + args.steps)
    print(json.dumps({"profile_case": f"{args.precision} {GRID[0]}^3", "steps": args.warmup + args.steps,
                      "axis": args.axis, "pass_ms": sim.time_axis_pass(args.axis, reps=3)}))


TOL32 = 1e-5   # the FP32 form's bound on the relative L2 error of psi, rho, v against FP64


def timed_repeats(sim, K: int, min_s: float = 1.0, min_reps: int = 3, max_reps: int = 200) -> list[float]:
    """K-step device-timed windows, repeated until at least `min_s` of wall
    time and `min_reps` windows (so that the clock sampler sees the load)."""
    out, t0 = [], time.perf_counter()
    while len(out) < min_reps or (time.perf_counter() - t0 < min_s and len(out) < max_reps):
        out.append(sim.step_timed(K))
    return out


def median(v):
    v = sorted(v)
    return v[len(v) // 2] if len(v) % 2 else 0.5 * (v[len(v) // 2 - 1] + v[len(v) // 2])


def e2e_run(sim, psi0, K: int, n_cells: int, dist, gpus: int) -> dict:
    """The public C ABI with host buffers: quasi_set_psi (H2D of the initial
    field) + quasi_init + K steps with the reference's diagnostic cadence
    (every 50 steps: 3 FP64 scalars D2H) + quasi_get_field(psi) (D2H)."""
    dist_barrier(dist)
    t0 = time.perf_counter()
    sim.set_psi(psi0)
    sim.init()
    done = 0
    while done < K:
        n = min(50, K - done)
        sim.step(n)
        done += n
        if done % 50 == 0:
            sim.diagnostics()
    sim.field("psi")
    dt = dist_max(dist, time.perf_counter() - t0)
    return {"value": round(gpus * K / dt, 3), "unit": "steps/s", "h2d_bytes_per_step": n_cells * 8 / K,
            "d2h_bytes_per_step": (n_cells * 8 + (K // 50) * 3 * 8) / K,
            "note": "quasi_set_psi + quasi_init + K x quasi_step + quasi_diagnostics/50 steps + quasi_get_field(psi)"}


def run_gpu(args) -> None:
    import numpy as np

    import smaiso_quasi_b200 as q
    dist = dist_setup(args.gpus)
    rank = int(os.environ.get("RANK", 0))
    device = int(os.environ.get("LOCAL_RANK", 0))
    K, W = args.steps, args.warmup
    n_cells = GRID[0] * GRID[1] * GRID[2]
    pk = peaks()
    cfg32, s32 = make_sim(q, "fp32", device)
    cfg64, s64 = make_sim(q, "fp64", device)
    # the split-BF16 tensor-core form (plain x / y passes as contractions)
    cfg16 = q.default_config("quasi", *GRID, precision="bf16x3", device=device, autotune=0)   # the form as such
    s16 = q.Simulation(cfg16)
    psi0 = q.initial_condition(cfg32, IC_KIND, seed=1234)

    # ---- e2e through the public C ABI, host buffers, copies inside ----------
    e2e32 = e2e_run(s32, psi0, K, n_cells, dist, args.gpus)
    e2e64 = e2e_run(s64, psi0, K, n_cells, dist, args.gpus)

    # ---- device-timed K-step windows of both forms ---------------------------
    for s in (s32, s64, s16):
        s.set_psi(psi0)
        s.init()
        s.step(W)
    dist_barrier(dist)
    with ClockSampler(device) as clk:
        win32 = timed_repeats(s32, K)
        win64 = timed_repeats(s64, K)
    win16 = timed_repeats(s16, K, min_s=0.3)
    dist_barrier(dist)
    ms32 = dist_max(dist, median(win32))
    ms64 = dist_max(dist, median(win64))
    ms16 = dist_max(dist, median(win16))
    clocks = clk.summary()
    sps32 = args.gpus * K / (ms32 / 1e3)
    sps64 = args.gpus * K / (ms64 / 1e3)
    launches32, launches64 = s32.step_kernels(), s64.step_kernels()

    # ---- error of the FP32 form against FP64 after the workload's run ------
    for s in (s32, s64, s16):
        s.set_psi(psi0)
        s.init()
        s.step(args.err_steps)

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))
    v64 = [s64.field(c) for c in ("vx", "vy", "vz")]

    def errors(s):
        e = {"steps": args.err_steps, "psi": rel(s.field("psi"), s64.field("psi")),
             "rho": rel(s.field("rho"), s64.field("rho"))}
        v = [s.field(c) for c in ("vx", "vy", "vz")]
        e["v"] = float(math.sqrt(sum(np.linalg.norm(a - b) ** 2 for a, b in zip(v, v64)) /
                                 sum(np.linalg.norm(b) ** 2 for b in v64)))
        return e
    err, err16 = errors(s32), errors(s16)
    fp32_ok = all(err[k] <= TOL32 for k in ("psi", "rho", "v"))

    # ---- the plain passes alone: the roofline of the dominant kernel ---------
    # algorithmic bytes per launch: one field read + one field written
    passes = {}
    for axis, name in ((2, "z"), (1, "y"), (0, "x")):
        for prec, s, b in (("fp32", s32, 4), ("fp64", s64, 8), ("bf16x3", s16, 4)):
            if prec == "bf16x3" and axis == 2:
                continue   # z stays an FFT pass in that form
            ms = s.time_axis_pass(axis, reps=20)
            gbs = 2 * b * n_cells / (ms / 1e3) / 1e9
            passes[f"{name}_{prec}"] = {"us": round(ms * 1e3, 2), "gbs": round(gbs, 1),
                                        "frac": round(gbs / pk["hbm_gbs"], 4)}
    head = "fp32" if fp32_ok else "fp64"
    top = passes[f"z_{head}"]   # the z pass: the largest share of the step in the ncu launch list
    traffic = None
    prof = ROOT / "profiles" / "traffic.json"
    if prof.exists():
        t = json.loads(prof.read_text()).get(f"z_pass_{head}_256_bytes_per_launch")
        traffic = None if t is None else int(t * n_cells / 256 ** 3)
    roofline = {"bound": "hbm", "achieved": top["gbs"], "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": top["frac"],
                "traffic": traffic, "kernel": f"tma_zpass_kernel<{'float' if head == 'fp32' else 'double'},"
                                              f"{GRID[2]},P,0> (plain z pass)",
                "peak_source": pk["source"] + " (burst copy)"}

    def step_roof(sps, sb):
        b = 48 * sb * n_cells
        return {"b_alg_bytes": b, "achieved_gbs": round(b * sps / args.gpus / 1e9, 1),
                "frac": round(b * sps / args.gpus / 1e9 / pk["hbm_gbs"], 4)}

    cpu = None
    if rank == 0 and args.gpus == 1 and not args.no_cpu:
        cpu = cpu_baseline(samples=1)

    if rank == 0:
        sps, ms, e2e = (sps32, ms32, e2e32) if fp32_ok else (sps64, ms64, e2e64)
        line = {
            "metric": METRIC, "value": round(sps, 3), "unit": "steps/s", "n_gpus": args.gpus,
            "steps": K, "warmup": W, "ms_per_step": round(ms / K, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if fp32_ok else "f64", "data": "synthetic",
            "headline_form": ("fp32: float fields and transforms; psi^, psi, grad psi and the density chain in "
                              "double" if fp32_ok else "fp64 (the FP32 form missed its error bound)"),
            "config": {"workload": WORKLOAD, "grid": list(GRID), "parallelism": f"replicas x{args.gpus}",
                       "l2": "inputs larger than L2 (~30 fields of 64-128 MiB per step)",
                       "timing": f"median of {len(win32)} (fp32) / {len(win64)} (fp64) windows of K steps"},
            "fp32": {"steps_per_s": round(sps32, 3), "ms_per_step": round(ms32 / K, 4),
                     "step_roofline": step_roof(sps32, 4), "e2e": e2e32, "within_tolerance": fp32_ok},
            "fp64": {"steps_per_s": round(sps64, 3), "ms_per_step": round(ms64 / K, 4),
                     "step_roofline": step_roof(sps64, 8), "e2e": e2e64},
            "bf16x3": {"steps_per_s": round(args.gpus * K / (ms16 / 1e3), 3), "ms_per_step": round(ms16 / K, 4),
                       "err_vs_fp64": err16,
                       "form": "the FP32 form with its plain x / y passes as split-BF16 tensor-core contractions"},
            "autotune": {"fp32": s32.tuning(), "fp64": s64.tuning()},
            "speedup_fp32_vs_fp64": round(sps32 / sps64, 3),
            "cell_updates_per_s": round(sps * n_cells, 1),
            "err_vs_fp64": err, "err_tolerance": TOL32,
            "roofline": roofline, "passes": passes,
            "e2e": e2e,
            "gpu_launches": (launches32 if fp32_ok else launches64) * K,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def cpu_baseline(samples: int) -> dict | None:
    """The reference's own quasi.cpp on the host cores: `samples` steps of the
    workload's grid (its focal-conic IC; the per-step work does not depend on psi),
    loop wall time as the reference itself reports it (quasi.cpp:2298-2304)."""
    from oracle import ref_runner as rr
    if not rr.available("quasi"):
        return None
    cores = os.cpu_count() or 1
    ranks = max(2, cores - cores % 2)
    while GRID[0] % ranks:
        ranks -= 2
    with tempfile.TemporaryDirectory() as d:
        r = rr.run_reference("quasi", *GRID, None, ranks, samples, 10 ** 6, 10 ** 6, d, fc_size="24",
                             read_outputs=False, timeout=3600)
    m = re.findall(r"Finished in ([0-9.eE+-]+) seconds \[Wall Clock\]", r["stdout"])
    loop_s = float(m[-1]) if m else r["wall_s"]
    return {"value": round(samples / loop_s, 5), "unit": "steps/s", "cores": ranks, "kind": "reference",
            "sample": f"{samples} step(s) of {GRID[0]}x{GRID[1]}x{GRID[2]}, reference quasi.cpp built on oracle/shim "
                      f"(FFTW r2r restated, {ranks} MPI ranks as threads), loop wall time"}


def run_ensemble(args) -> None:
    """The batched stability analysis: 48 perturbed planar interfaces
    (quasi-stb model) on grids drawn from 64^2x128, 96^2x192, 128^2x256, all
    stepped together (one graph launch per step for the whole ensemble); the
    FP32 form's growth rates against the same ensemble in FP64."""
    import numpy as np

    from smaiso_quasi_b200 import ensemble as en
    members = en.make_members(48, 2024)
    K = args.steps
    cells = sum(mb.cells for mb in members)
    r32 = en.run_members(members, K, "fp32", chunk=K)
    r64 = en.run_members(members, K, "fp64", chunk=K)
    g32, g64 = np.array(r32["growth"]), np.array(r64["growth"])
    rel_err = np.abs(g32 - g64) / np.abs(g64)
    print(json.dumps({
        "metric": "instance-steps/s, 48-member stability ensemble (quasi-stb), FP32 form",
        "value": round(r32["instance_steps_per_s"], 2), "unit": "instance-steps/s", "n_gpus": 1, "steps": K,
        "warmup": 0, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "48 perturbed planar interfaces, eps log-uniform [0.01, 0.1], m in 1..8, "
                               "grids from 64^2x128 / 96^2x192 / 128^2x256", "cells": cells,
                   "timing": "wall clock around quasi_ensemble_step (synchronous) after quasi_ensemble_init"},
        "cell_updates_per_s": round(r32["cell_updates_per_s"], 1),
        "fp64": {"instance_steps_per_s": round(r64["instance_steps_per_s"], 2)},
        "growth_rel_err_vs_fp64": {"max": float(rel_err.max()), "median": float(np.median(rel_err)), "steps": K},
    }), flush=True)


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    from oracle import ref_runner as rr
    if not rr.available("quasi"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/quasi_ref not built "
                          "(oracle/build_ref.sh needs the reference sources)"}))
        return
    K = max(1, min(args.steps, 3))
    cb = cpu_baseline(samples=K)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "steps/s", "n_gpus": args.gpus,
            "steps": K, "warmup": 0, "ms_per_step": round(1e3 / cb["value"], 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": list(GRID), "precision": "fp64 (the reference)"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: 400 at 256^3, 100 at 512^3: about a second of FP32 steps or more)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--err-steps", type=int, default=None,
                    help="steps after which FP32 is compared with FP64 (default: the workload's run length)")
    ap.add_argument("--workload", default="interface256", choices=sorted(WORKLOADS) + ["ensemble48"])
    ap.add_argument("--profile", action="store_true", help="one engine only (for ncu captures)")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64", "bf16x3"], help="engine of --profile")
    ap.add_argument("--axis", type=int, default=1, choices=[0, 1, 2], help="pass timed at the end of --profile")
    args = ap.parse_args()
    global GRID, IC_KIND, METRIC, WORKLOAD
    if args.workload == "ensemble48":
        if args.steps is None:
            args.steps = 200
        run_ensemble(args)
        return
    GRID, IC_KIND, METRIC, WORKLOAD, run_len = WORKLOADS[args.workload]
    if args.err_steps is None:
        args.err_steps = run_len
    if args.steps is None:
        args.steps = 400 if GRID[0] <= 256 else 100
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.profile:
        run_profile_case(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
