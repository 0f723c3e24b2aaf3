"""Throughput of the quasi-incompressible smectic-isotropic step at 256^3.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload interface256|droplet512]

Workload: the planar smectic-isotropic interface at 256x256x256 (seeded
+-1e-3 noise), the reference's quasi.cpp model at its default coefficients,
FP32 against FP64 after its 1000 steps; --workload droplet512: a smectic
droplet (r = 0.3 L) at 512x512x512, compared after its 200 steps.
One "step" is one time step of the whole model (24 r2r transforms plus the
fused pointwise stages).  The chosen form (FP32 fields and transforms, FP64
constants/update/reductions) is the headline; the plain FP64 form is timed on
the same GPU and reported beside it, with the FP32-vs-FP64 error.

Timing: W untimed warm-up steps, then K steps between CUDA events on the
engine's stream, bracketed by a barrier and a device synchronise, max over
ranks.  Every step touches ~30 fields of 64-128 MiB: inputs are far larger
than the 126 MB L2, so no flush is needed between steps.

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
import threading
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
    the committed ncu summaries capture."""
    import smaiso_quasi_b200 as q
    cfg, sim = make_sim(q, args.precision, 0)
    sim.set_psi(q.initial_condition(cfg, IC_KIND, seed=1234))
    sim.init()
    sim.step(args.warmup + args.steps)
    print(json.dumps({"profile_case": f"{args.precision} {GRID[0]}^3", "steps": args.warmup + args.steps,
                      "axis": args.axis, "pass_ms": sim.time_axis_pass(args.axis, reps=3)}))


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
    psi0 = q.initial_condition(cfg32, IC_KIND, seed=1234)

    # ---- e2e through the public C ABI, host buffers, copies inside ----------
    # set_psi (H2D of the initial field) + init + K steps with the reference's
    # diagnostic cadence (every 50 steps: 3 FP64 scalars D2H) + the final psi D2H.
    out = np.empty(GRID)
    dist_barrier(dist)
    t0 = time.perf_counter()
    s32.set_psi(psi0)
    s32.init()
    done = 0
    while done < K:
        n = min(50, K - done)
        s32.step(n)
        done += n
        if done % 50 == 0:
            s32.diagnostics()
    psi_out = s32.field("psi")
    e2e_s = time.perf_counter() - t0
    e2e_s = dist_max(dist, e2e_s)
    n_diag = K // 50
    e2e = {"value": args.gpus * K / e2e_s, "unit": "steps/s",
           "h2d_bytes_per_step": n_cells * 8 / K,
           "d2h_bytes_per_step": (n_cells * 8 + n_diag * 3 * 8) / K,
           "note": "quasi_set_psi + quasi_init + K x quasi_step + quasi_diagnostics/50 steps + quasi_get_field(psi)"}
    del out

    # ---- device-timed K steps of the chosen form (FP32) ---------------------
    s32.set_psi(psi0)
    s32.init()
    s32.step(W)
    dist_barrier(dist)
    with ClockSampler(device) as clk:
        ms32 = s32.step_timed(K)
    dist_barrier(dist)
    ms32 = dist_max(dist, ms32)
    clocks = clk.summary()
    launches_per_step = s32.step_kernels()
    steps_per_s = args.gpus * K / (ms32 / 1e3)

    # dominant kernel: the plain y-axis pass (largest share of the step in the
    # ncu launch list); algorithmic bytes = one field read + one field written
    pass_ms = s32.time_axis_pass(1, reps=20)
    pass_bytes = 2 * 4 * n_cells
    achieved = pass_bytes / (pass_ms / 1e3) / 1e9
    traffic = None
    prof = ROOT / "profiles" / "traffic.json"
    if prof.exists():
        # captured at 256^3; other grids scale it by the cells a launch processes
        t256 = json.loads(prof.read_text()).get("y_pass_fp32_256_bytes_per_launch")
        traffic = None if t256 is None else int(t256 * n_cells / 256 ** 3)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": round(achieved / pk["hbm_gbs"], 4), "traffic": traffic,
                "kernel": f"tma_pass_kernel<float,{GRID[1]},1,P> (plain y pass)",
                "peak_source": pk["source"] + " (burst copy)"}
    b_alg32 = 48 * 4 * n_cells
    step_roofline = {"b_alg_bytes": b_alg32, "achieved_gbs": round(b_alg32 * steps_per_s / args.gpus / 1e9, 1),
                     "frac": round(b_alg32 * steps_per_s / args.gpus / 1e9 / pk["hbm_gbs"], 4)}

    # ---- the plain FP64 form on the same GPU, same IC ------------------------
    cfg64, s64 = make_sim(q, "fp64", device)
    s64.set_psi(psi0)
    s64.init()
    s64.step(W)
    ms64 = s64.step_timed(K)
    ms64 = dist_max(dist, ms64)
    fp64_sps = args.gpus * K / (ms64 / 1e3)
    b_alg64 = 48 * 8 * n_cells

    # error of the FP32 form against FP64 from the same IC, after the
    # workload's run length (both continue untimed past the timed window)
    n_err = max(W + K, args.err_steps)
    if n_err > W + K:
        s32.step(n_err - (W + K))
        s64.step(n_err - (W + K))

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))
    err = {"steps": n_err, "psi": rel(s32.field("psi"), s64.field("psi")),
           "rho": rel(s32.field("rho"), s64.field("rho"))}
    v32 = [s32.field(c) for c in ("vx", "vy", "vz")]
    v64 = [s64.field(c) for c in ("vx", "vy", "vz")]
    err["v"] = float(math.sqrt(sum(np.linalg.norm(a - b) ** 2 for a, b in zip(v32, v64)) /
                               sum(np.linalg.norm(b) ** 2 for b in v64)))
    del psi_out

    cpu = None
    if rank == 0 and args.gpus == 1 and not args.no_cpu:
        cpu = cpu_baseline(samples=1)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(steps_per_s, 3), "unit": "steps/s", "n_gpus": args.gpus,
            "steps": K, "warmup": W, "ms_per_step": round(ms32 / K, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": list(GRID), "precision": "fp32 fields/transforms, fp64 update+reductions",
                       "parallelism": f"replicas x{args.gpus}", "l2": "inputs larger than L2 (~30 fields of 64 MiB)"},
            "fp64": {"steps_per_s": round(fp64_sps, 3), "ms_per_step": round(ms64 / K, 4),
                     "step_roofline_frac": round(b_alg64 * fp64_sps / args.gpus / 1e9 / pk["hbm_gbs"], 4)},
            "speedup_vs_fp64": round(steps_per_s / fp64_sps, 3),
            "cell_updates_per_s": round(steps_per_s * n_cells, 1),
            "err_vs_fp64": err,
            "step_roofline": step_roofline,
            "roofline": roofline,
            "e2e": e2e,
            "gpu_launches": launches_per_step * K,
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
    ap.add_argument("--workload", default="interface256", choices=sorted(WORKLOADS))
    ap.add_argument("--profile", action="store_true", help="one engine only (for ncu captures)")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"], help="engine of --profile")
    ap.add_argument("--axis", type=int, default=1, choices=[0, 1, 2], help="pass timed at the end of --profile")
    args = ap.parse_args()
    global GRID, IC_KIND, METRIC, WORKLOAD
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
