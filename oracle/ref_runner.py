"""Run the reference binary built by ``oracle/build_ref.sh`` and read its dumps.

TEST INFRASTRUCTURE ONLY (fixture generation and the CPU reference arm of
``bench.py``).  The initial psi is handed to the reference through its own
restart path (``argv[4] == 1`` reads ``save/psi<rank>.dat`` one value per line
in (i_local, j, k) order, quasi.cpp:692-717), written with 17 significant
digits so that the doubles round-trip exactly.
"""
from __future__ import annotations

import os
import pathlib
import subprocess
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"


def binary(variant: str) -> pathlib.Path:
    return REF_DIR / ("quasi_ref" if variant == "quasi" else "quasi-stb_ref")


def available(variant: str = "quasi") -> bool:
    return binary(variant).exists()


def _read(path: pathlib.Path) -> np.ndarray:
    if not path.exists() or path.stat().st_size == 0:
        return np.zeros(0)
    return np.loadtxt(path, dtype=np.float64, ndmin=1)


def run_reference(variant: str, nx: int, ny: int, nz: int, psi0: np.ndarray | None, ranks: int,
                  steps: int, step_l1: int, step_save: int, workdir: str | os.PathLike,
                  nu_arg: str = "1", ep_arg: str = "675", fc_size: str = "6",
                  timeout: float = 3600.0, read_outputs: bool = True) -> dict:
    """Run ``steps`` steps with ``ranks`` emulated MPI ranks.  ``psi0=None`` uses
    the reference's own focal-conic IC (argv[4] = 0) with size ``fc_size``.
    Returns the parsed dumps plus ``wall_s`` (the process wall time)."""
    work = pathlib.Path(workdir)
    prefix = work / "run-nu"
    run_dir = pathlib.Path(str(prefix) + nu_arg + "-e0d" + ep_arg)
    (run_dir / "save").mkdir(parents=True, exist_ok=True)
    n0 = nx // ranks
    load = "0"
    if psi0 is not None:
        load = "1"
        psi0 = np.asarray(psi0, dtype=np.float64).reshape(nx, ny, nz)
        for r in range(ranks):
            np.savetxt(run_dir / "save" / f"psi{r}.dat", psi0[r * n0:(r + 1) * n0].reshape(-1), fmt="%.17g")
    env = dict(os.environ)
    env.update(QUASI_RANKS=str(ranks), QUASI_NX=str(nx), QUASI_NY=str(ny), QUASI_NZ=str(nz),
               QUASI_OUTDIR=str(prefix), QUASI_MAXSTEPS=str(steps), QUASI_STEPL1=str(step_l1),
               QUASI_STEPSAVE=str(step_save))
    t0 = time.perf_counter()
    proc = subprocess.run([str(binary(variant)), nu_arg, ep_arg, fc_size, load], env=env, cwd=work,
                          capture_output=True, text=True, timeout=timeout)
    wall = time.perf_counter() - t0
    if proc.returncode != 0:
        raise RuntimeError(f"reference failed rc={proc.returncode}: {proc.stderr[-2000:]}")
    out = {"wall_s": wall, "stdout": proc.stdout}
    if not read_outputs:
        return out
    names = ["L1", "mass", "energy", "psiMid", "vx", "vy", "vz", "divv", "p", "rho",
             "dtpsi", "fourier", "growth"]
    for nm in names:
        out[nm] = _read(run_dir / f"{nm}.dat")
    parts = [_read(run_dir / f"psi{r}.dat") for r in range(ranks)]
    if all(p.size == n0 * ny * nz for p in parts):
        out["psi"] = np.concatenate(parts).reshape(nx, ny, nz)
    return out
