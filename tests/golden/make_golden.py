"""Generate the committed golden fixtures from the reference's own code.

Run in a container that has the reference sources:
    oracle/build_ref.sh && python tests/golden/make_golden.py
Each case runs ``oracle/_ref/quasi_ref`` (the reference's quasi.cpp or
quasi-stb.cpp compiled against ``oracle/shim``) with the seeded initial
condition handed in through the reference's restart path, and stores its
17-digit dumps in ``tests/golden/<case>.npz``:
    ic        the initial psi (nx, ny, nz)
    psi       psi after the last step (full field, ``psi<rank>.dat``)
    <name>    mid-slice dumps (saves, nx*nz) for psiMid vx vy vz divv p rho
              (quasi) or psiMid dtpsi fourier (stb)
    L1 mass energy growth   per-diagnostic series
    meta      JSON: variant, grid, ranks, steps, cadence, IC parameters
"""
from __future__ import annotations

import json
import pathlib
import sys
import tempfile

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import quasi_oracle as qo  # noqa: E402
from oracle import ref_runner as rr    # noqa: E402

OUT = pathlib.Path(__file__).resolve().parent

CASES = [
    # name, variant, grid, ranks, steps, stepL1, stepSave, ic, seed
    ("quasi_16x16x32_np2_s3", "quasi", (16, 16, 32), 2, 3, 1, 1, "planar", 7),
    ("quasi_16x16x32_np4_s3", "quasi", (16, 16, 32), 4, 3, 1, 1, "planar", 7),
    ("quasi_16x16x32_np2_s203", "quasi", (16, 16, 32), 2, 203, 1, 203, "planar", 11),
    ("quasi_8x16x16_np4_s205", "quasi", (8, 16, 16), 4, 205, 5, 41, "undulated", 5),
    ("stb_16x16x32_np2_s6", "stb", (16, 16, 32), 2, 6, 1, 1, "stb", 3),
    ("quasi_16x16x16_np2_fc_s2", "quasi", (16, 16, 16), 2, 2, 1, 2, "focal_conic", 0),
    # the 64x64x128 planar interface as `mpirun -np 4` runs it: 500 steps,
    # diagnostics every 50 steps, a dump every 2nd diagnostic (kept small:
    # psi mid-slices per dump, every field's mid-slice of the last dump, no
    # full fields)
    ("quasi_64x64x128_np4_s500", "quasi", (64, 64, 128), 4, 500, 50, 2, "planar", 1234),
]
# cases stored without full fields (their initial psi is the seeded IC, which
# tests regenerate)
SLIM = {"quasi_64x64x128_np4_s500"}


def make(case) -> None:
    name, variant, (nx, ny, nz), ranks, steps, l1, save, ic, seed = case
    if variant == "quasi":
        m = qo.Model(nx=nx, ny=ny, nz=nz, emulate_ranks=ranks)
    else:
        m = qo.Model.stb(nx=nx, ny=ny, nz=nz, emulate_ranks=ranks)
    psi0 = None if ic == "focal_conic" else qo.ic_field(m, ic, seed=seed)
    with tempfile.TemporaryDirectory() as d:
        ref = rr.run_reference(variant, nx, ny, nz, psi0, ranks, steps, l1, save, d, fc_size="6")
    nsl = nx * nz
    arrays = {}
    slim = name in SLIM
    if "psi" in ref and not slim:        # quasi-stb.cpp:2051-2062 (full psi dump) is commented out
        arrays["psi"] = ref["psi"]
    if psi0 is not None and not slim:
        arrays["ic"] = psi0
    slices = ["psiMid", "vx", "vy", "vz", "divv", "p", "rho"] if variant == "quasi" else ["psiMid", "dtpsi", "fourier"]
    for nm in slices:
        a = ref[nm].reshape(-1, nsl)
        arrays[nm] = a if (nm == "psiMid" or not slim) else a[-1:]
    for nm in ["L1", "mass", "energy", "growth"]:
        if ref[nm].size:
            arrays[nm] = ref[nm]
    meta = dict(variant=variant, nx=nx, ny=ny, nz=nz, ranks=ranks, steps=steps, step_l1=l1, step_save=save,
                ic=ic, seed=seed, nu_arg="1", ep_arg="675", fc_size="6")
    np.savez_compressed(OUT / f"{name}.npz", meta=json.dumps(meta), **arrays)
    print(name, {k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    if not rr.available("quasi") or not rr.available("stb"):
        sys.exit("build the reference first: oracle/build_ref.sh")
    only = set(sys.argv[1:])
    for c in CASES:
        if not only or c[0] in only:
            make(c)
