"""Command-line driver with the reference's argument convention and dumps.

    python -m smaiso_quasi_b200.run NU EP_ARG FC_SIZE LOAD [options]

mirrors ``quasi <nu> <ep*1000> <aE> <load>`` (quasi.cpp:136,176-193): LOAD=1
restarts from ``<out>/save/psi<rank>.dat`` text files (one value per line,
(i_local, j, k) order, quasi.cpp:692-717), LOAD=0 builds the initial
condition (``--ic``; the reference's own is ``focal_conic``).  The run writes
the reference's outputs into ``--out``: ``info``, ``L1.dat``, ``mass.dat``,
``energy.dat`` every ``--step-l1`` steps and, every ``--step-save``
diagnostics, ``psi<rank>.dat`` and the j = Ny/2 mid-slices ``psiMid.dat``,
``vx.dat``, ``vy.dat``, ``vz.dat``, ``divv.dat``, ``p.dat``, ``rho.dat``
(quasi.cpp:1969-2280).  ``--digits 6`` reproduces the reference's default
ostream precision; the default is 17 significant digits.
The loop runs ``--steps`` steps (the reference loops until L1 < 1e-6; give
``--until-l1`` for that).
"""
from __future__ import annotations

import argparse
import pathlib
import sys
import time

import numpy as np

from . import quasi as q


def _fmt(digits: int):
    return f"%.{digits}g"


def write_text(path: pathlib.Path, values: np.ndarray, digits: int, append: bool) -> None:
    with open(path, "a" if append else "w") as f:
        np.savetxt(f, np.asarray(values).reshape(-1), fmt=_fmt(digits))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m smaiso_quasi_b200.run")
    ap.add_argument("nu", type=float)
    ap.add_argument("ep_arg", type=float)
    ap.add_argument("fc_size", type=float)
    ap.add_argument("load", type=int)
    ap.add_argument("--variant", default="quasi", choices=["quasi", "stb"])
    ap.add_argument("--grid", type=int, nargs=3, default=[64, 64, 128])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--ranks", type=int, default=1, help="emulate an MPI run of this many ranks")
    ap.add_argument("--ic", default="focal_conic",
                    choices=["planar", "undulated", "interface", "droplet", "stb", "focal_conic"])
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--until-l1", type=float, default=None)
    ap.add_argument("--step-l1", type=int, default=50)
    ap.add_argument("--step-save", type=int, default=10)
    ap.add_argument("--digits", type=int, default=17)
    ap.add_argument("--out", default="quasi_out")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)

    nx, ny, nz = a.grid
    cfg = q.default_config(a.variant, nx, ny, nz, precision=a.precision, emulate_ranks=a.ranks,
                           device=a.device, nu_arg=a.nu, ep_arg=a.ep_arg)
    out = pathlib.Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    n0 = nx // a.ranks
    if a.load == 1:
        parts = [np.loadtxt(out / "save" / f"psi{r}.dat") for r in range(a.ranks)]
        psi0 = np.concatenate(parts).reshape(nx, ny, nz)
    else:
        psi0 = q.initial_condition(cfg, a.ic, seed=a.seed, fc_size=a.fc_size)
    ep = -0.001 * a.ep_arg
    dx = 2.0 * np.pi / (cfg.q0 * cfg.nw)
    info = [("Nx", nx), ("Ny", ny), ("Nz", nz), ("Points per wavelength (nw)", cfg.nw), ("q0 (z direction)", cfg.q0),
            ("epsilon", ep), ("beta", cfg.beta), ("gamma", cfg.gamma), ("Viscosity (nu)", a.nu), ("dx", dx),
            ("dt", cfg.dt), ("stepL1", a.step_l1), ("stepSave", a.step_save), ("divv switch", cfg.divv_switch),
            ("Initial amp", cfg.amp), ("kp", cfg.kp), ("rho_0", cfg.rho_0), ("Focal conic initial size (fc)", a.fc_size)]
    (out / "info").write_text("".join(f"{k}: {v}\n" for k, v in info))   # quasi.cpp:609-629
    names = ["L1", "mass", "energy", "psiMid", "vx", "vy", "vz", "divv", "rho", "p"]
    if a.variant == "stb":
        names += ["dtpsi", "fourier", "growth"]
    for nm in names:
        (out / f"{nm}.dat").write_text("")

    sim = q.Simulation(cfg)
    sim.set_psi(psi0)
    sim.init()
    t0 = time.perf_counter()
    count_l1 = count_save = 0
    l1 = 1.0
    while True:
        if a.until_l1 is not None:
            if not l1 > a.until_l1:
                break
        elif sim.nloop >= a.steps:
            break
        sim.step(1)
        count_l1 += 1
        if a.variant == "stb":
            dtpsi = sim.field("dtpsi")
        if count_l1 == a.step_l1:
            l1, mass, energy = sim.diagnostics()
            write_text(out / "L1.dat", [l1], a.digits, True)
            write_text(out / "mass.dat", [mass], a.digits, True)
            if a.variant == "quasi":
                write_text(out / "energy.dat", [energy], a.digits, True)
            count_l1 = 0
            count_save += 1
            if count_save == a.step_save:
                count_save = 0
                psi = sim.field("psi")
                for r in range(a.ranks):
                    write_text(out / f"psi{r}.dat", psi[r * n0:(r + 1) * n0], a.digits, False)
                write_text(out / "psiMid.dat", psi[:, ny // 2, :], a.digits, True)
                if a.variant == "quasi":
                    for nm in ["vx", "vy", "vz", "divv", "p", "rho"]:
                        write_text(out / f"{nm}.dat", sim.field(nm)[:, ny // 2, :], a.digits, True)
                else:
                    write_text(out / "dtpsi.dat", dtpsi[:, ny // 2, :], a.digits, True)
                    write_text(out / "fourier.dat", sim.field("psiq")[:, 0, :], a.digits, True)
                    if sim.nloop > 1:
                        write_text(out / "growth.dat", [sim.growth_rate()], a.digits, True)
    wall = time.perf_counter() - t0
    print(f"{sim.nloop} steps in {wall:.3f} s wall ({sim.nloop / wall:.2f} steps/s)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
