"""The CUDA step (through the C ABI) against the oracle and the reference's
own dumps (tests/golden)."""
import json
import pathlib

import numpy as np
import pytest

from oracle import quasi_oracle as qo

pytestmark = pytest.mark.gpu
GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"

# FP64: same arithmetic as the reference up to FMA contraction and transform
# round-off; the bar is 1e-12 relative L2 (v: of the velocity vector).
TOL64 = 1e-12


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb else np.linalg.norm(a)


def vec_err(got, ref):
    num = sum(np.linalg.norm(got[c] - ref[c]) ** 2 for c in ("vx", "vy", "vz"))
    den = sum(np.linalg.norm(ref[c]) ** 2 for c in ("vx", "vy", "vz"))
    return np.sqrt(num / den) if den else np.sqrt(num)


def make_pair(variant, grid, ranks=1, precision="fp64", ic="planar", seed=7):
    import smaiso_quasi_b200 as q
    cfg = q.default_config(variant, *grid, emulate_ranks=ranks, precision=precision)
    m = qo.Model(nx=grid[0], ny=grid[1], nz=grid[2], emulate_ranks=ranks) if variant == "quasi" else \
        qo.Model.stb(nx=grid[0], ny=grid[1], nz=grid[2], emulate_ranks=ranks)
    psi0 = qo.ic_field(m, ic, seed=seed)
    sim = q.Simulation(cfg)
    sim.set_psi(psi0)
    sim.init()
    o = qo.QuasiOracle(m)
    o.set_psi(psi0)
    o.init()
    return sim, o


def compare(sim, o, tol):
    got = {f: sim.field(f) for f in ("psi", "rho", "vx", "vy", "vz", "p", "divv", "psiq")}
    ref = {"psi": o.psi, "rho": o.rho, "vx": o.velx, "vy": o.vely, "vz": o.velz, "p": o.p, "divv": o.divv,
           "psiq": o.psiq}
    errs = {f: rel(got[f], ref[f]) for f in ("psi", "rho", "p", "psiq")}
    errs["v"] = vec_err(got, ref)
    if np.linalg.norm(ref["divv"]) > 0:
        errs["divv"] = rel(got["divv"], ref["divv"])
    bad = {k: v for k, v in errs.items() if not v < tol}
    assert not bad, (errs, tol)
    return errs


def test_init_projection_matches_oracle():
    sim, o = make_pair("quasi", (16, 16, 32))
    assert rel(sim.field("psi"), o.psi) < 1e-14
    assert rel(sim.field("psiq"), o.psiq) < 1e-14


@pytest.mark.parametrize("ranks", [1, 2, 4])
@pytest.mark.parametrize("steps", [1, 2, 10])
def test_step_fp64_matches_oracle(ranks, steps):
    sim, o = make_pair("quasi", (16, 16, 32), ranks=ranks)
    for _ in range(steps):
        o.step()
    sim.step(steps)
    assert sim.nloop == steps
    compare(sim, o, TOL64)
    d_gpu, d_ref = np.array(sim.diagnostics()), np.array(o.diagnostics())
    np.testing.assert_allclose(d_gpu, d_ref, rtol=1e-11)


def test_step_fp64_crosses_divv_and_pressure_switches():
    """Steps 199-203: divv turns on after step 200, the p coupling after 201."""
    sim, o = make_pair("quasi", (16, 16, 32), ranks=2, seed=11)
    for _ in range(198):
        o.step()
    sim.step(198)
    for _ in range(5):
        o.step()
        sim.step(1)
        compare(sim, o, 1e-11)


@pytest.mark.parametrize("grid", [(32, 32, 64), (96, 96, 192), (16, 16, 512), (256, 256, 32), (32, 256, 256)])
def test_step_fp64_larger_grids(grid):
    """Includes N = 256 on x and y (the headline grid's transform lengths)."""
    sim, o = make_pair("quasi", grid, ranks=2)
    for _ in range(3):
        o.step()
    sim.step(3)
    compare(sim, o, TOL64)


def test_step_stb_matches_oracle():
    sim, o = make_pair("stb", (16, 16, 32), ranks=2, ic="stb", seed=3)
    for s in range(6):
        o.step()
        sim.step(1)
        assert rel(sim.field("psi"), o.psi) < TOL64
        assert rel(sim.field("dtpsi"), o.dtpsi) < 1e-10
        if s > 0:
            assert abs(sim.growth_rate() - o.growth_rate()) <= 1e-9 * abs(o.growth_rate())


def _full_fixtures():
    return sorted(p.stem for p in GOLDEN.glob("quasi_*.npz") if "psi" in np.load(p).files)


@pytest.mark.parametrize("name", _full_fixtures())
def test_step_matches_reference_dumps(name):
    """GPU against the reference's own 17-digit dumps (no oracle in between)."""
    import smaiso_quasi_b200 as q
    z = np.load(GOLDEN / f"{name}.npz")
    meta = json.loads(str(z["meta"]))
    grid = (meta["nx"], meta["ny"], meta["nz"])
    cfg = q.default_config("quasi", *grid, emulate_ranks=meta["ranks"])
    psi0 = z["ic"] if "ic" in z.files else q.initial_condition(cfg, "focal_conic", fc_size=float(meta["fc_size"]))
    sim = q.Simulation(cfg)
    sim.set_psi(psi0)
    sim.init()
    sim.step(meta["steps"])
    assert rel(sim.field("psi"), z["psi"]) < 1e-12
    nsl = grid[0] * grid[2]
    got = {f: sim.field(f)[:, grid[1] // 2, :].reshape(-1) for f in ("vx", "vy", "vz", "rho", "p")}
    ref = {f: z[f][-1] for f in ("vx", "vy", "vz", "rho", "p")}
    assert rel(got["rho"], ref["rho"]) < 1e-12
    assert rel(got["p"], ref["p"]) < 1e-10
    assert vec_err(got, ref) < 1e-11
    assert len(got["vx"]) == nsl


def test_config1_matches_reference_500_steps():
    """The 64x64x128 planar interface as the reference runs it with 4 MPI
    ranks: 500 steps, diagnostics every 50 steps and a mid-slice dump every
    second diagnostic (quasi.cpp:1969-2280), against the reference's own
    17-digit dumps."""
    import smaiso_quasi_b200 as q
    z = np.load(GOLDEN / "quasi_64x64x128_np4_s500.npz")
    meta = json.loads(str(z["meta"]))
    grid = (meta["nx"], meta["ny"], meta["nz"])
    cfg = q.default_config("quasi", *grid, emulate_ranks=meta["ranks"])
    sim = q.Simulation(cfg)
    sim.set_psi(q.initial_condition(cfg, meta["ic"], seed=meta["seed"]))
    sim.init()
    mid = lambda f: sim.field(f)[:, grid[1] // 2, :].reshape(-1)
    diags, psi_mid = [], []
    for s in range(1, meta["steps"] // meta["step_l1"] + 1):
        sim.step(meta["step_l1"])
        diags.append(sim.diagnostics())
        if s % meta["step_save"] == 0:   # a dump every step_save diagnostics (quasi.cpp:2037)
            psi_mid.append(mid("psi"))
    d = np.array(diags)
    np.testing.assert_allclose(d[:, 0], z["L1"], rtol=1e-10)
    np.testing.assert_allclose(d[:, 1], z["mass"], rtol=1e-12)
    np.testing.assert_allclose(d[:, 2], z["energy"], rtol=1e-11)
    assert len(psi_mid) == len(z["psiMid"])
    for got, ref in zip(psi_mid, z["psiMid"]):
        assert rel(got, ref) < TOL64
    got = {f: mid(f) for f in ("vx", "vy", "vz", "rho", "p", "divv")}
    assert rel(got["rho"], z["rho"][-1]) < TOL64
    assert rel(got["p"], z["p"][-1]) < 1e-10
    assert rel(got["divv"], z["divv"][-1]) < 1e-10
    # 300 steps past the divv switch the difference quotient has amplified
    # round-off: the oracle itself is 1.9e-11 from these dumps in v
    assert vec_err(got, {f: z[f][-1] for f in ("vx", "vy", "vz")}) < 1e-10


# The FP32 form's tolerance against the FP64 form: 1e-5 relative L2 in psi,
# rho and the velocity vector.
TOL32 = 1e-5


@pytest.mark.parametrize("grid", [(32, 32, 64), (64, 64, 128)])
def test_fp32_error_vs_fp64_past_divv_switch(grid):
    """The FP32 form against the FP64 form on the same GPU after 320 steps,
    past the divv switch (step 200) where the difference quotient
    (rho - rho_old)/dt amplifies any rounding noise in rho."""
    import smaiso_quasi_b200 as q
    cfg64 = q.default_config("quasi", *grid)
    cfg32 = q.default_config("quasi", *grid, precision="fp32")
    psi0 = q.initial_condition(cfg64, "planar", seed=5)
    sims = []
    for cfg in (cfg64, cfg32):
        s = q.Simulation(cfg)
        s.set_psi(psi0)
        s.init()
        s.step(320)
        sims.append(s)
    a, b = sims[1], sims[0]
    errs = {"psi": rel(a.field("psi"), b.field("psi")), "rho": rel(a.field("rho"), b.field("rho")),
            "v": vec_err({f: a.field(f) for f in ("vx", "vy", "vz")}, {f: b.field(f) for f in ("vx", "vy", "vz")})}
    assert all(v < TOL32 for v in errs.values()), errs


def test_checkpoint_round_trip(tmp_path):
    import smaiso_quasi_b200 as q
    cfg = q.default_config("quasi", 16, 16, 32)
    psi0 = q.initial_condition(cfg, "planar", seed=2)
    a = q.Simulation(cfg)
    a.set_psi(psi0)
    a.init()
    a.step(5)
    a.save(tmp_path / "ck.bin")
    a.step(7)
    b = q.Simulation(cfg)
    b.load(tmp_path / "ck.bin")
    assert b.nloop == 5
    b.step(7)
    assert np.array_equal(a.field("psi"), b.field("psi"))


def test_autotuner_choices_do_not_change_results():
    """quasi_create's autotuner picks among kernels that compute the same
    transform (CTA or warp tiles of the z pass; the compiler may contract
    their multiply-adds differently): a tuned and an untuned FP32 handle agree
    to float rounding, and tuning also covers shapes the TMA passes do not."""
    import smaiso_quasi_b200 as q
    out = []
    for tune in (1, 0):
        cfg = q.default_config("quasi", 32, 32, 64, precision="fp32", autotune=tune)
        s = q.Simulation(cfg)
        t = s.tuning()
        assert t["measured"] == bool(tune)
        s.set_psi(q.initial_condition(cfg, "planar", seed=4))
        s.init()
        s.step(5)
        out.append(s.field("psi"))
    assert rel(out[0], out[1]) < 1e-6
    small = q.Simulation(q.default_config("stb", 16, 16, 32, precision="fp32"))   # no TMA z pass here
    assert small.tuning()["measured"]


@pytest.mark.parametrize("grid", [(32, 32, 64), (64, 64, 128), (96, 96, 192)])
def test_warp_tile_kernels_match_oracle(grid):
    """Every pass as warp tiles (autotune = 2: the z, x and y kernels the
    autotuner may pick) against the oracle, FP64, 3 steps."""
    import smaiso_quasi_b200 as q
    cfg = q.default_config("quasi", *grid, emulate_ranks=2, autotune=2)
    m = qo.Model(nx=grid[0], ny=grid[1], nz=grid[2], emulate_ranks=2)
    psi0 = qo.ic_field(m, "planar", seed=8)
    sim = q.Simulation(cfg)
    t = sim.tuning()
    assert set(t["warp_tiles_double"]) == {"z", "x", "y"}
    sim.set_psi(psi0)
    sim.init()
    o = qo.QuasiOracle(m)
    o.set_psi(psi0)
    o.init()
    for _ in range(3):
        o.step()
    sim.step(3)
    compare(sim, o, TOL64)
