"""Failure detection through the C ABI, with every failure made on the host
or by a bounded wait that is meant to run out (nothing faults, traps or hangs
the GPU): corrupt, truncated and mismatched checkpoints, a non-finite initial
condition, and a tile copy that is never issued."""
import numpy as np
import pytest

from oracle import quasi_oracle as qo

pytestmark = pytest.mark.gpu

ERR_INVALID, ERR_IO, ERR_TIMEOUT = -1, -5, -8


def _sim(grid=(16, 16, 32), steps=3, precision="fp64"):
    import smaiso_quasi_b200 as q
    cfg = q.default_config("quasi", *grid, precision=precision)
    s = q.Simulation(cfg)
    s.set_psi(q.initial_condition(cfg, "planar", seed=2))
    s.init()
    s.step(steps)
    return q, cfg, s


def _code(fn, *a):
    import smaiso_quasi_b200 as q
    with pytest.raises(q.QuasiError) as ei:
        fn(*a)
    return ei.value.code


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_truncated_checkpoint_is_rejected(tmp_path, precision):
    q, cfg, a = _sim(precision=precision)
    path = tmp_path / "ck.bin"
    a.save(path)
    raw = path.read_bytes()
    (tmp_path / "short.bin").write_bytes(raw[: len(raw) // 2])
    b = q.Simulation(cfg)
    assert _code(b.load, tmp_path / "short.bin") == ERR_IO
    (tmp_path / "long.bin").write_bytes(raw + b"\0" * 8)
    assert _code(b.load, tmp_path / "long.bin") == ERR_IO


def test_corrupt_checkpoint_is_rejected_and_leaves_the_handle(tmp_path):
    q, cfg, a = _sim()
    a.save(tmp_path / "ck.bin")
    raw = bytearray((tmp_path / "ck.bin").read_bytes())
    raw[len(raw) // 3] ^= 0x40                      # one flipped bit in a field
    (tmp_path / "bad.bin").write_bytes(bytes(raw))
    b = q.Simulation(cfg)
    b.load(tmp_path / "ck.bin")
    before = b.field("psi")
    assert _code(b.load, tmp_path / "bad.bin") == ERR_IO
    assert b.nloop == 3 and np.array_equal(b.field("psi"), before)
    b.step(2)
    a.step(2)
    assert np.array_equal(a.field("psi"), b.field("psi"))


def test_checkpoint_of_another_grid_is_rejected(tmp_path):
    q, cfg, a = _sim()
    a.save(tmp_path / "ck.bin")
    other = q.Simulation(q.default_config("quasi", 32, 16, 32))
    assert _code(other.load, tmp_path / "ck.bin") == ERR_IO
    assert _code(other.load, tmp_path / "missing.bin") == ERR_IO


def test_nonfinite_initial_condition_is_rejected():
    import smaiso_quasi_b200 as q
    cfg = q.default_config("quasi", 16, 16, 32)
    s = q.Simulation(cfg)
    psi = q.initial_condition(cfg, "planar", seed=1)
    psi[3, 4, 5] = np.nan
    assert _code(s.set_psi, psi) == ERR_INVALID
    psi[3, 4, 5] = np.inf
    assert _code(s.set_psi, psi) == ERR_INVALID
    assert _code(s.init) == -4                       # nothing was accepted


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_tile_wait_timeout_reaches_the_host(precision):
    """The copy of one tile is never issued: its bounded wait runs out, the
    kernel flags it and returns, the call reports QUASI_ERR_TIMEOUT, and the
    same plan then transforms correctly (the context is still usable)."""
    import smaiso_quasi_b200 as q
    grid = (64, 64, 128)
    a = np.random.default_rng(1).standard_normal(grid)
    p = q.R2RPlan(*grid, "iCT", precision=precision)
    p.inject_wait_timeout(skip_tile=0, poll_limit=64)
    assert _code(p.execute_host, a) == ERR_TIMEOUT
    ref = qo.r2r3d(a, qo.PLAN_KINDS["iCT"])
    got = p.execute_host(a)
    tol = 1e-14 if precision == "fp64" else 2e-6
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < tol
