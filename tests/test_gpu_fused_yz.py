"""The optional one-pass y+z cluster kernel (QUASI_FUSED_YZ=1), run in a
child process so the setting cannot leak: transforms and steps must match
the oracle exactly as the default two-pass path does."""
import os
import subprocess
import sys
import textwrap

import pytest

pytestmark = pytest.mark.gpu

SCRIPT = textwrap.dedent('''
    import sys
    import numpy as np
    sys.path.insert(0, ".")
    import smaiso_quasi_b200 as q
    from oracle import quasi_oracle as qo
    def rel(a, b): return np.linalg.norm(a - b) / np.linalg.norm(b)
    rng = np.random.default_rng(1)
    for grid in [(16, 16, 32), (64, 64, 128), (96, 96, 192)]:
        for plan in ["CT", "iCT", "STy", "iSTz"]:
            a = rng.standard_normal(grid)
            for prec, tol in (("fp64", 1e-14), ("fp32", 2e-6)):
                got = q.R2RPlan(*grid, plan, precision=prec).execute_host(a)
                e = rel(got, qo.r2r3d(a, qo.PLAN_KINDS[plan]))
                assert e < tol, (grid, plan, prec, e)
    cfg = q.default_config("quasi", 32, 32, 64, emulate_ranks=2)
    psi0 = q.initial_condition(cfg, "planar", seed=4)
    sim = q.Simulation(cfg); sim.set_psi(psi0); sim.init(); sim.step(3)
    o = qo.QuasiOracle(qo.Model(nx=32, ny=32, nz=64, emulate_ranks=2)); o.set_psi(psi0); o.init()
    for _ in range(3): o.step()
    assert rel(sim.field("psi"), o.psi) < 1e-12
    print("fused yz ok")
''')


def test_fused_yz_matches_oracle():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, QUASI_FUSED_YZ="1")
    r = subprocess.run([sys.executable, "-c", SCRIPT], cwd=root, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fused yz ok" in r.stdout
