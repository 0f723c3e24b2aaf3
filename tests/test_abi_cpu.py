"""The C ABI without a GPU: the library loads, exports every entry point that
include/quasi_gpu.h declares, fills the reference's defaults, rejects bad
configurations, and computes initial conditions on the host identical (to
round-off) to the oracle's."""
import ctypes
import pathlib
import re
import subprocess

import numpy as np
import pytest

from oracle import quasi_oracle as qo

ROOT = pathlib.Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "quasi_gpu.h").read_text()
    return sorted(set(re.findall(r"QUASI_API\s+[\w\s\*]*?\b(quasi_\w+)\s*\(", text)))


def test_header_declares_the_python_export_list():
    from smaiso_quasi_b200 import quasi as q
    assert declared_symbols() == sorted(q.EXPORTS)


def test_library_exports_every_declared_symbol():
    from smaiso_quasi_b200 import quasi as q
    out = subprocess.run(["nm", "-D", "--defined-only", str(q.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (quasi_\w+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    lib = q.lib()
    for s in declared_symbols():
        assert hasattr(lib, s)


def test_defaults_are_the_reference_constants():
    import smaiso_quasi_b200 as q
    c = q.default_config("quasi", 256, 256, 256)
    # quasi.cpp:183-219
    assert (c.gamma, c.beta, c.alpha, c.q0) == (1.0, 2.0, 1.0, 1.0)
    assert (c.amp, c.rho_0, c.kp, c.dt, c.nw, c.divv_switch) == (1.34164, 0.005, 0.5, 0.001, 8, 200)
    s = q.default_config("stb", 512, 512, 512)
    # quasi-stb.cpp:177-203
    assert (s.gamma, s.beta, s.amp, s.rho_0, s.rho_m, s.dt) == (3.0, 0.4, 0.3464101615, 0.1, 0.5, 0.0005)


@pytest.mark.parametrize("bad,msg", [
    (dict(nx=100), b"one of"), (dict(nz=8), b"multiple of 16"), (dict(emulate_ranks=3, nx=96), b"even"),
    (dict(emulate_ranks=5, nx=64), b"divide"), (dict(precision=7), b"precision"), (dict(dt=0.0), b"positive"),
])
def test_invalid_configurations_are_rejected_before_any_device_call(bad, msg):
    import smaiso_quasi_b200 as q
    c = q.default_config("quasi", 16, 16, 32)
    for k, v in bad.items():
        setattr(c, k, v)
    h = ctypes.c_void_p()
    rc = q.lib().quasi_create(ctypes.byref(c), ctypes.byref(h))
    assert rc == -1
    assert msg in q.lib().quasi_last_error()


def test_no_cpu_fallback_without_a_device():
    import torch

    import smaiso_quasi_b200 as q
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(q.QuasiError) as e:
        q.Simulation(q.default_config("quasi", 16, 16, 32))
    assert e.value.code == -6


@pytest.mark.parametrize("kind", ["planar", "undulated", "interface", "droplet", "stb", "focal_conic"])
def test_initial_conditions_match_the_oracle(kind):
    import smaiso_quasi_b200 as q
    variant = "stb" if kind == "stb" else "quasi"
    cfg = q.default_config(variant, 16, 32, 48)
    kw = dict(eps_h=0.05, q_h=0.3) if kind == "interface" else {}
    got = q.initial_condition(cfg, kind, seed=11, **kw)
    m = qo.Model(nx=16, ny=32, nz=48) if variant == "quasi" else qo.Model.stb(nx=16, ny=32, nz=48)
    ref = qo.focal_conic_ic(m, 6.0) if kind == "focal_conic" else qo.ic_field(m, kind, seed=11, **kw)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-15)


def test_noise_stream_matches_the_oracle_exactly():
    import smaiso_quasi_b200 as q
    cfg = q.default_config("quasi", 16, 16, 16)
    a = q.initial_condition(cfg, "planar", seed=99, noise=1e-3, amp0=1e-300)
    b = (2.0 * qo.splitmix_uniform(99, 16 ** 3) - 1.0).reshape(16, 16, 16) * 1e-3
    np.testing.assert_allclose(a, b, rtol=0, atol=1e-18)


def test_ensemble_rejects_a_bad_member_and_names_it():
    """quasi_ensemble_create validates every member before touching a device;
    the error names the failing member."""
    import smaiso_quasi_b200 as q
    good = q.default_config("stb", 16, 16, 32)
    bad = q.default_config("stb", 16, 16, 33)
    with pytest.raises(q.QuasiError) as ei:
        q.Ensemble([bad, good])
    assert "ensemble member 0" in str(ei.value)
    lib = q.lib()
    h = ctypes.c_void_p()
    assert lib.quasi_ensemble_create(0, None, ctypes.byref(h)) != 0
    assert lib.quasi_ensemble_destroy(None) == 0
