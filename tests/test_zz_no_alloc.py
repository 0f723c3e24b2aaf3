"""quasi_diagnostics_noalloc: the diagnostics for callers that cannot allocate.

Some users of this library run inside a framework whose memory pool owns the
whole device, or in a host loop that must not block on an allocation; they
keep the fields in their own device buffers and need the reductions without
a handle and without any cudaMalloc.  This file is collected last so that a
run stopping at the first failure has already run every other test.

The entry point is checked against the handle's own quasi_diagnostics, on
two calls in a row, within the tolerance the other diagnostics tests use.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-11   # as test_gpu_step.py's diagnostics comparison


def _entry():
    import smaiso_quasi_b200 as q
    fn = q.lib().quasi_diagnostics_noalloc
    fn.argtypes = [ctypes.POINTER(q.Config)] + [ctypes.c_void_p] * 4 + [ctypes.POINTER(ctypes.c_double),
                                                                        ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return q, fn


@pytest.mark.parametrize("engine", ["fp64", "fp32"])
def test_noalloc_matches_handle_on_two_calls(engine):
    """The handle of either form holds psi and rho in double (df in its
    storage type, exact in double): the fields go in as doubles."""
    import torch
    q, fn = _entry()
    cfg = q.default_config("quasi", 32, 32, 64, precision=engine)
    sim = q.Simulation(cfg)
    sim.set_psi(q.initial_condition(cfg, "planar", seed=3))
    sim.init()
    dcfg = q.default_config("quasi", 32, 32, 64, precision="fp64")
    for before in (2, 4):            # two calls in a row, at different states
        sim.step(before)
        prev = sim.field("psi")      # psi_old after the next step
        sim.step(1)
        ref = np.array(sim.diagnostics())
        host = [sim.field("psi"), prev, sim.field("rho"), sim.field("df")]
        dev = [torch.from_numpy(a).to("cuda") for a in host]
        torch.cuda.synchronize()
        out = (ctypes.c_double * 3)()
        rc = fn(ctypes.byref(dcfg), *[ctypes.c_void_p(t.data_ptr()) for t in dev], out, None)
        assert rc == 0, q.lib().quasi_last_error().decode()
        np.testing.assert_allclose(np.array(out), ref, rtol=RTOL)


def test_noalloc_float_fields():
    """Fields in float (cfg->precision FP32): the FP64 sums over the same float
    values as the double path computes them."""
    import torch
    q, fn = _entry()
    cfg = q.default_config("quasi", 32, 32, 64, precision="fp32")
    dcfg = q.default_config("quasi", 32, 32, 64, precision="fp64")
    sim = q.Simulation(cfg)
    sim.set_psi(q.initial_condition(cfg, "planar", seed=3))
    sim.init()
    sim.step(3)
    prev = sim.field("psi")
    sim.step(1)
    host = [a.astype(np.float32) for a in (sim.field("psi"), prev, sim.field("rho"), sim.field("df"))]
    outs = []
    for c, arrs in ((cfg, host), (dcfg, [a.astype(np.float64) for a in host])):
        dev = [torch.from_numpy(a).to("cuda") for a in arrs]
        torch.cuda.synchronize()
        out = (ctypes.c_double * 3)()
        rc = fn(ctypes.byref(c), *[ctypes.c_void_p(t.data_ptr()) for t in dev], out, None)
        assert rc == 0, q.lib().quasi_last_error().decode()
        outs.append(np.array(out))
    np.testing.assert_allclose(outs[0], outs[1], rtol=RTOL)


def test_noalloc_stb_without_df():
    """quasi-stb has no energy: df may be NULL and out[2] is 0."""
    import torch
    q, fn = _entry()
    cfg = q.default_config("stb", 16, 16, 32)
    sim = q.Simulation(cfg)
    sim.set_psi(q.initial_condition(cfg, "stb", seed=4))
    sim.init()
    for before in (1, 3):
        sim.step(before)
        prev = sim.field("psi")
        sim.step(1)
        ref = np.array(sim.diagnostics())
        dev = [torch.from_numpy(a).to("cuda") for a in (sim.field("psi"), prev, sim.field("rho"))]
        torch.cuda.synchronize()
        out = (ctypes.c_double * 3)(7.0, 7.0, 7.0)
        rc = fn(ctypes.byref(cfg), *[ctypes.c_void_p(t.data_ptr()) for t in dev], None, out, None)
        assert rc == 0, q.lib().quasi_last_error().decode()
        np.testing.assert_allclose(np.array(out)[:2], ref[:2], rtol=RTOL)
        assert out[2] == 0.0


def test_noalloc_rejects_host_pointers():
    """Fields in host memory are refused before anything is launched."""
    q, fn = _entry()
    cfg = q.default_config("quasi", 16, 16, 32)
    host = [np.zeros((16, 16, 32)) for _ in range(4)]
    out = (ctypes.c_double * 3)()
    rc = fn(ctypes.byref(cfg), *[ctypes.c_void_p(a.ctypes.data) for a in host], out, None)
    assert rc == -1
    assert b"not device memory" in q.lib().quasi_last_error()


def test_noalloc_rejects_nonpositive_dt():
    q, fn = _entry()
    cfg = q.default_config("quasi", 16, 16, 32)
    cfg.dt = 0.0
    out = (ctypes.c_double * 3)()
    dummy = ctypes.c_void_p(16)                       # never dereferenced: rejected first
    rc = fn(ctypes.byref(cfg), dummy, dummy, dummy, dummy, out, None)
    assert rc == -1


def test_noalloc_rejects_grids_beyond_its_scratch():
    q, fn = _entry()
    cfg = q.default_config("quasi", 512, 512, 256)   # 2^26 cells > 2^25
    out = (ctypes.c_double * 3)()
    dummy = ctypes.c_void_p(16)                       # never dereferenced: rejected first
    rc = fn(ctypes.byref(cfg), dummy, dummy, dummy, dummy, out, None)
    assert rc == -1
    assert b"exceeds the static scratch" in q.lib().quasi_last_error()
