"""GPU r2r transforms (the quasi_r2r_* C ABI) against the oracle's FFTW-kind
restatement (scipy.fft.dct/dst, norm=None)."""
import numpy as np
import pytest

from oracle import quasi_oracle as qo

pytestmark = pytest.mark.gpu

# N = 256 on each axis (the headline grid) among them: (256, 16, 32), (16, 256, 32)
GRIDS = [(16, 16, 32), (8, 16, 16), (32, 64, 16), (96, 96, 192), (64, 64, 128), (128, 32, 256), (512, 16, 32),
         (16, 32, 512), (256, 16, 32), (16, 256, 32)]


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("grid", GRIDS)
@pytest.mark.parametrize("plan", sorted(qo.PLAN_KINDS))
def test_r2r_fp64_matches_fftw_kinds(grid, plan):
    import smaiso_quasi_b200 as q
    rng = np.random.default_rng(hash((grid, plan)) % 2**32)
    a = rng.standard_normal(grid)
    ref = qo.r2r3d(a, qo.PLAN_KINDS[plan])
    p = q.R2RPlan(*grid, plan, precision="fp64")
    got = p.execute_host(a)
    assert rel(got, ref) < 1e-14


@pytest.mark.parametrize("grid", [(16, 16, 32), (64, 64, 128), (96, 96, 192), (16, 32, 512), (256, 16, 32),
                                  (16, 256, 32)])
@pytest.mark.parametrize("plan", ["CT", "iCT", "STx", "iSTy", "iSTz"])
def test_r2r_fp32_error(grid, plan):
    import smaiso_quasi_b200 as q
    rng = np.random.default_rng(3)
    a = rng.standard_normal(grid)
    ref = qo.r2r3d(a, qo.PLAN_KINDS[plan])
    got = q.R2RPlan(*grid, plan, precision="fp32").execute_host(a)
    assert rel(got, ref) < 2e-6   # float32 FFT: ~ eps_32 * log2(N) growth


def test_r2r_round_trip_scale():
    """iCT(CT(x)) * 0.125/(NxNyNz) == x  (quasi.cpp:219,440-446)."""
    import smaiso_quasi_b200 as q
    g = (64, 64, 128)
    a = np.random.default_rng(5).standard_normal(g)
    b = q.R2RPlan(*g, "iCT").execute_host(q.R2RPlan(*g, "CT").execute_host(a)) * (0.125 / np.prod(g))
    assert rel(b, a) < 1e-14


# Split-BF16 tensor-core form: x and y of length 256 as contractions with the
# folded DCT/DST matrices (three BF16 products, FP32 accumulation), z by FFT.
# Each contraction pass is ~3.9e-6 relative L2 (tests/cpu/tc_layout.cpp): bound 2e-5
# for the 3-D transform.
TOL_TC = 2e-5


@pytest.mark.parametrize("grid", [(256, 16, 64), (16, 256, 64), (256, 256, 64), (256, 8, 16)])
@pytest.mark.parametrize("plan", sorted(qo.PLAN_KINDS))
def test_r2r_bf16x3_tensor_core(grid, plan):
    import smaiso_quasi_b200 as q
    rng = np.random.default_rng(11)
    a = rng.standard_normal(grid)
    ref = qo.r2r3d(a, qo.PLAN_KINDS[plan])
    got = q.R2RPlan(*grid, plan, precision="bf16x3").execute_host(a)
    err = rel(got, ref)
    assert err < TOL_TC, err
