"""The tile transforms' index arithmetic on the CPU: the device code of
r2r_core.cuh (x / y tiles of a CTA and of one warp) and z_pass.cuh (z tiles of a CTA and of one warp,
with and without the one-row shift of the z gradients) compiled for the host and run serially,
against FFTW's REDFT10/01 and RODFT10/01 definitions in long double."""
import pathlib
import shutil
import subprocess

import pytest

HERE = pathlib.Path(__file__).resolve().parent


@pytest.fixture(scope="module")
def results(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path_factory.mktemp("tiles") / "tiles"
    subprocess.run([cxx, "-std=c++17", "-O1", "-o", str(exe), str(HERE / "cpu" / "tiles.cpp")], check=True,
                   capture_output=True, text=True, timeout=600)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=600).stdout
    rows = [line.split() for line in out.splitlines() if line.strip()]
    return {(r[0], r[1], int(r[2])): float(r[3]) for r in rows}


def test_every_case_ran(results):
    assert sum(1 for k in results if k[0] == "tile") == 12
    assert sum(1 for k in results if k[0] == "wtile") == 8
    assert sum(1 for k in results if k[0] == "ztile") == 16
    assert sum(1 for k in results if k[0] == "zwtile") == 10


@pytest.mark.parametrize("family", ["tile", "wtile", "ztile", "zwtile"])
def test_tiles_match_the_definitions(results, family):
    for (fam, typ, n), err in results.items():   # ztile n: 10 N + row blocks
        if fam != family:
            continue
        tol = 1e-14 if typ == "f64" else 1e-6
        assert err < tol, (fam, typ, n, err)
