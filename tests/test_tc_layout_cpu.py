"""The tensor-core pass's shared-memory layouts, thread mappings and split-BF16
arithmetic on the CPU (tests/cpu/tc_layout.cpp includes the kernel's own
header): offsets are bijective and in bounds, every tile element is loaded and
every output row written exactly once, and the folded three-product
contraction matches FFTW's kinds within the split-BF16 error."""
import pathlib
import shutil
import subprocess

import pytest

HERE = pathlib.Path(__file__).resolve().parent


@pytest.fixture(scope="module")
def lines(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path_factory.mktemp("tc") / "tc_layout"
    subprocess.run([cxx, "-std=c++17", "-O2", "-o", str(exe), str(HERE / "cpu" / "tc_layout.cpp")], check=True,
                   capture_output=True, text=True, timeout=600)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=600).stdout
    return [line.split() for line in out.splitlines() if line.strip()]


def test_layouts_are_bijective(lines):
    lay = [r for r in lines if r[0] == "layout"]
    assert len(lay) == 5
    for r in lay:
        assert len(set(r[2:])) == 1, r   # expected count == distinct offsets / rows


def test_split_bf16_contraction_matches_fftw_kinds(lines):
    errs = [float(r[2]) for r in lines if r[0] == "kind"]
    assert len(errs) == 4
    assert all(e < 1e-5 for e in errs), errs   # ~3.9e-6 per pass (17 significant bits)
