"""Build libquasi_gpu.so (and the quasi_run host driver) in-tree for sm_100a.

    python -m smaiso_quasi_b200.build        (or __graft_entry__.build())

nvcc cross-compiles without a GPU.  Objects go to smaiso_quasi_b200/_build/
(git-ignored); the shared library lands next to this file so it travels with
the source tree.  Rebuilds only what changed (mtime of sources and headers).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libquasi_gpu.so"
DRIVER = PKG / "quasi_run"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "-I", str(ROOT / "include")]
UNITS = ["abi.cu", "r2r_api.cu", "engine_f64.cu", "engine_f32.cu", "ic.cpp", "noalloc.cu"]


def nvcc() -> str:
    for cand in [os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"]:
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[pathlib.Path]:
    return list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))


def _stale(target: pathlib.Path, deps: list[pathlib.Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.stderr.strip():
        sys.stderr.write(r.stderr)


def build(verbose: bool = False, jobs: int | None = None, ptxas_info: bool = False) -> pathlib.Path:
    BUILD.mkdir(exist_ok=True)
    cc = nvcc()
    hdrs = _headers()
    objs, todo = [], []
    for u in UNITS:
        src = CSRC / u
        obj = BUILD / (u + ".o")
        objs.append(obj)
        if _stale(obj, [src] + hdrs) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            todo.append([cc, *ARCH, *NVFLAGS, *extra, "-c", str(src), "-o", str(obj)])
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        list(ex.map(_run, todo))
    if todo or not LIB.exists():
        _run([cc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart", "-lpthread"])
    drv_src = CSRC / "quasi_run.cpp"
    if drv_src.exists() and _stale(DRIVER, [drv_src, LIB] + hdrs):
        _run(["g++", "-O2", "-std=c++17", "-I", str(ROOT / "include"), str(drv_src), "-o", str(DRIVER),
              "-L", str(PKG), "-lquasi_gpu", "-Wl,-rpath,$ORIGIN"])
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
