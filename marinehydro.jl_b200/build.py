"""Build recipe of libmarinehydro_b200.so (sm_100a only).

    python marinehydro.jl_b200/build.py        # incremental
    python marinehydro.jl_b200/build.py --force

Each ``csrc/*.cu`` is compiled by nvcc for ``compute_100a``/``sm_100a`` with
``-lineinfo`` and linked into ``lib/libmarinehydro_b200.so`` in-tree (the CUDA
runtime static, cuBLAS/cuSOLVER dynamic with an rpath).  ``-Xptxas -v`` output
(registers, spills, shared memory per kernel) is kept in
``_build/ptxas_<unit>.txt``.
"""
from __future__ import annotations

import argparse
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
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libmarinehydro_b200.so"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _cuda_home() -> pathlib.Path:
    env = os.environ.get("CUDA_HOME") or os.environ.get("CUDA_PATH")
    if env:
        return pathlib.Path(env)
    nvcc = shutil.which("nvcc")
    if nvcc:
        return pathlib.Path(nvcc).resolve().parent.parent
    return pathlib.Path("/usr/local/cuda")


def _nvcc() -> str:
    return str(_cuda_home() / "bin" / "nvcc")


def _flags():
    return ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                   "-I", str(INCLUDE), "-I", str(CSRC), "--expt-relaxed-constexpr",
                   "-Xptxas", "-v"]


def _headers():
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))


def _stale(target: pathlib.Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: pathlib.Path, force: bool) -> pathlib.Path:
    obj = BUILD / (src.stem + ".o")
    if not force and not _stale(obj, [src, *_headers()]):
        return obj
    cmd = [_nvcc(), *_flags(), "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    (BUILD / f"ptxas_{src.stem}.txt").write_text(r.stdout + r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"nvcc failed on {src.name}")
    return obj


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(sources))) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), sources))
    if force or _stale(LIB, objs):
        cuda_lib = _cuda_home() / "lib64"
        cmd = [_nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs),
               "-L", str(cuda_lib), "-lcusolver", "-lcublas",
               "-Xlinker", f"-rpath,{cuda_lib}"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link of libmarinehydro_b200.so failed")
    if verbose:
        for f in sorted(BUILD.glob("ptxas_*.txt")):
            print(f.read_text())
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
