"""Build libtide_b200.so in-tree with nvcc for sm_100a.

Every translation unit is compiled with ``-gencode arch=compute_100a,code=sm_100a``
and ``--fmad=false`` (no FMA contraction, IEEE division), which keeps the
stencil arithmetic in the reference's rounding order.  Objects go to
``tide-gpr_b200/_build/``; the shared library lands next to this file.
"""

from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = ROOT / "csrc"
BUILD = ROOT / "_build"
LIB = PKG / "libtide_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    *ARCH, "-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
]
SOURCES = ["tb_common.cu", "tm2d_abi.cu", "em3d.cu"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _stale(obj: pathlib.Path, src: pathlib.Path) -> bool:
    if not obj.exists():
        return True
    deps = [src, *CSRC.glob("*.cuh"), *(ROOT.parent / "include").glob("*.h"), pathlib.Path(__file__)]
    return any(d.exists() and d.stat().st_mtime > obj.stat().st_mtime for d in deps)


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    BUILD.mkdir(exist_ok=True)
    exe = nvcc()
    jobs = []
    objs = []
    for name in SOURCES:
        src = CSRC / name
        obj = BUILD / (name.rsplit(".", 1)[0] + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            jobs.append([exe, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr:
            print(r.stderr)

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(run, jobs))
    if force or jobs or not LIB.exists():
        run([exe, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs)])
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
