"""Builds libclspmv_b200.so in-tree with nvcc for sm_100a.

Every ``csrc/*.cu`` and ``csrc/*.cpp`` file is compiled to an object under
``clspmv_mic_b200/_build/`` (rebuilt when the source or any header is newer)
and linked into ``clspmv_mic_b200/libclspmv_b200.so``. No GPU is needed.

    python -m clspmv_mic_b200.build          # or: python clspmv_mic_b200/build.py
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_build"
LIB = PKG / "libclspmv_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC",
          f"-I{ROOT / 'include'}", f"-I{CSRC}"]


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").glob("*.h")))


def _compile(src: Path, newest_header: float, verbose: bool) -> Path:
    obj = OUT_DIR / (src.name + ".o")
    if obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, newest_header):
        return obj
    cmd = [NVCC, *ARCH, "-lineinfo", *COMMON, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd = [os.environ.get("CXX", "g++"), "-O3", "-std=c++17", "-fPIC", f"-I{ROOT / 'include'}",
               f"-I{CSRC}", "-I/usr/local/cuda/include", "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    return obj


def build(verbose: bool = False) -> Path:
    OUT_DIR.mkdir(exist_ok=True)
    sources = sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))
    newest_header = max((h.stat().st_mtime for h in _headers()), default=0.0)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, newest_header, verbose), sources))
    if LIB.exists() and LIB.stat().st_mtime >= max(o.stat().st_mtime for o in objs):
        return LIB
    # --no-undefined: a missing definition fails the build instead of the first load
    cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-Xlinker", "--no-undefined", "-o", str(LIB), *map(str, objs)]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
