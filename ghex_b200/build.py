"""Builds libghex_b200.so in-tree for sm_100a.

Host-only sources (pattern builders) are compiled with g++, sources that touch CUDA with nvcc
(`-gencode arch=compute_100a,code=sm_100a -lineinfo`), and everything is linked with nvcc into
ghex_b200/libghex_b200.so with the static CUDA runtime. Objects go to ghex_b200/_build/ and are
rebuilt when a source or header is newer than the object.

    python -m ghex_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libghex_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-v"] + ARCH
GXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wextra", "-Wno-unused-parameter"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build ghex_b200")


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.hpp")) + sorted(INCLUDE.glob("*.h"))


def _stale(obj: Path, src: Path, headers: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in headers)


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    nvcc = _nvcc()
    headers = _headers()
    objs = []
    ptxas_log = []
    for src in sorted(CSRC.glob("*.cpp")) + sorted(CSRC.glob("*.cu")):
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if not force and not _stale(obj, src, headers):
            continue
        if src.suffix == ".cpp":
            cmd = ["g++", *GXX_FLAGS, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
        else:
            cmd = [nvcc, *NVCC_FLAGS, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError(f"compilation of {src.name} failed")
        if src.suffix == ".cu":
            ptxas_log.append(f"== {src.name}\n{res.stderr}")
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc, "-shared", *ARCH, "-cudart", "static", "-o", str(LIB), *map(str, objs)]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("linking libghex_b200.so failed")
    if ptxas_log:
        (BUILD / "ptxas.log").write_text("\n".join(ptxas_log))
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    main()
