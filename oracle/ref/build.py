"""Builds oracle/_ref/libghex_ref.so: GHEX 0.4.0's own exchange code and test checks, compiled from
the reference sources where they lie, against the stand-ins of oracle/ref/shim — test
infrastructure only.

    python oracle/ref/build.py --reference <GHEX source tree> [--force]
    GHEX_REFERENCE=<GHEX source tree> python oracle/ref/build.py

Nothing is copied from the reference tree; without it the build is skipped. The product never
links or loads this library. It is compiled with -O3 -march=x86-64-v2: it is built where the
reference sources are and runs on other hosts (the GPU machines), so it cannot target the build
host's own instruction set; memcpy, the reference's hot loop, dispatches on the CPU at run time.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE.parent / "_ref"
LIB = OUT / "libghex_ref.so"
SOURCES = ["ghex_ref.cpp", "cs_checks.cpp"]


def build(reference: str | None = None, force: bool = False) -> Path | None:
    """Builds the library from the GHEX tree at `reference` (default: $GHEX_REFERENCE); returns
    None without building when no tree is given or found."""
    reference = reference or os.environ.get("GHEX_REFERENCE")
    if not reference:
        return None
    ref = Path(reference)
    if not (ref / "include" / "ghex").is_dir():
        return None
    OUT.mkdir(exist_ok=True)
    deps = [HERE / s for s in SOURCES] + list((HERE / "shim").rglob("*"))
    if LIB.exists() and not force and all(p.stat().st_mtime <= LIB.stat().st_mtime for p in deps if p.is_file()):
        return LIB
    cmd = ["g++", "-std=c++17", "-O3", "-march=x86-64-v2", "-DNDEBUG", "-fPIC", "-shared",
           "-I", str(HERE / "shim"), "-I", str(ref / "include"), "-I", str(ref),
           *[str(HERE / s) for s in SOURCES], str(ref / "src" / "context.cpp"), "-o", str(LIB)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stderr[-8000:])
        raise RuntimeError("building the reference oracle failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="GHEX source tree (default: $GHEX_REFERENCE)")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.reference, a.force))
