"""The boundary as C and C++ callers see it: include/ghex_b200.h compiles as C99 and C++17 and
every function it declares links against libghex_b200.so (a program referencing each symbol); the
C++ front end include/ghex_b200.hpp compiles against it and, on a GPU, runs a regular exchange with
GHEX's call shapes (make_pattern, wrap_field, make_communication_object, exchange().wait()),
checked against the closed-form periodic owners. The library's own sources include ghex_b200.h,
so a definition that drifts from its declaration fails to compile there."""
import os
import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
INCLUDE = ROOT / "include"
LIBDIR = ROOT / "ghex_b200"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))

needs_compilers = pytest.mark.skipif(not (shutil.which("gcc") and shutil.which("g++")), reason="no C/C++ compiler")


def declared():
    return sorted(set(re.findall(r"^int (ghexb_\w+)\(", (INCLUDE / "ghex_b200.h").read_text(), flags=re.M)))


def link_flags():
    return ["-L", str(LIBDIR), "-lghex_b200", f"-Wl,-rpath,{LIBDIR}"]


@needs_compilers
@pytest.mark.parametrize("lang", ["c", "c++"])
def test_header_compiles_and_every_symbol_links(tmp_path, lang):
    src = tmp_path / ("abi.c" if lang == "c" else "abi.cpp")
    refs = ",\n    ".join(f"(void (*)(void)){n}" for n in declared())
    src.write_text('#include "ghex_b200.h"\n#include <stdio.h>\n'
                   f"static void (*const syms[])(void) = {{\n    {refs}\n}};\n"
                   "int main(void) { printf(\"%d\\n\", (int)(sizeof syms / sizeof syms[0])); return 0; }\n")
    exe = tmp_path / "abi"
    cc = ["gcc", "-std=c99", "-pedantic"] if lang == "c" else ["g++", "-std=c++17"]
    cmd = cc + ["-Wall", "-Wextra", "-Werror", "-I", str(INCLUDE), str(src), "-o", str(exe)] + link_flags()
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and int(out.stdout) == len(declared())


def build_shim(tmp_path) -> Path:
    exe = tmp_path / "shim_exchange"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", str(INCLUDE), "-I", str(CUDA / "include"),
           str(ROOT / "tests" / "cpp" / "shim_exchange.cpp"), "-o", str(exe)] + link_flags() + \
          ["-L", str(CUDA / "lib64"), "-lcudart", f"-Wl,-rpath,{CUDA / 'lib64'}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return exe


@needs_compilers
@pytest.mark.skipif(not (CUDA / "include" / "cuda_runtime.h").exists(), reason="no CUDA toolkit")
def test_cpp_front_end_compiles(tmp_path):
    assert build_shim(tmp_path).exists()


@needs_compilers
@pytest.mark.gpu
def test_cpp_front_end_exchange(tmp_path, cuda):
    exe = build_shim(tmp_path)
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "shim: ok" in res.stdout
