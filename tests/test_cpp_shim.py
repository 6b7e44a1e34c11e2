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


def build_shim(tmp_path, name: str = "shim_exchange") -> Path:
    exe = tmp_path / name
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", str(INCLUDE), "-I", str(CUDA / "include"),
           str(ROOT / "tests" / "cpp" / f"{name}.cpp"), "-o", str(exe)] + link_flags() + \
          ["-L", str(CUDA / "lib64"), "-lcudart", f"-Wl,-rpath,{CUDA / 'lib64'}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return exe


@needs_compilers
@pytest.mark.skipif(not (CUDA / "include" / "cuda_runtime.h").exists(), reason="no CUDA toolkit")
@pytest.mark.parametrize("name", ["shim_exchange", "shim_cubed"])
def test_cpp_front_end_compiles(tmp_path, name):
    assert build_shim(tmp_path, name).exists()


@needs_compilers
@pytest.mark.gpu
def test_cpp_front_end_exchange(tmp_path, cuda):
    exe = build_shim(tmp_path)
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "shim: ok" in res.stdout


@needs_compilers
@pytest.mark.gpu
@pytest.mark.parametrize("arch", ["gpu", "cpu"])
@pytest.mark.parametrize("is_vector", [False, True])
def test_cpp_front_end_cubed_sphere(tmp_path, cuda, arch, is_vector):
    """The cubed-sphere test of GHEX (cube edge 10, 2x2 domains per tile, halo 2, 8 float
    components) through the C++ front end, device and host fields, scalar and vector: bit-exact
    against the oracle, which the reference's own known answers pin."""
    import numpy as np
    import cs_cases as CC
    from oracle import cubed_sphere as O
    doms = CC.domains()
    fields = CC.fields()
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        np.array([CC.EDGE, CC.LEVELS, CC.HALO, CC.MEM_HALO, CC.N, CC.NCOMP, len(doms)], dtype=np.int32).tofile(f)
        np.array(doms, dtype=np.int32).tofile(f)
        for a in fields:
            np.asfortranarray(a).ravel(order="F").tofile(f)
    exe = build_shim(tmp_path, "shim_cubed")
    res = subprocess.run([str(exe), str(inp), str(out), arch, "1" if is_vector else "0"], capture_output=True, text=True,
                         timeout=300)
    assert res.returncode == 0 and "shim_cubed: ok" in res.stdout, res.stdout + res.stderr
    got = np.fromfile(out, dtype=np.float32)
    odoms = [O.Domain(t, (x0, x1), (y0, y1), CC.LEVELS) for t, x0, x1, y0, y1 in doms]
    exp = [a.copy(order="F") for a in fields]
    O.exchange(O.make_pattern(CC.EDGE, (CC.HALO,) * 4, odoms), odoms, exp, [(CC.MEM_HALO, CC.MEM_HALO, 0)] * len(doms),
               CC.EDGE, is_vector)
    want = np.concatenate([e.ravel(order="F") for e in exp])
    assert got.size == want.size
    assert np.count_nonzero(got.view(np.uint32) != want.view(np.uint32)) == 0
