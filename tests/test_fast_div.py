"""fast_div (descriptors.hpp), used for every kernel index decomposition, divides exactly for all
divisors and dividends the kernels use (n < 2^31). Compiled from the header's host path."""
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

SRC = r"""
#include <cstdio>
#include <cstdint>
#include <random>
#include "descriptors.hpp"
int main() {
    using ghexb::fast_div;
    long bad = 0;
    // every divisor up to 5000 against every dividend up to 200000
    for (uint32_t d = 1; d <= 5000; ++d) {
        const fast_div f = fast_div::make(d);
        for (uint32_t n = 0; n < 200000; ++n) bad += f.div(n) != n / d;
    }
    // random divisors and dividends up to 2^31 - 1, plus the extremes
    std::mt19937_64 g(1);
    for (int t = 0; t < 2000; ++t) {
        const uint32_t d = 1 + (uint32_t)(g() % 0x7fffffffu);
        const fast_div f = fast_div::make(d);
        for (uint32_t n : {0u, d - 1, d, d + 1, 0x7fffffffu, 0x7ffffffeu}) bad += f.div(n) != n / d;
        for (int k = 0; k < 2000; ++k) { const uint32_t n = (uint32_t)(g() % 0x80000000u); bad += f.div(n) != n / d; }
    }
    std::printf("%ld\n", bad);
    return bad != 0;
}
"""


def test_fast_div_exact(tmp_path):
    src = tmp_path / "fd.cpp"
    exe = tmp_path / "fd"
    src.write_text(SRC)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", str(ROOT / "ghex_b200" / "csrc"), str(src), "-o", str(exe)],
                   check=True)
    res = subprocess.run([str(exe)], capture_output=True, text=True)
    assert res.returncode == 0 and res.stdout.strip() == "0", res.stdout
