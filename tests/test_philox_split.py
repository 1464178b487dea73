"""The Philox generator with its first two rounds split into a per-sweep part
and a per-site part (philox_fix / philox_c0 in philox.cuh, used by the sweep
kernels) equals the plain Philox4x32-10 for every input.  Compiled for the host
from the same header the kernels include."""
import pathlib
import subprocess

ROOT = pathlib.Path(__file__).resolve().parents[1]

SRC = r"""
#include "philox.cuh"
#include <cstdio>
#include <random>
int main() {
    std::mt19937_64 g(12345);
    long bad = 0;
    for (int i = 0; i < 300000; ++i) {
        uint32_t c[4], k[2];
        for (auto& x : c) x = (uint32_t)g();
        for (auto& x : k) x = (uint32_t)g();
        if (i % 7 == 0) c[0] = 0xFFFFFFFFu;  // edges of the site word
        if (i % 11 == 0) c[0] = 0u;
        const auto a = csg::philox4x32_10(c[0], c[1], c[2], c[3], k[0], k[1]);
        const auto b = csg::philox_c0(c[0], csg::philox_fix(c[1], c[2], c[3], k[0], k[1]));
        bad += a.v0 != b.v0 || a.v1 != b.v1 || a.v2 != b.v2 || a.v3 != b.v3;
    }
    std::printf("%ld\n", bad);
    return bad != 0;
}
"""


def test_split_philox_equals_full_generator(tmp_path):
    src = tmp_path / "split.cpp"
    src.write_text(SRC)
    exe = tmp_path / "split"
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{ROOT / 'spin-glass_b200' / 'csrc'}",
                    str(src), "-o", str(exe)], check=True, timeout=300)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == "0", out.stdout
