"""The C++ wrapper (include/mlfma_b200.hpp) compiles against the C ABI and
drives the host-side calls (no GPU needed)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SRC = r"""
#include <cstdio>
#include <random>
#include "mlfma_b200.hpp"
int main() {
    mlfma_config cfg;
    mlfma_config_default(&cfg);
    cfg.max_node_srcs = 16;
    mlfma_planewave pw{1.0, {1, 0, 0}, {0, 0, -1}, 6.283185307179586};
    std::vector<double> pos, mom;
    std::mt19937 g(3);
    std::uniform_real_distribution<double> u(-2.0, 2.0);
    for (int i = 0; i < 500; ++i) {
        for (int k = 0; k < 3; ++k) pos.push_back(u(g));
        mom.push_back(1.0); mom.push_back(0.0); mom.push_back(0.0);
    }
    auto op = mlfma_b200::Operator::dipoles(cfg, pw, pos, mom);
    auto b = op.rhs();
    std::printf("%d %.17g %.17g\n", op.numSrcs(), b[0].real(), b[0].imag());
    auto b2 = op.rhs(pw);  // mlfma_rhs_planewave with the operator's own wave
    std::printf("%d\n", b2 == b ? 1 : 0);
    try {
        std::vector<double> bad(pos.size(), 10.0);
        mlfma_b200::Operator::dipoles(cfg, pw, bad, mom);
    } catch (const std::runtime_error& e) {
        std::printf("caught %s\n", e.what());
    }
    return 0;
}
"""


def test_cpp_wrapper_host_calls(tmp_path):
    lib = os.path.join(ROOT, "mlfma_b200", "libmlfma_b200.so")
    if not os.path.exists(lib):
        pytest.skip("library not built")
    src = tmp_path / "t.cpp"
    src.write_text(SRC)
    exe = tmp_path / "t"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT}/include", str(src), lib, f"-Wl,-rpath,{ROOT}/mlfma_b200",
                    "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    n, re_, im_ = out[0].split()
    assert int(n) == 500
    # reference-compatible voltage: -(-amp e^{ik.r} p0 pol_x) with p0 = 1e-8
    assert abs(complex(float(re_), float(im_))) == pytest.approx(1e-8, rel=1e-12)
    assert out[1] == "1"
    assert out[2].startswith("caught mlfma_b200:") and "root box" in out[2]
