"""The tensor-core interpolation passes' index arithmetic (tc_plan.hpp), run on
the CPU by tests/cpp/tc_check.cpp under AddressSanitizer: the dense weights,
the reflection table, the loads, the stores and the chunking of items, against
a direct application of the interpolation stencils in double, on real plans
(a 4-wavelength cube and the grids of the 8-wavelength sphere, up to 58 x 116
directions); plus the shared-memory layout of every pass."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_tc_passes_match_stencils_and_stay_in_bounds(tmp_path):
    exe = tmp_path / "tc_check"
    csrc = os.path.join(ROOT, "mlfma_b200", "csrc")
    subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address", f"-I{csrc}", f"-I{ROOT}/include",
                    "-I/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp", "tc_check.cpp"),
                    os.path.join(csrc, "plan.cpp"), "-o", str(exe), "-lpthread"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "ALL OK" in out.stdout
