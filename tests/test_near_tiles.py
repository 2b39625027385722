"""The near-field tiling and the near-field kernels' index arithmetic, checked
on the CPU (tests/cpp/near_tiles_check.cpp compiled against plan.cpp): every
copy and read in bounds, every stored entry in exactly one tile, every partial
written once, and the symmetric application equal to the block-row form.  Cases
cover leaves larger than a tile (row-by-row tiles), wide (leaf, node) blocks,
one- and two-source operators, with and without self terms."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_near_tiles_cover_and_stay_in_bounds(tmp_path):
    exe = tmp_path / "near_tiles_check"
    csrc = os.path.join(ROOT, "mlfma_b200", "csrc")
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{csrc}", f"-I{ROOT}/include",
                    os.path.join(ROOT, "tests", "cpp", "near_tiles_check.cpp"), os.path.join(csrc, "plan.cpp"),
                    "-o", str(exe), "-lpthread"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "ALL OK" in out.stdout
