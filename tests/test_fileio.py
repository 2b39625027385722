"""The reference's text formats behind the C ABI (no GPU): plane wave, dipoles
and RWG mesh readers (importPlaneWave, importDipoles, importRWG,
src/fileio.h:8-27,110-202) and the solution writer (Solver::printSols,
src/solver.cpp:149-165).  Operators created from files must equal operators
created from the same arrays (right-hand side bit for bit), must agree with
the reference's own importers reading the same files, and malformed files must
be rejected as the reference rejects them."""
import os

import numpy as np
import pytest

from conftest import needs_ref
from mlfma_b200 import MLFMA, _lib, inputs, read_planewave, write_solution
from mlfma_b200._lib import MlfmaError

PW = inputs.PlaneWave(amplitude=1.3, pol=(0.0, 1.0, 0.0), khat=(0.6, 0.0, -0.8), wavenum=2.0 * np.pi)


def files_rwg(tmp_path, level=2, radius=1.0):
    m = inputs.make_icosphere(level, radius=radius)
    d = str(tmp_path / "rwg")
    inputs.write_rwg(d, m)
    pwp = str(tmp_path / "pwave.txt")
    inputs.write_planewave(pwp, PW)
    return m, [os.path.join(d, f) for f in ("vertices.txt", "faces.txt", "rwgs.txt")], pwp


def test_planewave_roundtrip(tmp_path):
    p = tmp_path / "pw.txt"
    inputs.write_planewave(str(p), PW)
    q = read_planewave(str(p))
    assert q.amplitude == PW.amplitude and q.wavenum == PW.wavenum
    assert tuple(q.pol) == PW.pol and tuple(q.khat) == PW.khat
    # extra values on the line are ignored, as by the reference's istringstream
    p.write_text(p.read_text().strip() + " 9 9\n")
    assert read_planewave(str(p)).wavenum == PW.wavenum


def test_rwg_from_files_equals_arrays(tmp_path):
    m, paths, pwp = files_rwg(tmp_path)
    pw = read_planewave(pwp)
    a = MLFMA.rwg_from_files(*paths, pw, max_node_srcs=16)
    b = MLFMA.rwg(m, PW, max_node_srcs=16)
    assert a.n == b.n == m.n
    assert np.array_equal(a.rhs(), b.rhs())
    assert a.stats() == b.stats()
    a.close()
    b.close()


def test_dipoles_from_file_equals_arrays(tmp_path):
    d = inputs.make_dipoles(500, seed=4)
    p = str(tmp_path / "dip.txt")
    inputs.write_dipoles(p, d)
    a = MLFMA.dipoles_from_file(p, PW, max_node_srcs=16)
    b = MLFMA.dipoles(d, PW, max_node_srcs=16)
    assert a.n == 500 and np.array_equal(a.rhs(), b.rhs())
    a.close()
    b.close()


@pytest.mark.parametrize("bad", ["missing", "short", "blank", "text"])
def test_malformed_files_rejected(tmp_path, bad):
    m, paths, pwp = files_rwg(tmp_path)
    f = paths[2]
    if bad == "missing":
        os.remove(f)
        msg = "Unable to find file"
    else:
        lines = open(f).read().splitlines()
        lines[3] = {"short": "1 2 3", "blank": "", "text": "a b c d"}[bad]
        open(f, "w").write("\n".join(lines) + "\n")
        msg = "Unable to parse line"
    with pytest.raises(MlfmaError) as ei:
        MLFMA.rwg_from_files(*paths, PW, max_node_srcs=16)
    assert ei.value.code == _lib.MLFMA_ERR_ARG
    assert msg in str(ei.value)


def test_solution_writer_format(tmp_path):
    x = np.array([1.5 - 2.25e-3j, -3.0e-12 + 0j, 7.123456789012345e5 + 1j])
    p = tmp_path / "sol.txt"
    write_solution(str(p), x)
    lines = p.read_text().splitlines()
    # std::complex through an ostream with setprecision(15) scientific
    assert lines[0] == "(1.500000000000000e+00,-2.250000000000000e-03)"
    assert lines[1] == "(-3.000000000000000e-12,0.000000000000000e+00)"
    back = np.array([complex(*map(float, ln.strip("()").split(","))) for ln in lines])
    assert np.allclose(back, x, rtol=1e-14, atol=0)


@needs_ref
def test_readers_match_reference_importers(tmp_path):
    from oracle import ref_lib
    m, paths, pwp = files_rwg(tmp_path, level=3, radius=1.0)
    ours = MLFMA.rwg_from_files(*paths, read_planewave(pwp), max_node_srcs=16)
    ref = ref_lib.RefProblem.from_files("rwg", paths, pwp, max_node_srcs=16)
    assert ours.n == ref.n
    assert np.array_equal(ours.rhs(), ref.rhs())  # bit-exact right-hand side
    ours.close()
    d = inputs.make_dipoles(400, seed=6)
    p = str(tmp_path / "dip.txt")
    inputs.write_dipoles(p, d)
    ours = MLFMA.dipoles_from_file(p, read_planewave(pwp), max_node_srcs=16)
    ref = ref_lib.RefProblem.from_files("dipole", p, pwp, max_node_srcs=16)
    assert ours.n == ref.n
    ours.close()
    # both reject the same malformed file
    lines = open(paths[1]).read().splitlines()
    lines[0] = "0 1"
    open(paths[1], "w").write("\n".join(lines) + "\n")
    with pytest.raises(MlfmaError):
        MLFMA.rwg_from_files(*paths, PW, max_node_srcs=16)
    with pytest.raises(RuntimeError):
        ref_lib.RefProblem.from_files("rwg", paths, pwp, max_node_srcs=16)
