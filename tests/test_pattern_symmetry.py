"""The symmetry the mixed far field stores half its radiation patterns by: on
each level's angular grid the antipode of direction (ith, iph) is
(nth - 1 - ith, iph + nph / 2), and for a real basis function the pattern
there is (conj R_theta, -conj R_phi) of the pattern at (ith, iph).  Checked on
the oracle's grids and patterns (CPU): to rounding for dipoles; to the
conditioning of the closed-form triangle integrals (about 1e-8 relative) for
RWGs, which is why the FP64 far field keeps every direction."""
import numpy as np
import pytest

from mlfma_b200 import inputs
from oracle import mlfma_oracle as O

PW = inputs.PlaneWave()


def antipode_pairs(lv):
    nth, nph = lv.nth, lv.nph
    d = np.arange(nth * nph // 2)
    ith, iph = d // nph, d % nph
    return d, (nth - 1 - ith) * nph + (iph + nph // 2) % nph


@pytest.mark.parametrize("level", [2, 3, 4])
def test_grid_is_antipodally_symmetric(level):
    lv = O.make_level(level, PW.wavenum, 4.0, 3, 2.0, 3)
    d, a = antipode_pairs(lv)
    assert sorted(np.concatenate([d, a]).tolist()) == list(range(lv.nth * lv.nph))
    assert np.max(np.abs(lv.khat[a] + lv.khat[d])) <= 1e-14
    th, ph = lv.thph.reshape(-1, 2, 3)[:, 0], lv.thph.reshape(-1, 2, 3)[:, 1]
    assert np.max(np.abs(th[a] - th[d])) <= 1e-14   # theta-hat unchanged
    assert np.max(np.abs(ph[a] + ph[d])) <= 1e-14   # phi-hat flips


def _check(src, n, tol):
    lv = O.make_level(3, PW.wavenum, 4.0, 3, 2.0, 3)
    d, a = antipode_pairs(lv)
    center = np.array([0.25, -0.5, 0.75])
    R = src.patterns(np.arange(n), center, lv.khat, lv.thph.reshape(-1, 2, 3), PW.wavenum)
    err_th = np.abs(R[:, a, 0] - np.conj(R[:, d, 0])).max() / np.abs(R).max()
    err_ph = np.abs(R[:, a, 1] + np.conj(R[:, d, 1])).max() / np.abs(R).max()
    assert max(err_th, err_ph) <= tol, (err_th, err_ph)


def test_dipole_patterns_antipodal_to_rounding():
    d = inputs.make_dipoles(200, seed=3, side=1.0)
    _check(O.DipoleSources(d.pos * 0.5, d.mom, PW), 200, 1e-12)


def test_rwg_patterns_antipodal_to_integral_conditioning():
    # measured 1.3e-8: the closed-form triangle integrals amplify the 1e-16
    # difference between a direction and the negated antipode
    m = inputs.make_icosphere(2, radius=0.5)
    _check(O.RWGSources(m.vertices, m.faces, m.rwgs, PW, quad_prec=2), m.rwgs.shape[0], 1e-7)
