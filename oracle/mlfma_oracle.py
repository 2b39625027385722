"""CPU restatement of the reference MLFMA (ellilu11/MLFMA) in numpy.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the
checker and by bench.py's CPU-baseline leg.  The product never calls it.

Pinning: tests/test_oracle.py checks this module against the reference itself,
compiled from its own sources into oracle/_ref (tables, grids, right-hand side
and matvec on seeded dipole and RWG problems), and against the committed
fixtures in tests/golden/ made by tests/golden/make_golden.py from that build.

Every function cites the reference function it restates.  Sizes are meant
for problems of a few thousand unknowns (dense near-field blocks, python loops
over boxes).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

PI = math.acos(-1.0)
C0 = 299792458.0          # src/phys.h:6
MU0 = 1.256637e-6         # src/phys.h:7
P0 = 1.0e-8               # src/phys.h:8
PHYS_C = -1j * C0 * MU0 / (4.0 * PI)  # src/phys.h:10
FEPS = 1.0e-6             # Math::FEPS, src/math.h:16
EPS_NR = 1.0e-9           # FMM::EPS_NR, src/fmm/fmm.h:11

# Direction order of FMM::Dir (src/fmm/fmm.h:13-17) as (dx, dy, dz).
DIRS = [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1),
        (-1, -1, 0), (1, -1, 0), (-1, 1, 0), (1, 1, 0),
        (-1, 0, -1), (1, 0, -1), (-1, 0, 1), (1, 0, 1),
        (0, -1, -1), (0, 1, -1), (0, -1, 1), (0, 1, 1),
        (-1, -1, -1), (1, -1, -1), (-1, 1, -1), (1, 1, -1),
        (-1, -1, 1), (1, -1, 1), (-1, 1, 1), (1, 1, 1)]


# ------------------------------------------------------------------ special functions

def legendre_p(x: float, n: int):
    """P_n(x), P_n'(x) by recurrence (Math::legendreP, src/math.cpp:25-42)."""
    pnm = 1.0
    if n == 0:
        return pnm, 0.0
    pn = x
    for i in range(1, n):
        pnp = ((2.0 * i + 1) * x * pn - i * pnm) / float(i + 1)
        pnm, pn = pn, pnp
    return pn, n * (x * pn - pnm) / (x * x - 1.0)


def gauss_legendre(l: int, eps: float, a: float, b: float):
    """Newton-refined GL nodes and weights (Interp::gaussLegendre, src/interp.cpp:12-52)."""
    leng, mid = b - a, (a + b) / 2.0
    nodes, weights = np.zeros(l), np.zeros(l)
    kmax = l // 2
    if l % 2:
        nodes[kmax] = mid
        _, dp = legendre_p(0.0, l)
        weights[kmax] = leng / (dp * dp)
    for k in range(kmax):
        xk = math.cos(PI * (4.0 * (kmax - k) - 1) / (4.0 * l + 2.0))
        while True:
            p, dp = legendre_p(xk, l)
            xk -= p / dp
            if abs(p / dp) <= eps:
                dpk = dp
                break
        kp = kmax + 1 + k if l % 2 else kmax + k
        km = kmax - 1 - k
        nodes[kp] = leng / 2.0 * xk + mid
        nodes[km] = -leng / 2.0 * xk + mid
        weights[kp] = leng / ((1.0 - xk * xk) * dpk * dpk)
        weights[km] = weights[kp]
    return nodes, weights


def near_gl_node_idx(xi: float, m: int, a: float, b: float) -> int:
    """Interp::getNearGLNodeIdx (src/interp.cpp:63-77)."""
    leng, mid = b - a, (a + b) / 2.0
    x = 2.0 * (xi - mid) / leng
    return int(m - math.floor(((4.0 * m + 2.0) * math.acos(x) / PI + 1.0) / 4.0) - 1)


def lagrange(x: float, xs, k: int) -> float:
    """Interp::evalLagrangeBasis (src/interp.cpp:86-100)."""
    prod = 1.0
    for j in range(len(xs)):
        if j != k:
            prod *= (x - xs[j]) / (xs[k] - xs[j])
    return prod


def flip_idx(i: int, size: int) -> int:  # Math::flipIdxToRange, src/math.h:144-154
    if i < 0:
        return -i - 1
    if i >= size:
        return 2 * size - i - 1
    return i


def wrap_idx(i: int, size: int) -> int:  # Math::wrapIdxToRange, src/math.h:156-166
    if i < 0:
        return i + size
    if i >= size:
        return i - size
    return i


def spherical_hankel1_all(x: float, nmax: int):
    """h_0..h_nmax by upward recurrence (Math::sphericalHankel1, src/math.cpp:66-81)."""
    h = np.zeros(nmax + 1, dtype=complex)
    hnm = -1j * np.exp(1j * x) / x
    h[0] = hnm
    if nmax == 0:
        return h
    hn = -np.exp(1j * x) * (1.0 / x + 1j / (x * x))
    h[1] = hn
    for i in range(1, nmax):
        hnp = (2.0 * i + 1.0) / x * hn - hnm
        hnm, hn = hn, hnp
        h[i + 1] = hn
    return h


def legendre_all(x: float, lmax: int):
    P = np.zeros(lmax + 1)
    P[0] = 1.0
    if lmax:
        pnm, pn = 1.0, x
        P[1] = pn
        for i in range(1, lmax):
            pnp = ((2.0 * i + 1) * x * pn - i * pnm) / float(i + 1)
            pnm, pn = pn, pnp
            P[i + 1] = pn
    return P


def offsets316():
    """The 316 M2L offsets in Math::getINodeDistVecs order (src/math.cpp:106-122)."""
    out = []
    for dz in range(-3, 4):
        for dy in range(-3, 4):
            for dx in range(-3, 4):
                if max(abs(dx), abs(dy), abs(dz)) > 1:
                    out.append((dx, dy, dz))
    return out


OFFSETS = offsets316()
OFFSET_ID = {o: i for i, o in enumerate(OFFSETS)}


# ------------------------------------------------------------------ sources

def dyadic_uv(X, k, u, v):
    """u^T G(X) v (Math::dyadicG, src/math.h:132-142), vectorised over rows of X.

    G is singular at X = 0; those entries come back as 0 (every caller masks
    coincident points: the zero diagonal, coincident triangles), so no
    divide-by-zero is evaluated and a NaN elsewhere stays visible."""
    r0 = np.linalg.norm(X, axis=-1)
    at0 = r0 == 0.0
    r = np.where(at0, 1.0, r0)
    X = np.where(at0[..., None], 1.0, X)
    kr = k * r
    invkrsq = 1.0 / (kr * kr)
    iinvkr = 1j / kr
    rh = X / r[..., None]
    a = 1.0 + iinvkr - invkrsq
    b = 1.0 + 3.0 * iinvkr - 3.0 * invkrsq
    uv = np.sum(u * v, axis=-1)
    urv = np.sum(u * rh, axis=-1) * np.sum(rh * v, axis=-1)
    return np.where(at0, 0.0, np.exp(1j * kr) / r * (a * uv - b * urv))


QUAD_RULES = {  # Triangle::buildQuads (src/sources/triangle.cpp:45-130): (bary or None, weight)
    0: [(None, 0.5)],
    1: [((2 / 3, 1 / 6, 1 / 6), 1 / 6), ((1 / 6, 2 / 3, 1 / 6), 1 / 6), ((1 / 6, 1 / 6, 2 / 3), 1 / 6)],
    2: [(None, 0.1125)] +
       [(p, 0.066197076394253) for p in [(0.059715871789770, 0.470142064105115, 0.470142064105115),
                                          (0.470142064105115, 0.059715871789770, 0.470142064105115),
                                          (0.470142064105115, 0.470142064105115, 0.059715871789770)]] +
       [(p, 0.0629695902724135) for p in [(0.797426985353087, 0.101286507323456, 0.101286507323456),
                                           (0.101286507323456, 0.797426985353087, 0.101286507323456),
                                           (0.101286507323456, 0.101286507323456, 0.797426985353087)]],
    3: [(None, -0.074785022233841)] +
       [(p, 0.087807628716604) for p in [(0.479308067841920, 0.260345966079040, 0.260345966079040),
                                          (0.260345966079040, 0.479308067841920, 0.260345966079040),
                                          (0.260345966079040, 0.260345966079040, 0.479308067841920)]] +
       [(p, 0.026673617804419) for p in [(0.869739794195568, 0.065130102902216, 0.065130102902216),
                                          (0.065130102902216, 0.869739794195568, 0.065130102902216),
                                          (0.065130102902216, 0.065130102902216, 0.869739794195568)]] +
       [(p, 0.0385568804451285) for p in [(0.048690315425316, 0.312865496004874, 0.638444188569810),
                                           (0.638444188569810, 0.048690315425316, 0.312865496004874),
                                           (0.312865496004874, 0.638444188569810, 0.048690315425316),
                                           (0.048690315425316, 0.638444188569810, 0.312865496004874),
                                           (0.312865496004874, 0.048690315425316, 0.638444188569810),
                                           (0.638444188569810, 0.312865496004874, 0.048690315425316)]],
}


# ------------------------------------------------------------------ self terms
# No reference counterpart: the reference leaves out coincident triangles and
# the diagonal (rwg.cpp:97,113-116, dipole.h:65).  With self_terms the dipole
# operator gets a unit diagonal and RWG pairs whose triangles touch are
# integrated in mixed-potential form with the 1/R singularity extracted.

def tri_potentials(P, r):
    """Closed-form potential integrals of the flat triangle with vertices
    P[..., 3, 3] seen from r[..., 3]:
        I0 = int_T 1/|r - r'| dS',   I1 = int_T (rho' - rho)/|r - r'| dS',
    rho being r projected onto the triangle's plane (returned as well).
    Edge-by-edge formulas of Wilton et al., IEEE Trans. Antennas Propag. 32(3),
    1984, and Graglia, IEEE Trans. Antennas Propag. 41(10), 1993."""
    P = np.asarray(P, dtype=float)
    r = np.asarray(r, dtype=float)
    nrm = np.cross(P[..., 1, :] - P[..., 0, :], P[..., 2, :] - P[..., 0, :])
    nrm = nrm / np.linalg.norm(nrm, axis=-1, keepdims=True)
    h = np.sum(nrm * (r - P[..., 0, :]), axis=-1)
    rho = r - h[..., None] * nrm
    ah = np.abs(h)
    I0 = np.zeros(np.broadcast(h, h).shape)
    I1 = np.zeros(rho.shape)
    for i in range(3):
        p, q = P[..., i, :], P[..., (i + 1) % 3, :]
        L = q - p
        ll = np.linalg.norm(L, axis=-1, keepdims=True)
        lh = L / ll
        u = np.cross(lh, nrm)
        t0 = np.sum((p - rho) * u, axis=-1)
        lm = np.sum((p - rho) * lh, axis=-1)
        lp = np.sum((q - rho) * lh, axis=-1)
        r0sq = t0 * t0 + h * h
        rm = np.sqrt(r0sq + lm * lm)
        rp = np.sqrt(r0sq + lp * lp)
        tiny = r0sq <= (1e-12 * ll[..., 0]) ** 2
        with np.errstate(divide="ignore", invalid="ignore"):
            f = np.where(lm >= 0, np.log((rp + lp) / (rm + lm)),
                         np.where(lp <= 0, np.log((rm - lm) / (rp - lp)), np.log((rp + lp) * (rm - lm) / r0sq)))
        f = np.where(tiny, 0.0, f)
        I0 = I0 + t0 * f - ah * (np.arctan2(t0 * lp, r0sq + ah * rp) - np.arctan2(t0 * lm, r0sq + ah * rm))
        I1 = I1 + u * (0.5 * (r0sq * f + lp * rp - lm * rm))[..., None]
    return I0, I1, rho


def smooth_green(R, k):
    """(e^{ikR} - 1)/R without cancellation; ik at R = 0."""
    with np.errstate(divide="ignore", invalid="ignore"):
        v = (-2.0 * np.sin(0.5 * k * R) ** 2 + 1j * np.sin(k * R)) / R
    return np.where(R > 0, v, 1j * k)


class DipoleSources:
    """Dipole (src/sources/dipole.h)."""

    kind = "dipole"
    self_terms = False

    def __init__(self, pos, mom, pw):
        self.pos = np.asarray(pos, dtype=float)
        self.mom = np.asarray(mom, dtype=float)
        self.phat = self.mom / np.linalg.norm(self.mom, axis=1)[:, None]
        self.pw = pw
        self.n = self.pos.shape[0]
        self.centers = self.pos

    def voltage(self):
        # Dipole::buildVoltage (dipole.h:29-32) runs in the delegated ctor with the
        # default moment (Phys::p0, 0, 0) before the given moment is stored
        # (dipole.h:10-24), so the voltage ignores the moment.
        kv = self.pw.wavenum * np.asarray(self.pw.khat)
        p = np.array([P0, 0.0, 0.0])
        return -self.pw.amplitude * np.exp(1j * (self.pos @ kv)) * float(p @ np.asarray(self.pw.pol))

    def patterns(self, idx, center, khat, thph, k):
        """T(dir) e^{ik khat.(c - r_n)} phat_n  (Dipole::getRadAlongDir, dipole.h:47-51;
        Leaf::buildRadPats, leaf.cpp:185-207).  Returns [nsrc, ndir, 2]."""
        ph = np.exp(1j * k * ((center[None, :] - self.pos[idx]) @ khat.T))  # [s, d]
        v = ph[:, :, None] * self.phat[idx][:, None, :]                      # [s, d, 3]
        return np.einsum("drc,sdc->sdr", thph, v)

    def block(self, rows, cols, k):
        """Z[rows, cols], the operator being C k Z (Dipole::getIntegratedRad, dipole.h:62-70)."""
        X = self.pos[rows][:, None, :] - self.pos[cols][None, :, :]
        same = np.all(X == 0.0, axis=-1)
        Xs = np.where(same[..., None], 1.0, X)
        z = dyadic_uv(Xs, k, self.phat[rows][:, None, :], self.phat[cols][None, :, :])
        # self_terms: unit diagonal Z_mm = 1 (the operator is C k Z)
        return np.where(same, 1.0 if self.self_terms else 0.0, z)


class RWGSources:
    """RWG on a triangle mesh (src/sources/rwg.*, triangle.*)."""

    kind = "rwg"
    self_terms = False

    def __init__(self, verts, faces, rwgs, pw, quad_prec=2):
        V = np.asarray(verts, dtype=float)
        F = np.asarray(faces, dtype=int)
        E = np.asarray(rwgs, dtype=int)
        self.pw = pw
        self.n = E.shape[0]
        X = V[F]                                   # [f, 3 verts, 3]
        self.F = F
        self.P = X
        self.area = 0.5 * np.linalg.norm(np.cross(X[:, 1] - X[:, 0], X[:, 2] - X[:, 0]), axis=1)
        self.X0 = X[:, 0]
        self.D0 = X[:, 1] - X[:, 0]
        self.D2 = X[:, 0] - X[:, 2]
        cen = X.mean(axis=1)
        rule = QUAD_RULES[quad_prec]
        self.qw = np.array([w for _, w in rule])
        self.qpts = np.stack([cen if b is None else b[0] * X[:, 0] + b[1] * X[:, 1] + b[2] * X[:, 2]
                              for b, _ in rule], axis=1)  # [f, q, 3]
        self.tri = E[:, 2:4]
        x0, x1 = V[E[:, 0]], V[E[:, 1]]
        self.centers = (x0 + x1) / 2.0
        self.leng = np.linalg.norm(x0 - x1, axis=1)
        self.xpm = np.zeros((self.n, 2, 3))
        for t in range(2):
            fv = F[E[:, 2 + t]]
            free = (fv != E[:, 0:1]) & (fv != E[:, 1:2])
            last = 2 - np.argmax(free[:, ::-1], axis=1)  # last matching vertex
            self.xpm[:, t] = V[fv[np.arange(self.n), last]]

    def integral(self, idx, kvec):
        """I(k) closed form per triangle (RWG::getIntegratedPlaneWave, rwg.cpp:46-86).
        idx: [s]; kvec: [d, 3]. Returns [s, d, 3]."""
        rad = 0.0
        for t in range(2):
            tr = self.tri[idx, t]
            alpha = kvec @ self.D0[tr].T        # [d, s]
            beta = -(kvec @ self.D2[tr].T)
            alpha, beta = alpha.T, beta.T       # [s, d]
            gamma = alpha - beta
            ea, eb = np.exp(1j * alpha), np.exp(1j * beta)
            za, zb, zg = np.abs(alpha) < FEPS, np.abs(beta) < FEPS, np.abs(gamma) < FEPS
            with np.errstate(divide="ignore", invalid="ignore"):
                f0a = np.where(za, -1j, (1.0 - ea) / alpha)
                f0b = np.where(zb, -1j, (1.0 - eb) / beta)
                f1a = np.where(za, -0.5, (1.0 - (1.0 - 1j * alpha) * ea) / (alpha * alpha))
                f1b = np.where(zb, -0.5, (1.0 - (1.0 - 1j * beta) * eb) / (beta * beta))
                f2 = (ea * (alpha * alpha + 2j * alpha - 2.0) + 2.0) / (2.0 * alpha * alpha * alpha)
                I0 = (f0a - f0b) / gamma
                I1 = 1j * (I0 + f1a)
                I2 = -1j * (I0 + f1b)
            dx = (self.X0[tr] - self.xpm[idx, t])[:, None, :]
            D0, D2 = self.D0[tr][:, None, :], self.D2[tr][:, None, :]
            with np.errstate(divide="ignore", invalid="ignore"):
                gen = I0[..., None] * dx + (I1[..., None] * D0 - I2[..., None] * D2) / gamma[..., None]
            deg = -f1a[..., None] * dx - 1j * f2[..., None] * (D0 - D2)
            rv = np.where(zg[..., None], deg, gen)
            ph = np.exp(1j * (kvec @ self.X0[tr].T)).T  # [s, d]
            rad = rad + ph[..., None] * rv * (-1.0 if t else 1.0)
        return self.leng[idx][:, None, None] * rad

    def voltage(self):
        # RWG::buildVoltage (rwg.h:18-21): -amp conj(I . pol), I conjugated by the dot.
        kv = (self.pw.wavenum * np.asarray(self.pw.khat))[None, :]
        I = self.integral(np.arange(self.n), kv)[:, 0, :]
        return -self.pw.amplitude * np.conj(np.conj(I) @ np.asarray(self.pw.pol))

    def patterns(self, idx, center, khat, thph, k):
        """T e^{ik khat.c} conj(I(k khat)) (RWG::getRadAlongDir, rwg.h:23-25). [s, d, 2]."""
        kv = k * khat
        I = self.integral(np.asarray(idx), kv)
        v = np.exp(1j * (kv @ center))[None, :, None] * np.conj(I)
        return np.einsum("drc,sdc->sdr", thph, v)

    def block(self, rows, cols, k):
        """Z[rows, cols] (operator C k Z) by double quadrature over the four triangle pairs,
        skipping coincident triangles and coincident RWGs (RWG::getIntegratedRad,
        rwg.cpp:92-140)."""
        rows, cols = np.asarray(rows), np.asarray(cols)
        out = np.zeros((rows.size, cols.size), dtype=complex)
        nq = self.qw.size
        for ot in range(2):
            to = self.tri[rows, ot]
            ro = self.qpts[to]                             # [r, q, 3]
            uo = ro - self.xpm[rows, ot][:, None, :]
            for st in range(2):
                ts = self.tri[cols, st]
                rs = self.qpts[ts]                         # [c, q, 3]
                vs = rs - self.xpm[cols, st][:, None, :]
                X = ro[:, None, :, None, :] - rs[None, :, None, :, :]   # [r, c, q, q', 3]
                g = dyadic_uv(X, k, uo[:, None, :, None, :], vs[None, :, None, :, :])
                acc = np.einsum("rcpq,p,q->rc", g, self.qw, self.qw)
                mask = to[:, None] != ts[None, :]
                sgn = -1.0 if (ot ^ st) else 1.0
                out += np.where(mask, sgn * acc, 0.0)
        same = np.all(self.centers[rows][:, None, :] == self.centers[cols][None, :, :], axis=-1)
        out = out * (self.leng[rows][:, None] * self.leng[cols][None, :])
        out = np.where(same, 0.0, out)
        if self.self_terms:
            ti, tj = np.nonzero(self.touching(rows, cols))
            m, n = rows[ti], cols[tj]
            out[ti, tj] = 0.5 * (self.mpie(m, n, k) + self.mpie(n, m, k))
        return out

    def touching(self, rows, cols):
        """[r, c]: some triangle of RWG r shares a vertex with some triangle of RWG c."""
        vr = self.F[self.tri[rows]].reshape(len(rows), 6)
        vc = self.F[self.tri[cols]].reshape(len(cols), 6)
        return np.any(vr[:, None, :, None] == vc[None, :, None, :], axis=(2, 3))

    def mpie(self, m, n, k):
        """Z_mn (operator C k Z) for RWG pairs (m[i], n[i]) in mixed-potential form,
        int int [f_m.f_n - (div f_m)(div f_n)/k^2] e^{ikR}/R, with f = s l/(2A) (r - X)
        on triangle T of area A (s = +1 on T+, -1 on T-; div f = s l/A).  The
        source triangle's integral of 1/R is closed form (tri_potentials), the
        rest (e^{ikR} - 1)/R by the triangle rule; the observation triangle by
        the triangle rule."""
        m, n = np.asarray(m), np.asarray(n)
        w2 = 2.0 * self.qw                       # weights summing to 1
        out = np.zeros(m.size, dtype=complex)
        for ot in range(2):
            T = self.tri[m, ot]
            A = self.area[T]
            X = self.xpm[m, ot]
            ro = self.qpts[T]                    # [i, p, 3]
            for st in range(2):
                Tp = self.tri[n, st]
                Ap = self.area[Tp]
                Xp = self.xpm[n, st]
                rs = self.qpts[Tp]               # [i, q, 3]
                I0, I1, rho = tri_potentials(self.P[Tp][:, None, :, :], ro)      # [i, p], [i, p, 3]
                J0 = I0.astype(complex)
                J1 = (I1 + (rho - Xp[:, None, :]) * I0[..., None]).astype(complex)
                R = np.linalg.norm(ro[:, :, None, :] - rs[:, None, :, :], axis=-1)  # [i, p, q]
                gs = smooth_green(R, k) * (Ap[:, None, None] * w2[None, None, :])
                J0 = J0 + gs.sum(axis=-1)
                J1 = J1 + np.einsum("ipq,iqc->ipc", gs, rs - Xp[:, None, :])
                AAp = (A * Ap)[:, None]
                inner = np.einsum("ipc,ipc->ip", ro - X[:, None, :], J1) / (4.0 * AAp) - J0 / (k * k * AAp)
                sgn = -1.0 if (ot ^ st) else 1.0
                out += sgn * A * (inner @ w2)
        return out * self.leng[m] * self.leng[n]


# ------------------------------------------------------------------ tree

class Node:
    __slots__ = ("level", "parent", "branch", "children", "srcs", "center", "leng", "ijk",
                 "nbors", "ilist", "leaf_ilist", "near_nbors", "coeffs", "local", "id", "pat")

    def __init__(self, srcs, level, parent, branch, center, leng, ijk):
        self.level, self.parent, self.branch = level, parent, branch
        self.children = []
        self.srcs = srcs
        self.center, self.leng, self.ijk = center, leng, ijk
        self.nbors, self.ilist, self.leaf_ilist, self.near_nbors = [], [], [], []
        self.coeffs = None
        self.local = None

    @property
    def leaf(self):
        return not self.children


def build_tree(centers, root_leng, max_node_srcs):
    """Count-split octree, strict src > centre bucketing, input order kept
    (Stem ctor, src/fmm/stem.cpp:3-26; Node ctor, src/fmm/node.cpp:33-44)."""
    nodes = []

    def make(srcs, level, parent, branch):
        if parent is None:
            center, leng, ijk = np.zeros(3), root_leng, (0, 0, 0)
        else:
            leng = parent.leng / 2.0
            pm = np.array([1.0 if branch & 1 else -1.0, 1.0 if branch & 2 else -1.0,
                           1.0 if branch & 4 else -1.0])
            center = parent.center + leng / 2.0 * pm
            ijk = (2 * parent.ijk[0] + (branch & 1), 2 * parent.ijk[1] + ((branch >> 1) & 1),
                   2 * parent.ijk[2] + ((branch >> 2) & 1))
        nd = Node(srcs, level, parent, branch, center, leng, ijk)
        nd.id = len(nodes)
        nodes.append(nd)
        if len(srcs) > max_node_srcs:
            c = centers[srcs]
            b = (c[:, 0] > center[0]) + 2 * (c[:, 1] > center[1]) + 4 * (c[:, 2] > center[2])
            for k in range(8):
                nd.children.append(make(srcs[b == k], level + 1, nd, k))
        return nd

    root = make(np.arange(centers.shape[0]), 0, None, 0)
    return root, nodes


def nbr_geq(nd, d):
    """Equal-or-greater-size neighbour along d, each coarser leaf reported once
    (Node::getNeighborGeqSize, src/fmm/nbor.cpp:10-483)."""
    if nd.parent is None:
        return None
    b = (nd.branch & 1, (nd.branch >> 1) & 1, (nd.branch >> 2) & 1)
    mask, dout, all_out, any_out = 0, [0, 0, 0], True, False
    for a in range(3):
        if d[a] == 0:
            continue
        mask |= 1 << a
        out = (d[a] > 0 and b[a] == 1) or (d[a] < 0 and b[a] == 0)
        if out:
            dout[a], any_out = d[a], True
        else:
            all_out = False
    target = nd.branch ^ mask
    if not any_out:
        return nd.parent.children[target]
    nb = nbr_geq(nd.parent, dout)
    if nb is None:
        return None
    if nb.leaf:
        return nb if all_out else None
    return nb.children[target]


def nbrs_leq(nb, d):
    """Leaves of nb touching across d, breadth first (Node::getNeighborsLeqSize, nbor.cpp:490-643)."""
    out, queue = [], [nb]
    while queue:
        cur = queue.pop(0)
        if cur.leaf:
            out.append(cur)
            continue
        for c in range(8):
            cb = (c & 1, (c >> 1) & 1, (c >> 2) & 1)
            if all(not ((d[a] > 0 and cb[a] != 0) or (d[a] < 0 and cb[a] != 1)) for a in range(3)):
                queue.append(cur.children[c])
    return out


def build_lists(nodes):
    """Neighbours, list 2, list 4, near neighbours (buildLists, stem.cpp:48-57, leaf.cpp:50-58;
    buildInteractionList, node.cpp:61-84)."""
    for nd in nodes:
        if nd.parent is None:
            continue
        for d in DIRS:
            nb = nbr_geq(nd, d)
            if nb is None:
                continue
            nd.nbors.append(nb)
            if nd.leaf:
                nd.near_nbors += nbrs_leq(nb, d)
    for nd in nodes:
        if nd.parent is None:
            continue
        ids = {id(x) for x in nd.nbors}
        for bn in nd.parent.nbors:
            if len(bn.srcs) == 0:
                continue
            if bn.leaf and id(bn) not in ids:
                nd.leaf_ilist.append(bn)
                continue
            for ch in bn.children:
                if id(ch) not in ids and len(ch.srcs) > 0:
                    nd.ilist.append(ch)


# ------------------------------------------------------------------ levels and tables

@dataclass
class Level:
    level: int
    nth: int
    nph: int
    L: int
    nps: int
    leng: float
    thetas: np.ndarray
    weights: np.ndarray
    phis: np.ndarray
    khat: np.ndarray
    thph: np.ndarray
    transl: np.ndarray = field(default=None)


def make_level(level, k, root_leng, digits, over_interp, order):
    """Angles::buildAngularSamples/Matrices (src/fmm/angles.cpp:3-55) and the
    translation table (Tables::getAlpha/getInterpPsi/buildTranslationTable,
    src/fmm/tables.cpp:90-220)."""
    leng = root_leng / 2.0 ** level
    tau = int(math.ceil(1.73 * k * leng + 2.16 * digits ** (2.0 / 3.0) * (k * leng) ** (1.0 / 3.0)))
    L = int(math.floor(0.5 * tau))
    nth = tau + 1
    th, w = gauss_legendre(nth, EPS_NR, 0.0, PI)
    w = w * np.sin(th)
    nph = 2 * nth
    ph = np.array([2.0 * PI * i / float(nph) for i in range(nph)])
    TH, PH = np.meshgrid(th, ph, indexing="ij")
    khat = np.stack([np.sin(TH) * np.cos(PH), np.sin(TH) * np.sin(PH), np.cos(TH)], -1).reshape(-1, 3)
    thph = np.stack([np.stack([np.cos(TH) * np.cos(PH), np.cos(TH) * np.sin(PH), -np.sin(TH)], -1),
                     np.stack([-np.sin(PH), np.cos(PH), np.zeros_like(PH)], -1)], -2).reshape(-1, 2, 3)
    nps = int(math.floor(over_interp * (nth - 1)))
    lv = Level(level, nth, nph, L, nps, leng, th, w, ph, khat, thph)
    alpha = {}
    for o in OFFSETS:
        r2 = o[0] ** 2 + o[1] ** 2 + o[2] ** 2
        if r2 in alpha:
            continue
        kr = k * math.sqrt(r2) * leng
        h = spherical_hankel1_all(kr, L)
        a = np.zeros(nps, dtype=complex)
        for ips in range(nps):
            xi = math.cos(PI * ips / float(nps - 1))
            P = legendre_all(xi, L)
            coeff = sum((1j ** l) * (2.0 * l + 1.0) * h[l] * P[l] for l in range(L + 1))
            a[ips] = 1j * k / (4.0 * PI) * coeff
        alpha[r2] = a
    T = np.zeros((316, nth * nph), dtype=complex)
    for oi, o in enumerate(OFFSETS):
        X = np.array(o, dtype=float)
        rh = X / np.linalg.norm(X)
        a = alpha[o[0] ** 2 + o[1] ** 2 + o[2] ** 2]
        psi = np.arccos(np.clip(khat @ rh, -1.0, 1.0))
        near = np.floor((nps - 1) * psi / PI).astype(int)
        idx = near[:, None] + 1 - order + np.arange(2 * order)[None, :]     # [d, 2o]
        xs = PI * idx / float(nps - 1)
        t = np.zeros(nth * nph, dtype=complex)
        for kk in range(2 * order):
            prod = np.ones(nth * nph)
            for j in range(2 * order):
                if j != kk:
                    prod = prod * ((psi - xs[:, j]) / (xs[:, kk] - xs[:, j]))
            fl = np.where(idx[:, kk] < 0, -idx[:, kk] - 1,
                          np.where(idx[:, kk] >= nps, 2 * nps - idx[:, kk] - 1, idx[:, kk]))
            t = t + a[fl] * prod
        T[oi] = t
    lv.transl = T
    return lv


def interp_tables(parent: Level, child: Level, order: int):
    """theta/phi Lagrange tables child -> parent (Tables::getInterpTheta/Phi,
    src/fmm/tables.cpp:7-78): per target row, (near index, 2*order coefficients)."""
    mth, mph = child.nth, child.nph
    th = []
    for tgt in parent.thetas:
        near = near_gl_node_idx(tgt, mth, 0.0, PI)
        xs = []
        for i in range(near + 1 - order, near + order + 1):
            s = child.thetas[flip_idx(i, mth)]
            if i < 0:
                s = -s
            elif i >= mth:
                s = 2.0 * PI - s
            xs.append(s)
        th.append((near, np.array([lagrange(tgt, xs, kk) for kk in range(2 * order)])))
    phs = []
    for tgt in parent.phis:
        near = int(math.floor(mph * tgt / (2.0 * PI)))
        xs = [2.0 * PI * i / float(mph) for i in range(near + 1 - order, near + order + 1)]
        phs.append((near, np.array([lagrange(tgt, xs, kk) for kk in range(2 * order)])))
    return th, phs


def interp_matrices(parent: Level, child: Level, order: int):
    """Dense real matrices of the separable interpolation, with the pole reflection
    written as a half-turn phi shift and a sign flip (Stem::addInterpCoeffs,
    src/fmm/stem.cpp:133-184).  Returns (Ith [nth_p*mph, mth*mph], Iph [nph_p, mph])."""
    th, ph = interp_tables(parent, child, order)
    mth, mph = child.nth, child.nph
    Ith = np.zeros((parent.nth * mph, mth * mph))
    for j, (near, c) in enumerate(th):
        for kk, i in enumerate(range(near + 1 - order, near + order + 1)):
            f = flip_idx(i, mth)
            out = f != i
            for iph in range(mph):
                sp = iph + (mph // 2 if iph < mph // 2 else -mph // 2) if out else iph
                Ith[j * mph + iph, f * mph + sp] += c[kk] * (-1.0 if out else 1.0)
    Iph = np.zeros((parent.nph, mph))
    for j, (near, c) in enumerate(ph):
        for kk, i in enumerate(range(near + 1 - order, near + order + 1)):
            Iph[j, wrap_idx(i, mph)] += c[kk]
    return Ith, Iph


# ------------------------------------------------------------------ operator

class Oracle:
    """The reference's MLFMA operator and GMRES on small problems."""

    def __init__(self, srcs, digits=3, interp_order=3, over_interp=2.0, root_leng=4.0, max_node_srcs=64):
        self.srcs = srcs
        self.k = srcs.pw.wavenum
        self.order = interp_order
        self.root, self.nodes = build_tree(srcs.centers, root_leng, max_node_srcs)
        build_lists(self.nodes)
        self.leaves = [nd for nd in self.nodes if nd.leaf]
        self.max_level = max(nd.level for nd in self.leaves)
        self.levels = {l: make_level(l, self.k, root_leng, digits, over_interp, interp_order)
                       for l in range(2, self.max_level + 1)}
        self.interp = {l: interp_matrices(self.levels[l], self.levels[l + 1], interp_order)
                       for l in range(2, self.max_level)}
        # Radiation patterns (Leaf::buildRadPats, leaf.cpp:185-207).
        for nd in self.leaves:
            if nd.level >= 2 and len(nd.srcs):
                lv = self.levels[nd.level]
                nd.pat = srcs.patterns(nd.srcs, nd.center, lv.khat, lv.thph, self.k)
        # Near-field blocks (Leaf::buildNearRads, leaf.cpp:108-180).
        self.near = []
        for a in self.leaves:
            for b in a.near_nbors:
                if a.id < b.id and len(a.srcs) and len(b.srcs):
                    self.near.append((a.srcs, b.srcs, srcs.block(a.srcs, b.srcs, self.k)))
        for nd in self.nodes:
            for lf in nd.leaf_ilist:
                if len(nd.srcs):
                    self.near.append((lf.srcs, nd.srcs, srcs.block(lf.srcs, nd.srcs, self.k)))
        self.self_blocks = []
        self.diag = np.zeros(srcs.n, dtype=complex)
        for a in self.leaves:
            if len(a.srcs) > 1 or (srcs.self_terms and len(a.srcs)):
                Z = srcs.block(a.srcs, a.srcs, self.k)
                self.self_blocks.append((a.srcs, np.tril(Z, -1)))
                self.diag[a.srcs] = np.diag(Z)  # zero unless self_terms
        for nd in self.nodes:
            if nd.level >= 2 and len(nd.srcs):
                lv = self.levels[nd.level]
                nd.local = np.zeros((lv.nth * lv.nph, 2), dtype=complex)

    # ---- stages
    def _upward(self, nd, x):
        """S2M (Leaf::buildMpoleCoeffs, leaf.cpp:212-230) and M2M with the shift on
        the child grid (Stem::buildMpoleCoeffs, stem.cpp:72-103)."""
        lv = self.levels[nd.level]
        if nd.leaf:
            nd.coeffs = np.einsum("s,sdr->dr", x[nd.srcs], nd.pat)
            return
        Ith, Iph = self.interp[nd.level]
        acc = np.zeros((lv.nth, lv.nph, 2), dtype=complex)
        for ch in nd.children:
            if not len(ch.srcs):
                continue
            self._upward(ch, x)
            cl = self.levels[ch.level]
            dX = nd.center - ch.center
            sh = np.exp(1j * self.k * (cl.khat @ dX))[:, None] * ch.coeffs
            inner = (Ith @ sh).reshape(lv.nth, cl.nph, 2)
            acc += np.einsum("pm,tmr->tpr", Iph, inner)
        nd.coeffs = acc.reshape(-1, 2)

    def _m2l(self, nd, ref_compat=True):
        """Node::buildMpoleToLocalCoeffs (node.cpp:105-134)."""
        lv = self.levels[nd.level]
        if not nd.ilist:
            if not ref_compat:
                nd.local = np.zeros_like(nd.local)
            return
        acc = np.zeros((lv.nth * lv.nph, 2), dtype=complex)
        for s in nd.ilist:
            off = tuple(int(v) for v in np.array(nd.ijk) - np.array(s.ijk))
            acc += lv.transl[OFFSET_ID[off]][:, None] * s.coeffs
        w = np.repeat(lv.weights, lv.nph) * (2.0 * PI / float(lv.nph))
        nd.local = acc * w[:, None]

    def _l2l(self, parent, child, ref_compat=True):
        """Stem::getShiftedLocalCoeffs + addAnterpCoeffs (stem.cpp:109-131,186-244):
        the transpose of the interpolation, shift on the parent grid."""
        if ref_compat and not parent.ilist:
            return
        pl, cl = self.levels[parent.level], self.levels[child.level]
        Ith, Iph = self.interp[parent.level]
        dX = child.center - parent.center
        sh = (np.exp(1j * self.k * (pl.khat @ dX))[:, None] * parent.local).reshape(pl.nth, pl.nph, 2)
        inner = np.einsum("pm,tpr->tmr", Iph, sh).reshape(-1, 2)      # [nth_p*mph, 2]
        child.local = child.local + (Ith.T @ inner)

    def matvec(self, x, ref_compat=True):
        """y = A x (Solver::evalRvec, src/solver.cpp:41-57); local state persists."""
        x = np.asarray(x, dtype=complex)
        y = np.zeros(self.srcs.n, dtype=complex)
        if self.max_level >= 2:
            for nd in self.nodes:
                if nd.level == 2 and len(nd.srcs):
                    self._upward(nd, x)
            for nd in self.nodes:
                if nd.level >= 2 and len(nd.srcs):
                    self._m2l(nd, ref_compat)
            for l in range(2, self.max_level):
                for nd in self.nodes:
                    if nd.level == l and not nd.leaf:
                        for ch in nd.children:
                            if len(ch.srcs):
                                self._l2l(nd, ch, ref_compat)
            for nd in self.leaves:  # L2T (Leaf::evalFarSols, leaf.cpp:257-280)
                if nd.level >= 2 and len(nd.srcs):
                    y[nd.srcs] += np.einsum("sdr,dr->s", np.conj(nd.pat), nd.local)
        for r, c, Z in self.near:  # evalPairSols / evalNearNonNborSols (leaf.cpp:318-355)
            y[r] += Z @ x[c]
            y[c] += Z.T @ x[r]
        for s, Z in self.self_blocks:  # evalSelfSols (leaf.cpp:361-383)
            y[s] += Z @ x[s] + Z.T @ x[s]
        y += self.diag * x
        return PHYS_C * self.k * y

    def rhs(self):
        return -self.srcs.voltage()

    def dense(self):
        """The exact operator C k Z (zero diagonal unless self_terms), for small N."""
        n = self.srcs.n
        idx = np.arange(n)
        return PHYS_C * self.k * self.srcs.block(idx, idx, self.k)


def farfield(srcs, currents, khat, k):
    """C k (I - khat khat^T) sum_n I_n f_n(k khat) along unit directions khat [d, 3]
    (Node::printFarSols, src/fmm/node.cpp:155-164).  f_n = e^{-i k khat . r_n} phat_n
    for a dipole (dipole.h:53-57), conj(I_n(k khat)) for an RWG (rwg.h:27-29).
    Returns [d, 3] complex."""
    kh = np.asarray(khat, dtype=float).reshape(-1, 3)
    cur = np.asarray(currents, dtype=complex)
    if srcs.kind == "dipole":
        ph = np.exp(-1j * k * (srcs.pos @ kh.T))                 # [s, d]
        v = np.einsum("s,sd,sc->dc", cur, ph, srcs.phat)
    else:
        I = srcs.integral(np.arange(srcs.n), k * kh)             # [s, d, 3]
        v = np.einsum("s,sdc->dc", cur, np.conj(I))
    v = v - kh * np.einsum("dc,dc->d", kh, v)[:, None]
    return PHYS_C * k * v


def gmres_reference(matvec, b, max_iter=500, eps=1e-6):
    """Unrestarted GMRES of the reference: MGS Arnoldi with the Hermitian dot,
    complex-symmetric Givens t = sqrt(z^2 + w^2), stop on |g_{k+1}|/g0, then an
    LU solve of the rotated k x k system (Solver::solve and helpers,
    src/solver.cpp:5-146; Math::givensRotation, src/math.h:168-172)."""
    n = b.shape[0]
    g0 = np.linalg.norm(b)
    Q = [b / g0]
    H = np.zeros((max_iter + 1, max_iter), dtype=complex)
    g = np.zeros(max_iter + 1, dtype=complex)
    g[0] = g0
    cs = np.zeros(max_iter, dtype=complex)
    sn = np.zeros(max_iter, dtype=complex)
    it = 0
    while True:
        k = it
        r = matvec(Q[k])
        h = np.zeros(k + 2, dtype=complex)
        for i in range(k + 1):
            h[i] = np.vdot(Q[i], r)
            r = r - h[i] * Q[i]
        h[k + 1] = np.linalg.norm(r)
        Q.append(r / h[k + 1])
        for i in range(k):
            hp = cs[i] * h[i] + sn[i] * h[i + 1]
            h[i + 1] = -sn[i] * h[i] + cs[i] * h[i + 1]
            h[i] = hp
        t = np.sqrt(h[k] * h[k] + h[k + 1] * h[k + 1])
        cs[k], sn[k] = h[k] / t, h[k + 1] / t
        h[k] = cs[k] * h[k] + sn[k] * h[k + 1]
        h[k + 1] = 0.0
        H[: k + 2, k] = h
        g[k + 1] = -sn[k] * g[k]
        g[k] = cs[k] * g[k]
        it += 1
        if not (abs(g[it]) / g0 > eps and it < max_iter):
            break
    y = np.linalg.solve(H[:it, :it], g[:it])
    x = np.stack(Q[:it], axis=1) @ y
    return x, it


def interp_kat(parent: Level, child: Level, order: int):
    """Known answer of test/tInterp.cpp:18-26,232-322: interpolate and
    anterpolate f = (sqrt(3/8pi) sin(th) e^{i ph}, cos th) between two levels and
    integrate <f, I f> with the quadrature weights; both equal
    int |f|^2 dOmega = 1 + 4 pi / 3 up to interpolation error.
    Returns (interp value, anterp value)."""
    Ith, Iph = interp_matrices(parent, child, order)

    def f(lv):
        TH, PH = np.meshgrid(lv.thetas, lv.phis, indexing="ij")
        return np.stack([0.345494149471336 * np.sin(TH) * np.exp(1j * PH), np.cos(TH) + 0j], -1).reshape(-1, 2)

    def w(lv):
        return np.repeat(lv.weights, lv.nph) * (2.0 * PI / lv.nph)

    fc, fp = f(child), f(parent)
    inner = (Ith @ fc).reshape(parent.nth, child.nph, 2)
    If = np.einsum("pm,tmr->tpr", Iph, inner).reshape(-1, 2)
    v_int = np.sum(w(parent)[:, None] * np.conj(fp) * If)
    # anterpolation: transpose applied to weighted parent samples
    wf = (w(parent)[:, None] * fp).reshape(parent.nth, parent.nph, 2)
    inner2 = np.einsum("pm,tpr->tmr", Iph, wf).reshape(-1, 2)
    Af = Ith.T @ inner2
    v_ant = np.sum(np.conj(Af) * fc)
    return v_int, v_ant
