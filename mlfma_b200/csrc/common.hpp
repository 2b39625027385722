// Shared complex arithmetic and per-source physics for the host setup code and
// the CUDA kernels.  Every formula cites the reference function it restates
// (paths within the ellilu11/MLFMA project).
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define MLFMA_HD __host__ __device__ __forceinline__
#else
#define MLFMA_HD inline
#endif

namespace mlfma {

constexpr double kPi = 3.14159265358979323846;  // == std::acos(-1.0), src/math.h:10
constexpr double kC0 = 299792458.0;             // src/phys.h:6
constexpr double kMu0 = 1.256637E-6;            // src/phys.h:7
constexpr double kFeps = 1.0E-6;                // Math::FEPS, src/math.h:16

// Complex double with the layout of cuDoubleComplex / std::complex<double>.
struct __attribute__((aligned(16))) zd {
    double x, y;
};

MLFMA_HD zd mkz(double re, double im = 0.0) { return zd{re, im}; }
MLFMA_HD zd operator+(zd a, zd b) { return zd{a.x + b.x, a.y + b.y}; }
MLFMA_HD zd operator-(zd a, zd b) { return zd{a.x - b.x, a.y - b.y}; }
MLFMA_HD zd operator-(zd a) { return zd{-a.x, -a.y}; }
MLFMA_HD zd operator*(zd a, zd b) { return zd{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
MLFMA_HD zd operator*(double s, zd a) { return zd{s * a.x, s * a.y}; }
MLFMA_HD zd operator*(zd a, double s) { return zd{a.x * s, a.y * s}; }
MLFMA_HD zd operator/(zd a, double s) { return zd{a.x / s, a.y / s}; }
MLFMA_HD zd operator/(zd a, zd b) {
    // Smith's algorithm keeps the quotient accurate when |b| spans a wide range.
    if (fabs(b.x) >= fabs(b.y)) {
        const double r = b.y / b.x, den = b.x + b.y * r;
        return zd{(a.x + a.y * r) / den, (a.y - a.x * r) / den};
    }
    const double r = b.x / b.y, den = b.x * r + b.y;
    return zd{(a.x * r + a.y) / den, (a.y * r - a.x) / den};
}
MLFMA_HD zd& operator+=(zd& a, zd b) { a.x += b.x; a.y += b.y; return a; }
MLFMA_HD zd& operator-=(zd& a, zd b) { a.x -= b.x; a.y -= b.y; return a; }
MLFMA_HD zd conj(zd a) { return zd{a.x, -a.y}; }
MLFMA_HD zd iu_times(zd a) { return zd{-a.y, a.x}; }  // i*a
MLFMA_HD double abs2(zd a) { return a.x * a.x + a.y * a.y; }
// e^{i t}
MLFMA_HD zd expi(double t) {
    double s, c;
    sincos(t, &s, &c);
    return zd{c, s};
}
// e^{i t} / r in one step
MLFMA_HD zd expi_over(double t, double r) {
    double s, c;
    sincos(t, &s, &c);
    return zd{c / r, s / r};
}

// Phys::C = -i c0 mu0 / (4 pi)  (src/phys.h:10)
MLFMA_HD zd phys_c() { return zd{0.0, -kC0 * kMu0 / (4.0 * kPi)}; }

MLFMA_HD double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

MLFMA_HD bool approx_zero(double x) { return fabs(x) < kFeps; }  // src/math.h:39-41

// ---------------------------------------------------------------- dyadic G
// u^T G(X) v for the free-space dyadic Green's function
//   G = e^{ikr}/r [ I (1 + i/kr - 1/(kr)^2) - rr^T (1 + 3i/kr - 3/(kr)^2) ]
// (Math::dyadicG, src/math.h:132-142).  u and v are real 3-vectors, so
// u^T G v = e^{ikr}/r [ a (u.v) - b (u.rhat)(rhat.v) ].
MLFMA_HD zd dyadic_uv(const double* X, double k, const double* u, const double* v) {
    const double r = sqrt(X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
    const double kr = k * r, invkrsq = 1.0 / (kr * kr), invkr = 1.0 / kr;
    const double rh[3] = {X[0] / r, X[1] / r, X[2] / r};
    const zd a = zd{1.0 - invkrsq, invkr};
    const zd b = zd{1.0 - 3.0 * invkrsq, 3.0 * invkr};
    const double uv = dot3(u, v);
    const double urv = dot3(u, rh) * dot3(rh, v);
    const zd e = expi_over(kr, r);
    return e * (a * uv - b * urv);
}

// ---------------------------------------------------------------- RWG
// Per-triangle data needed by the analytic plane-wave integral and the
// near-field quadrature (Triangle, src/sources/triangle.h:25-44).
struct TriGeom {
    double X0[3];  // first vertex Xs[0]
    double D0[3];  // Ds[0] = Xs[1] - Xs[0]
    double D2[3];  // Ds[2] = Xs[0] - Xs[2]
};

// Per-RWG data (RWG, src/sources/rwg.h:33-44, ctor src/sources/rwg.cpp:3-26).
struct RwgGeom {
    double center[3];  // midpoint of the shared edge
    double leng;       // length of the shared edge
    double xpm[2][3];  // free vertex of triangle + / -
    int tri[2];        // triangle indices (+, -)
};

// I(k) = l * sum_{T in +,-} s_T int_T (r - X_T) e^{i k.r} dS, evaluated in closed
// form per triangle (RWG::getIntegratedPlaneWave, src/sources/rwg.cpp:28-87, the
// analytic branch).  Writes the complex 3-vector into out[3].
MLFMA_HD void rwg_plane_wave_integral(const RwgGeom& g, const TriGeom* tris, const double* kvec, zd* out) {
    zd rad[3] = {mkz(0), mkz(0), mkz(0)};
    for (int t = 0; t < 2; ++t) {
        const TriGeom& T = tris[g.tri[t]];
        const double alpha = dot3(kvec, T.D0), beta = -dot3(kvec, T.D2), gamma = alpha - beta;
        const double alphasq = alpha * alpha, betasq = beta * beta;
        const zd ea = expi(alpha), eb = expi(beta);
        const zd one = mkz(1.0);
        const zd f0a = approx_zero(alpha) ? mkz(0, -1) : (one - ea) / alpha;
        const zd f0b = approx_zero(beta) ? mkz(0, -1) : (one - eb) / beta;
        const zd f1a = approx_zero(alpha) ? mkz(-0.5) : (one - zd{1.0, -alpha} * ea) / alphasq;
        const zd f1b = approx_zero(beta) ? mkz(-0.5) : (one - zd{1.0, -beta} * eb) / betasq;
        zd v[3];
        if (approx_zero(gamma)) {
            const zd f2 = (ea * zd{alphasq - 2.0, 2.0 * alpha} + mkz(2.0)) / (2.0 * alpha * alphasq);
            const zd if2 = iu_times(f2);
            for (int c = 0; c < 3; ++c)
                v[c] = -(f1a * (T.X0[c] - g.xpm[t][c])) - if2 * (T.D0[c] - T.D2[c]);
        } else {
            const zd I0 = (f0a - f0b) / gamma;
            const zd I1 = iu_times(I0 + f1a);
            const zd I2 = -iu_times(I0 + f1b);
            for (int c = 0; c < 3; ++c)
                v[c] = I0 * (T.X0[c] - g.xpm[t][c]) + (I1 * T.D0[c] - I2 * T.D2[c]) / gamma;
        }
        const zd ph = expi(dot3(kvec, T.X0));
        const double sgn = t ? -1.0 : 1.0;
        for (int c = 0; c < 3; ++c) rad[c] += (ph * v[c]) * sgn;
    }
    for (int c = 0; c < 3; ++c) out[c] = g.leng * rad[c];
}

// ---------------------------------------------------------------- self terms
// No reference counterpart (the reference skips coincident triangles and the
// diagonal, src/sources/rwg.cpp:97,113-116): used when Config::self_terms = 1.

MLFMA_HD void cross3(const double* a, const double* b, double* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// Closed-form potential integrals of the flat triangle P (3 vertices) seen
// from r:  I0 = int_T 1/|r - r'| dS',  I1 = int_T (rho' - rho)/|r - r'| dS',
// rho = r projected onto the plane (also returned).  Edge-by-edge formulas of
// Wilton et al., IEEE Trans. Antennas Propag. 32(3), 1984, and Graglia, IEEE
// Trans. Antennas Propag. 41(10), 1993; the logarithm is taken in the form
// that avoids cancellation for each sign pattern of the edge coordinates.
MLFMA_HD void tri_potentials(const double* P, const double* r, double* I0, double* I1, double* rho) {
    const double e1[3] = {P[3] - P[0], P[4] - P[1], P[5] - P[2]};
    const double e2[3] = {P[6] - P[0], P[7] - P[1], P[8] - P[2]};
    double nv[3];
    cross3(e1, e2, nv);
    const double nn = sqrt(dot3(nv, nv));
    for (int c = 0; c < 3; ++c) nv[c] /= nn;
    const double d0[3] = {r[0] - P[0], r[1] - P[1], r[2] - P[2]};
    const double h = dot3(nv, d0), ah = fabs(h);
    for (int c = 0; c < 3; ++c) rho[c] = r[c] - h * nv[c];
    double s0 = 0.0, s1[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < 3; ++i) {
        const double* p = P + 3 * i;
        const double* q = P + 3 * ((i + 1) % 3);
        const double L[3] = {q[0] - p[0], q[1] - p[1], q[2] - p[2]};
        const double ll = sqrt(dot3(L, L));
        const double lh[3] = {L[0] / ll, L[1] / ll, L[2] / ll};
        double u[3];
        cross3(lh, nv, u);
        const double pr[3] = {p[0] - rho[0], p[1] - rho[1], p[2] - rho[2]};
        const double qr[3] = {q[0] - rho[0], q[1] - rho[1], q[2] - rho[2]};
        const double t0 = dot3(pr, u), lm = dot3(pr, lh), lp = dot3(qr, lh);
        const double r0sq = t0 * t0 + h * h;
        const double rm = sqrt(r0sq + lm * lm), rp = sqrt(r0sq + lp * lp);
        double f = 0.0;
        if (r0sq > (1e-12 * ll) * (1e-12 * ll)) {
            if (lm >= 0.0) f = log((rp + lp) / (rm + lm));
            else if (lp <= 0.0) f = log((rm - lm) / (rp - lp));
            else f = log((rp + lp) * (rm - lm) / r0sq);
        }
        s0 += t0 * f - ah * (atan2(t0 * lp, r0sq + ah * rp) - atan2(t0 * lm, r0sq + ah * rm));
        const double g = 0.5 * (r0sq * f + lp * rp - lm * rm);
        for (int c = 0; c < 3; ++c) s1[c] += g * u[c];
    }
    *I0 = s0;
    for (int c = 0; c < 3; ++c) I1[c] = s1[c];
}

// (e^{ikR} - 1)/R without cancellation (1 - cos = 2 sin^2 of the half angle);
// ik at R = 0.
MLFMA_HD zd smooth_green(double R, double k) {
    if (!(R > 0.0)) return zd{0.0, k};
    const double sh = sin(0.5 * k * R);
    return zd{-2.0 * sh * sh / R, sin(k * R) / R};
}

MLFMA_HD double tri_area(const double* P) {
    const double e1[3] = {P[3] - P[0], P[4] - P[1], P[5] - P[2]};
    const double e2[3] = {P[6] - P[0], P[7] - P[1], P[8] - P[2]};
    double c[3];
    cross3(e1, e2, c);
    return 0.5 * sqrt(dot3(c, c));
}

// Z_mn (operator C k Z) of RWG m (observation) and n (source) in mixed-potential form:
//   int int [f_m . f_n - (div f_m)(div f_n)/k^2] e^{ikR}/R dS' dS,
// f = s l/(2A) (r - X) on a triangle of area A with free vertex X (s = +1 on
// T+, -1 on T-), div f = s l/A.  This equals the dyadic-Green form of the
// other entries (src/sources/rwg.cpp:92-140) after integrating the grad-grad
// term by parts over each RWG's two triangles.  On the source triangle 1/R
// is integrated in closed form (tri_potentials) and (e^{ikR} - 1)/R by the
// triangle rule; the observation triangle by the triangle rule.  quad_w sums
// to 1/2 per triangle (Triangle::buildQuads, src/sources/triangle.cpp:45-130).
MLFMA_HD zd rwg_mpie(const RwgGeom& go, const RwgGeom& gs, const double* tri_p, const double* tri_quad,
                     const double* quad_w, int nq, double k) {
    zd acc = mkz(0);
    for (int ot = 0; ot < 2; ++ot) {
        const double* P = tri_p + 9 * go.tri[ot];
        const double A = tri_area(P);
        const double* X = go.xpm[ot];
        const double* qo = tri_quad + static_cast<size_t>(go.tri[ot]) * nq * 3;
        for (int st = 0; st < 2; ++st) {
            const double* Pp = tri_p + 9 * gs.tri[st];
            const double Ap = tri_area(Pp);
            const double* Xp = gs.xpm[st];
            const double* qs = tri_quad + static_cast<size_t>(gs.tri[st]) * nq * 3;
            zd tri_acc = mkz(0);
            for (int p = 0; p < nq; ++p) {
                const double* ro = qo + 3 * p;
                double I0, I1[3], rho[3];
                tri_potentials(Pp, ro, &I0, I1, rho);
                zd J0 = mkz(I0);
                zd J1[3];
                for (int c = 0; c < 3; ++c) J1[c] = mkz(I1[c] + (rho[c] - Xp[c]) * I0);
                for (int q = 0; q < nq; ++q) {
                    const double* rs = qs + 3 * q;
                    const double d[3] = {ro[0] - rs[0], ro[1] - rs[1], ro[2] - rs[2]};
                    const zd g = smooth_green(sqrt(dot3(d, d)), k) * (2.0 * quad_w[q] * Ap);
                    J0 += g;
                    for (int c = 0; c < 3; ++c) J1[c] += g * (rs[c] - Xp[c]);
                }
                const double u[3] = {ro[0] - X[0], ro[1] - X[1], ro[2] - X[2]};
                const zd vec = u[0] * J1[0] + u[1] * J1[1] + u[2] * J1[2];
                const zd inner = vec / (4.0 * A * Ap) - J0 / (k * k * A * Ap);
                tri_acc += (2.0 * quad_w[p]) * inner;
            }
            acc += ((ot ^ st) ? -A : A) * tri_acc;
        }
    }
    return (go.leng * gs.leng) * acc;
}

// 2x3 projection onto (theta-hat, phi-hat) (Math::toThPh, src/math.h:90-95),
// stored row-major: [cth cph, cth sph, -sth; -sph, cph, 0].
MLFMA_HD void thph_apply(const double* T, const zd* v, zd* out) {
    out[0] = T[0] * v[0] + T[1] * v[1] + T[2] * v[2];
    out[1] = T[3] * v[0] + T[4] * v[1] + T[5] * v[2];
}

}  // namespace mlfma
