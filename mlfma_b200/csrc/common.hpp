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

// 2x3 projection onto (theta-hat, phi-hat) (Math::toThPh, src/math.h:90-95),
// stored row-major: [cth cph, cth sph, -sth; -sph, cph, 0].
MLFMA_HD void thph_apply(const double* T, const zd* v, zd* out) {
    out[0] = T[0] * v[0] + T[1] * v[1] + T[2] * v[2];
    out[1] = T[3] * v[0] + T[4] * v[1] + T[5] * v[2];
}

}  // namespace mlfma
