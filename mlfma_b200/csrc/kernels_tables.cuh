// M2L transfer functions built on the GPU (Tables::getAlpha, getInterpPsi,
// buildTranslationTable, src/fmm/tables.cpp:90-220; Math::sphericalHankel1,
// src/math.cpp:66-81; Math::legendreP, src/math.cpp:25-42).  Included once,
// by kernels.cu.
//
//   alpha(r, psi_j) = (i k / 4 pi) sum_{l=0}^{L} i^l (2l+1) h_l(k r d) P_l(cos psi_j),
//       psi_j = pi j / (nps - 1), for the 15 distinct offset lengths r;
//   T(X; khat) = sum_{q < 2 order} lagrange_q(psi) alpha(|X|, psi_{flip(near + 1 - order + q)}),
//       psi = acos(khat . X / |X|),
// for the 316 offsets X in [-3, 3]^3 with max |X_i| > 1, in the order of
// Math::getINodeDistVecs (src/math.cpp:106-122), and every direction of the
// level.  The recurrences and the sums run in the reference's order.
#pragma once

#include "common.hpp"
#include "zmath.cuh"

namespace mlfma {
namespace {

constexpr int kTabThreads = 128;
constexpr int kTabMaxOrder = 5;  // interp_order at most 5 (2 order <= 10 points)

// alpha[r][j] for r < nr (offset lengths r2[r]), j < nps; one thread each.
__global__ void k_tables_alpha(const int* __restrict__ r2, int nr, int nps, int L, double k, double leng,
                               double2* __restrict__ alpha) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nr * nps) return;
    const int ir = t / nps, ips = t - ir * nps;
    const double kr = k * sqrt(static_cast<double>(r2[ir])) * leng;
    const double xi = cos(kPi * ips / static_cast<double>(nps - 1));
    // h_l^(1)(kr) upward (h_0 = -i e^{ix}/x, h_1 = -e^{ix}(1/x + i/x^2)) and
    // P_l(xi) upward, accumulated term by term
    const zd e = expi(kr);
    zd hm = zd{0.0, -1.0} * e * (1.0 / kr);
    zd h = -1.0 * (e * zd{1.0 / kr, 1.0 / (kr * kr)});
    double pm = 1.0, p = xi;
    zd coeff = hm;  // l = 0: i^0 (2 0 + 1) h_0 P_0
    const zd powi[4] = {zd{1, 0}, zd{0, 1}, zd{-1, 0}, zd{0, -1}};
    if (L >= 1) coeff += powi[1] * (3.0 * p) * h;
    for (int l = 1; l < L; ++l) {
        const zd hp = ((2.0 * l + 1.0) / kr) * h - hm;
        const double pp = ((2.0 * l + 1) * xi * p - l * pm) / static_cast<double>(l + 1);
        hm = h;
        h = hp;
        pm = p;
        p = pp;
        coeff += powi[(l + 1) & 3] * ((2.0 * (l + 1) + 1.0) * p) * h;
    }
    const zd a = zd{0.0, k / (4.0 * kPi)} * coeff;
    alpha[t] = make_double2(a.x, a.y);
}

// transl[o][d] for o < 316, d < ndir; offset o: unit vector uhat[o], length
// index rix[o].
__global__ void k_tables_transl(const double* __restrict__ uhat, const int* __restrict__ rix,
                                const double2* __restrict__ alpha, int nps, int order, const double* __restrict__ khat,
                                int ndir, double2* __restrict__ transl) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= 316ll * ndir) return;
    const int o = static_cast<int>(t / ndir), d = static_cast<int>(t - static_cast<long long>(o) * ndir);
    const double* kh = khat + 3 * d;
    const double* u = uhat + 3 * o;
    double c = kh[0] * u[0] + kh[1] * u[1] + kh[2] * u[2];
    c = fmin(1.0, fmax(-1.0, c));
    const double psi = acos(c);
    const int near = static_cast<int>(floor((nps - 1) * psi / kPi));
    double psis[2 * kTabMaxOrder];
    for (int q = 0; q < 2 * order; ++q) psis[q] = kPi * (near + 1 - order + q) / static_cast<double>(nps - 1);
    const double2* a = alpha + static_cast<long long>(rix[o]) * nps;
    zd acc = mkz(0);
    for (int q = 0; q < 2 * order; ++q) {
        double w = 1.0;  // Lagrange basis q at psi (Interp::evalLagrangeBasis, src/interp.cpp:86-100)
        for (int j = 0; j < 2 * order; ++j)
            if (j != q) w *= (psi - psis[j]) / (psis[q] - psis[j]);
        int ips = near + 1 - order + q;  // one reflection into [0, nps) (Math::flipIdxToRange, src/math.h:144-154)
        if (ips < 0) ips = -ips - 1;
        if (ips >= nps) ips = 2 * nps - ips - 1;
        const double2 v = a[ips];
        acc += zd{v.x, v.y} * w;
    }
    transl[t] = make_double2(acc.x, acc.y);
}

}  // namespace
}  // namespace mlfma
