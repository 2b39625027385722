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

// Complex arithmetic without FMA contraction, in the operation order of
// std::complex<double> (the host tables are compiled with -ffp-contract=off),
// so that host and GPU differ only where sin and cos do.
struct nz {
    double x, y;
};
__device__ __forceinline__ nz nz_mul(nz a, nz b) {
    return nz{__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)), __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x))};
}
__device__ __forceinline__ nz nz_scale(nz a, double s) { return nz{__dmul_rn(a.x, s), __dmul_rn(a.y, s)}; }
__device__ __forceinline__ nz nz_div(nz a, double s) { return nz{__ddiv_rn(a.x, s), __ddiv_rn(a.y, s)}; }
__device__ __forceinline__ nz nz_add(nz a, nz b) { return nz{__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y)}; }
__device__ __forceinline__ nz nz_sub(nz a, nz b) { return nz{__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y)}; }

// alpha[r][j] for r < nr (offset lengths r2[r]), j < nps; one thread each.
__global__ void k_tables_alpha(const int* __restrict__ r2, int nr, int nps, int L, double k, double leng,
                               double2* __restrict__ alpha) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nr * nps) return;
    const int ir = t / nps, ips = t - ir * nps;
    const double kr = __dmul_rn(__dmul_rn(k, sqrt(static_cast<double>(r2[ir]))), leng);
    const double xi = cos(__ddiv_rn(__dmul_rn(kPi, static_cast<double>(ips)), static_cast<double>(nps - 1)));
    // h_l^(1)(kr) upward: h_0 = -i e^{ix} / x, h_1 = -e^{ix} (1/x + i/x^2),
    // h_{l+1} = (2l + 1)/x h_l - h_{l-1}; P_l(xi) upward; the sum term by term
    // as ((i^l (2l + 1)) h_l) P_l
    double s, c;
    sincos(kr, &s, &c);
    const nz e{c, s};
    nz hm = nz_div(nz_mul(nz{-0.0, -1.0}, e), kr);
    nz h = nz_mul(nz{-e.x, -e.y}, nz{__ddiv_rn(1.0, kr), __ddiv_rn(1.0, __dmul_rn(kr, kr))});
    double pm = 1.0, p = xi;
    const nz powi[4] = {nz{1, 0}, nz{0, 1}, nz{-1, 0}, nz{0, -1}};
    nz coeff = nz_scale(nz_mul(nz_scale(powi[0], 1.0), hm), 1.0);
    if (L >= 1) coeff = nz_add(coeff, nz_scale(nz_mul(nz_scale(powi[1], 3.0), h), p));
    for (int l = 1; l < L; ++l) {
        const nz hp = nz_sub(nz_scale(h, __ddiv_rn(__dadd_rn(__dmul_rn(2.0, l), 1.0), kr)), hm);
        const double pp = __ddiv_rn(__dsub_rn(__dmul_rn(__dmul_rn(__dadd_rn(__dmul_rn(2.0, l), 1.0), xi), p),
                                              __dmul_rn(static_cast<double>(l), pm)),
                                    static_cast<double>(l + 1));
        hm = h;
        h = hp;
        pm = p;
        p = pp;
        const double two_l1 = __dadd_rn(__dmul_rn(2.0, static_cast<double>(l + 1)), 1.0);
        coeff = nz_add(coeff, nz_scale(nz_mul(nz_scale(powi[(l + 1) & 3], two_l1), h), p));
    }
    const nz a = nz_mul(nz_div(nz{0.0, k}, __dmul_rn(4.0, kPi)), coeff);
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
    double c = __dadd_rn(__dadd_rn(__dmul_rn(kh[0], u[0]), __dmul_rn(kh[1], u[1])), __dmul_rn(kh[2], u[2]));
    c = fmin(1.0, fmax(-1.0, c));
    const double psi = acos(c);
    const int near = static_cast<int>(floor(__ddiv_rn(__dmul_rn(static_cast<double>(nps - 1), psi), kPi)));
    double psis[2 * kTabMaxOrder];
    for (int q = 0; q < 2 * order; ++q)
        psis[q] = __ddiv_rn(__dmul_rn(kPi, static_cast<double>(near + 1 - order + q)), static_cast<double>(nps - 1));
    const double2* a = alpha + static_cast<long long>(rix[o]) * nps;
    nz acc{0.0, 0.0};
    for (int q = 0; q < 2 * order; ++q) {
        double w = 1.0;  // Lagrange basis q at psi (Interp::evalLagrangeBasis, src/interp.cpp:86-100)
        for (int j = 0; j < 2 * order; ++j)
            if (j != q) w = __dmul_rn(w, __ddiv_rn(__dsub_rn(psi, psis[j]), __dsub_rn(psis[q], psis[j])));
        int ips = near + 1 - order + q;  // one reflection into [0, nps) (Math::flipIdxToRange, src/math.h:144-154)
        if (ips < 0) ips = -ips - 1;
        if (ips >= nps) ips = 2 * nps - ips - 1;
        const double2 v = a[ips];
        acc = nz_add(acc, nz_scale(nz{v.x, v.y}, w));
    }
    transl[t] = make_double2(acc.x, acc.y);
}

}  // namespace
}  // namespace mlfma
