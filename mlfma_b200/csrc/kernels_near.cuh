// Near-field kernels: block application (every matvec) and, at setup, the
// near-field entries and radiation patterns.  Included once, by kernels.cu.
#pragma once

#include "common.hpp"
#include "device.cuh"
#include "zmath.cuh"

namespace mlfma {
namespace {

// ------------------------------------------------------------ apply
// y = Z x for the near field (Leaf::evalPairSols, evalNearNonNborSols and
// evalSelfSols, src/fmm/leaf.cpp:318-383; C k is applied when the result is
// written out).  The reference stores each block once and applies it as Z and
// Z^T.
//
// Block-row form: every leaf stores its rows against all sources it meets in
// the near field (both orientations of each reference block, so no transposed
// sums), sharing one column list per leaf.  A warp owns a row: coalesced
// streaming reads of the row, gathers of x through the column list (the eight
// warps of a thread block work on rows of the same leaf, so those gathers hit
// L1), one shuffle reduction per row, a plain store (no atomics, fixed order).
constexpr int kNearRowThreads = 256;
constexpr int kNearRowsPerBlock = kNearRowThreads / 32;

__global__ void __launch_bounds__(kNearRowThreads)
k_near_rows(const DevNearRow* __restrict__ rows, const int4* __restrict__ items, const double2* __restrict__ Z,
            const int* __restrict__ cols, const double2* __restrict__ x, double2* __restrict__ y) {
    const int4 it = items[blockIdx.x];  // row block, first row, row count
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp >= it.z) return;
    const DevNearRow R = rows[it.x];
    const int i = it.y + warp;
    const double2* z = Z + R.off + static_cast<long long>(i) * R.ncol;
    const int* ci = cols + R.col_off;
    double2 a0 = z0(), a1 = z0(), a2 = z0(), a3 = z0();
    int k = lane;
    for (; k + 96 < R.ncol; k += 128) {
        const double2 z0v = ldg_stream(z + k), z1v = ldg_stream(z + k + 32);
        const double2 z2v = ldg_stream(z + k + 64), z3v = ldg_stream(z + k + 96);
        const int c0 = ci[k], c1 = ci[k + 32], c2 = ci[k + 64], c3 = ci[k + 96];
        a0 = cfma(z0v, x[c0], a0);
        a1 = cfma(z1v, x[c1], a1);
        a2 = cfma(z2v, x[c2], a2);
        a3 = cfma(z3v, x[c3], a3);
    }
    for (; k < R.ncol; k += 32) a0 = cfma(ldg_stream(z + k), x[ci[k]], a0);
    const double2 acc = warp_sum(cadd(cadd(a0, a1), cadd(a2, a3)));
    if (lane == 0) y[R.row0 + i] = acc;
}

// ------------------------------------------------------------ setup kernels
struct DevFarLeafGeom {
    double c[3];
};

// Radiation patterns R_n(dir) = T(dir) . e_n(dir) (Leaf::buildRadPats,
// src/fmm/leaf.cpp:185-207) with e_n = e^{ik khat.(c - r_n)} phat_n for a
// dipole (Dipole::getRadAlongDir, src/sources/dipole.h:47-51) and
// e^{ik khat.c} conj(I_n(k khat)) for an RWG (src/sources/rwg.h:23-25).
__global__ void k_patterns(const DevGeomLevel* __restrict__ lvs, const DevFarLeaf* __restrict__ leaves,
                           const DevFarLeafGeom* __restrict__ geo, DevSources S, double2* __restrict__ pat) {
    const DevFarLeaf lf = leaves[blockIdx.x];
    const DevGeomLevel lv = lvs[lf.level];
    const double* c = geo[blockIdx.x].c;
    const int ndir = lv.ndir;
    for (int e = threadIdx.x; e < lf.nsrc * ndir; e += blockDim.x) {
        const int s = e / ndir, d = e - s * ndir;
        const int src = lf.src0 + s;
        const double kv[3] = {lv.khat[3 * d] * S.k, lv.khat[3 * d + 1] * S.k, lv.khat[3 * d + 2] * S.k};
        zd v[3];
        if (S.kind == kDipole) {
            const double* r = S.pos + 3 * src;
            const double dx[3] = {c[0] - r[0], c[1] - r[1], c[2] - r[2]};
            const zd ph = expi(dot3(kv, dx));
            for (int a = 0; a < 3; ++a) v[a] = ph * S.phat[3 * src + a];
        } else {
            zd I[3];
            rwg_plane_wave_integral(S.rwg[src], S.tris, kv, I);
            const zd ph = expi(dot3(kv, c));
            for (int a = 0; a < 3; ++a) v[a] = ph * conj(I[a]);
        }
        zd out[2];
        thph_apply(lv.thph + 6 * d, v, out);
        double2* o = pat + (lf.pat_off + static_cast<long long>(s) * ndir + d) * 2;
        o[0] = make_double2(out[0].x, out[0].y);
        o[1] = make_double2(out[1].x, out[1].y);
    }
}

// True when some triangle of RWG a shares a vertex with some triangle of b.
__device__ bool rwg_touching(const DevSources& S, const RwgGeom& a, const RwgGeom& b) {
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
            for (int u = 0; u < 3; ++u)
                for (int v = 0; v < 3; ++v)
                    if (S.tri_v[3 * a.tri[i] + u] == S.tri_v[3 * b.tri[j] + v]) return true;
    return false;
}

// Z_mn (the operator is A = C k Z) for obs m, src n (Dipole/RWG::getIntegratedRad,
// src/sources/dipole.h:62-70, src/sources/rwg.cpp:92-140).  Coincident
// sources and coincident triangles contribute nothing, unless self_terms is
// set: then a dipole's diagonal is Z_mm = 1, and RWG pairs whose triangles
// touch take the symmetrised mixed-potential value (rwg_mpie).
__device__ zd near_entry(const DevSources& S, int m, int n) {
    if (S.kind == kDipole) {
        const double* a = S.pos + 3 * m;
        const double* b = S.pos + 3 * n;
        if (a[0] == b[0] && a[1] == b[1] && a[2] == b[2]) {
            return mkz(S.self_terms ? 1.0 : 0.0);
        }
        const double X[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
        return dyadic_uv(X, S.k, S.phat + 3 * m, S.phat + 3 * n);
    }
    const RwgGeom& go = S.rwg[m];
    const RwgGeom& gs = S.rwg[n];
    if (S.self_terms && rwg_touching(S, go, gs))
        return 0.5 * (rwg_mpie(go, gs, S.tri_p, S.tri_quad, S.quad_w, S.nq, S.k) +
                      rwg_mpie(gs, go, S.tri_p, S.tri_quad, S.quad_w, S.nq, S.k));
    if (go.center[0] == gs.center[0] && go.center[1] == gs.center[1] && go.center[2] == gs.center[2])
        return mkz(0);
    zd acc = mkz(0);
    for (int ot = 0; ot < 2; ++ot) {
        for (int st = 0; st < 2; ++st) {
            if (go.tri[ot] == gs.tri[st]) continue;
            const double sgn = (ot ^ st) ? -1.0 : 1.0;
            const double* qo = S.tri_quad + static_cast<size_t>(go.tri[ot]) * S.nq * 3;
            const double* qs = S.tri_quad + static_cast<size_t>(gs.tri[st]) * S.nq * 3;
            for (int p = 0; p < S.nq; ++p) {
                const double* ro = qo + 3 * p;
                const double u[3] = {ro[0] - go.xpm[ot][0], ro[1] - go.xpm[ot][1], ro[2] - go.xpm[ot][2]};
                zd inner = mkz(0);
                for (int q = 0; q < S.nq; ++q) {
                    const double* rs = qs + 3 * q;
                    const double v[3] = {rs[0] - gs.xpm[st][0], rs[1] - gs.xpm[st][1], rs[2] - gs.xpm[st][2]};
                    const double X[3] = {ro[0] - rs[0], ro[1] - rs[1], ro[2] - rs[2]};
                    inner += S.quad_w[q] * dyadic_uv(X, S.k, u, v);
                }
                acc += (sgn * S.quad_w[p]) * inner;
            }
        }
    }
    return (go.leng * gs.leng) * acc;
}

// Far field of currents I (caller order) along unit directions khat:
// F = C k (I - khat khat^T) sum_n I_n f_n(k khat), with f_n = e^{-i r_n . k khat}
// phat_n for a dipole (Dipole::getFarAlongDir, src/sources/dipole.h:53-57)
// and conj(I_n(k khat)) for an RWG (RWG::getFarAlongDir, src/sources/rwg.h:27-29);
// the sum and projection are those of Node::printFarSols
// (src/fmm/node.cpp:155-164).  One block per direction.
constexpr int kFarThreads = 256;

__global__ void __launch_bounds__(kFarThreads)
k_farfield(DevSources S, const int* __restrict__ perm, const double2* __restrict__ cur, int n,
           const double* __restrict__ khat, double2 ck, double2* __restrict__ out) {
    __shared__ double2 red[3][kFarThreads];
    const int d = blockIdx.x;
    const double kh[3] = {khat[3 * d], khat[3 * d + 1], khat[3 * d + 2]};
    const double kr[3] = {kh[0] * S.k, kh[1] * S.k, kh[2] * S.k};
    zd acc[3] = {mkz(0), mkz(0), mkz(0)};
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const double2 cv = cur[perm[t]];
        const zd c = zd{cv.x, cv.y};
        if (S.kind == kDipole) {
            const zd ph = c * expi(-dot3(S.pos + 3 * t, kr));
            for (int a = 0; a < 3; ++a) acc[a] += ph * S.phat[3 * t + a];
        } else {
            zd I[3];
            rwg_plane_wave_integral(S.rwg[t], S.tris, kr, I);
            for (int a = 0; a < 3; ++a) acc[a] += c * conj(I[a]);
        }
    }
    for (int a = 0; a < 3; ++a) red[a][threadIdx.x] = make_double2(acc[a].x, acc[a].y);
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (static_cast<int>(threadIdx.x) < s)
            for (int a = 0; a < 3; ++a) red[a][threadIdx.x] = cadd(red[a][threadIdx.x], red[a][threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double2 v[3] = {red[0][0], red[1][0], red[2][0]};
        const double proj = kh[0] * v[0].x + kh[1] * v[1].x + kh[2] * v[2].x;
        const double proji = kh[0] * v[0].y + kh[1] * v[1].y + kh[2] * v[2].y;
        for (int a = 0; a < 3; ++a) {
            const double2 t = make_double2(v[a].x - kh[a] * proj, v[a].y - kh[a] * proji);
            out[3 * d + a] = cmul(ck, t);
        }
    }
}

// Adjoint of the far-field map: g = M^H F for F (ndir x 3) along unit
// directions khat, M the linear map of k_farfield (currents -> far field):
//   g_n = conj(C k) sum_d conj(f_n(k khat_d)) . (I - khat_d khat_d^T) F_d,
// written in caller order.  PF holds the projected F_d (ndir x 3), formed
// first by k_project.  One thread per unknown.  No counterpart in the
// reference (the far-field power gradient uses it).
__global__ void k_project(const double* __restrict__ khat, const double2* __restrict__ F, int ndir,
                          double2* __restrict__ PF) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= ndir) return;
    const double* kh = khat + 3 * d;
    const double2* v = F + 3 * d;
    const double pr = kh[0] * v[0].x + kh[1] * v[1].x + kh[2] * v[2].x;
    const double pi = kh[0] * v[0].y + kh[1] * v[1].y + kh[2] * v[2].y;
    for (int a = 0; a < 3; ++a) PF[3 * d + a] = make_double2(v[a].x - kh[a] * pr, v[a].y - kh[a] * pi);
}

__global__ void k_farfield_adj(DevSources S, const int* __restrict__ perm, int n, const double* __restrict__ khat,
                               const double2* __restrict__ PF, int ndir, double2 ck, double2* __restrict__ g) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    zd acc = mkz(0);
    for (int d = 0; d < ndir; ++d) {
        const double kr[3] = {khat[3 * d] * S.k, khat[3 * d + 1] * S.k, khat[3 * d + 2] * S.k};
        zd cf[3];  // conj(f_t(k khat_d))
        if (S.kind == kDipole) {
            const zd ph = expi(dot3(S.pos + 3 * t, kr));
            for (int a = 0; a < 3; ++a) cf[a] = ph * S.phat[3 * t + a];
        } else {
            rwg_plane_wave_integral(S.rwg[t], S.tris, kr, cf);  // f = conj(I)
        }
        for (int a = 0; a < 3; ++a) {
            const double2 p = PF[3 * d + a];
            acc += cf[a] * zd{p.x, p.y};
        }
    }
    const zd r = zd{ck.x, -ck.y} * acc;
    g[perm[t]] = make_double2(r.x, r.y);
}

// Entries of the block rows: thread per entry.
__global__ void k_near_rows_assemble(const DevNearRow* __restrict__ rows, int nrows, long long total,
                                     const int* __restrict__ cols, DevSources S, double2* __restrict__ Z) {
    const long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= total) return;
    int lo = 0, hi = nrows - 1;
    while (lo < hi) {  // last row block with off <= e
        const int mid = (lo + hi + 1) >> 1;
        if (rows[mid].off <= e) lo = mid; else hi = mid - 1;
    }
    const DevNearRow R = rows[lo];
    const long long loc = e - R.off;
    const int i = static_cast<int>(loc / R.ncol);
    const int k = static_cast<int>(loc - static_cast<long long>(i) * R.ncol);
    const zd z = near_entry(S, R.row0 + i, cols[R.col_off + k]);
    Z[e] = make_double2(z.x, z.y);
}

}  // namespace
}  // namespace mlfma
