// CUDA kernels of the MLFMA matrix-vector product (FP64 path) and the device
// operator that owns their data.
//
// Data layout in HBM (all complex values interleaved re/im, double2):
//   * sources are permuted into tree order so every octree box owns a
//     contiguous range; x and y are gathered/scattered at the boundary;
//   * per level l: outgoing patterns A_l and local patterns B_l as
//     [box][direction][2 polarisation components];
//   * radiation patterns as [source][direction of its leaf level][2];
//   * transfer functions as [316 offsets][direction] per level;
//   * near-field blocks as dense row-major (list 1 and list 3/4 pairs) or
//     strict-lower packed (self blocks), each applied as Z and Z^T.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

#include "device.cuh"

namespace mlfma {

#define MLFMA_CK(call)                                                                  \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return std::string(#call) + ": " + cudaGetErrorString(e_);                  \
    } while (0)

namespace {

__device__ __forceinline__ double2 z0() { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a*b + c
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
// conj(a)*b + c
__device__ __forceinline__ double2 cjfma(double2 a, double2 b, double2 c) {
    return make_double2(fma(a.x, b.x, fma(a.y, b.y, c.x)), fma(a.x, b.y, fma(-a.y, b.x, c.y)));
}
__device__ __forceinline__ double2 cscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 warp_sum(double2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}
__device__ __forceinline__ void atomic_add_z(double2* p, double2 v) {
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
}

// ------------------------------------------------------------ boundary
__global__ void k_gather(const double2* __restrict__ x, const int* __restrict__ perm,
                         double2* __restrict__ xt, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) xt[t] = x[perm[t]];
}

// y[perm[t]] (+)= ck * (yfar[t] + ynear[t]); perm == nullptr keeps tree order.
__global__ void k_finish(const double2* __restrict__ yfar, const double2* __restrict__ ynear,
                         const int* __restrict__ perm, double2* __restrict__ y, int n, double2 ck,
                         int accumulate) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double2 v = cmul(ck, cadd(yfar[t], ynear[t]));
    const int o = perm ? perm[t] : t;
    y[o] = accumulate ? cadd(y[o], v) : v;
}

// ------------------------------------------------------------ S2M
// a_B[dir] = sum_n x_n R_n[dir]  (Leaf::buildMpoleCoeffs, src/fmm/leaf.cpp:212-230).
// One block per leaf; threads stride over directions, so each source's
// pattern row is read once, coalesced.
__global__ void k_s2m(const DevLevel* __restrict__ lvs, const DevFarLeaf* __restrict__ leaves,
                      const double2* __restrict__ pat, const double2* __restrict__ x) {
    const DevFarLeaf lf = leaves[blockIdx.x];
    const DevLevel lv = lvs[lf.level];
    const int ndir = lv.ndir;
    const double2* R = pat + lf.pat_off * 2;
    const double2* xs = x + lf.src0;
    for (int d = threadIdx.x; d < ndir; d += blockDim.x) {
        double2 a0 = z0(), a1 = z0();
        for (int s = 0; s < lf.nsrc; ++s) {
            const double2 xv = xs[s];
            const double2* r = R + (static_cast<size_t>(s) * ndir + d) * 2;
            a0 = cfma(xv, r[0], a0);
            a1 = cfma(xv, r[1], a1);
        }
        double2* A = lv.A + (static_cast<size_t>(lf.box) * ndir + d) * 2;
        A[0] = a0;
        A[1] = a1;
    }
}

// ------------------------------------------------------------ L2T
// y_m = sum_dir conj(R_m[dir]) . b_B[dir]  (Leaf::evalFarSols, src/fmm/leaf.cpp:257-280;
// the factor C k is applied in k_finish).  One warp per source.
__global__ void k_l2t(const DevLevel* __restrict__ lvs, const DevFarLeaf* __restrict__ leaves,
                      const double2* __restrict__ pat, double2* __restrict__ yfar) {
    const DevFarLeaf lf = leaves[blockIdx.x];
    const DevLevel lv = lvs[lf.level];
    const int ndir = lv.ndir;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const double2* Bb = lv.B + static_cast<size_t>(lf.box) * ndir * 2;
    const double2* R = pat + lf.pat_off * 2;
    for (int s = warp; s < lf.nsrc; s += nw) {
        const double2* r = R + static_cast<size_t>(s) * ndir * 2;
        double2 acc = z0();
        for (int d = lane; d < ndir; d += 32) {
            acc = cjfma(r[2 * d], Bb[2 * d], acc);
            acc = cjfma(r[2 * d + 1], Bb[2 * d + 1], acc);
        }
        acc = warp_sum(acc);
        if (lane == 0) yfar[lf.src0 + s] = acc;
    }
}

// ------------------------------------------------------------ M2M
// Parent outgoing pattern = sum over non-empty children of
// Interp[shift(child)]: shift on the child grid, theta pass with pole
// reflection, then periodic phi pass (Stem::buildMpoleCoeffs and
// addInterpCoeffs, src/fmm/stem.cpp:72-184).  Block (parent, row tile);
// the theta-pass result for the tile lives in shared memory and the parent
// outputs accumulate in registers across children.
template <int NOUT>
__global__ void k_m2m(const DevLevel* __restrict__ lvs, DevTrans T, int rows_per_block) {
    extern __shared__ double2 sm[];
    const int par = blockIdx.x;
    const DevLevel P = lvs[T.plevel];
    const DevLevel C = lvs[T.plevel + 1];
    const int nth = P.nth, nph = P.nph, mph = C.nph, halfm = C.nph / 2;
    const int r0 = blockIdx.y * rows_per_block;
    const int r1 = min(nth, r0 + rows_per_block);
    const int nrow = r1 - r0;
    if (nrow <= 0) return;
    const int nout = nrow * nph;
    double2 acc[NOUT][2];
#pragma unroll
    for (int j = 0; j < NOUT; ++j) acc[j][0] = acc[j][1] = z0();
    for (int ci = T.child_ptr[par]; ci < T.child_ptr[par + 1]; ++ci) {
        const int cbox = T.child_box[ci], oct = T.child_oct[ci];
        const double2* Ac = C.A + static_cast<size_t>(cbox) * C.ndir * 2;
        const double2* sh = C.shift_up + static_cast<size_t>(oct) * C.ndir;
        for (int e = threadIdx.x; e < nrow * mph; e += blockDim.x) {
            const int jr = e / mph, iph = e - jr * mph;
            const int jth = r0 + jr;
            double2 v0 = z0(), v1 = z0();
            for (int q = T.up_th.ptr[jth]; q < T.up_th.ptr[jth + 1]; ++q) {
                const int srow = T.up_th.src[q];
                const bool rf = T.up_th.refl[q];
                const int sp = rf ? (iph < halfm ? iph + halfm : iph - halfm) : iph;
                const double c = rf ? -T.up_th.coef[q] : T.up_th.coef[q];
                const int d = srow * mph + sp;
                const double2 ph = sh[d];
                v0 = cfma(make_double2(c, 0.0), cmul(ph, Ac[2 * d]), v0);
                v1 = cfma(make_double2(c, 0.0), cmul(ph, Ac[2 * d + 1]), v1);
            }
            sm[2 * e] = v0;
            sm[2 * e + 1] = v1;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < NOUT; ++j) {
            const int o = threadIdx.x + j * blockDim.x;
            if (o < nout) {
                const int jr = o / nph, jph = o - jr * nph;
                const double2* row = sm + static_cast<size_t>(jr) * mph * 2;
                for (int q = T.up_ph.ptr[jph]; q < T.up_ph.ptr[jph + 1]; ++q) {
                    const int s = T.up_ph.src[q];
                    const double c = T.up_ph.coef[q];
                    acc[j][0] = cadd(acc[j][0], cscale(c, row[2 * s]));
                    acc[j][1] = cadd(acc[j][1], cscale(c, row[2 * s + 1]));
                }
            }
        }
        __syncthreads();
    }
    const int pbox = T.par_box[par];
    double2* Ap = P.A + (static_cast<size_t>(pbox) * P.ndir + static_cast<size_t>(r0) * nph) * 2;
#pragma unroll
    for (int j = 0; j < NOUT; ++j) {
        const int o = threadIdx.x + j * blockDim.x;
        if (o < nout) {
            Ap[2 * o] = acc[j][0];
            Ap[2 * o + 1] = acc[j][1];
        }
    }
}

// ------------------------------------------------------------ M2L
// b_B = w_theta * (2 pi / nph) * sum_{S in list 2} T[c_B - c_S] a_S
// (Node::buildMpoleToLocalCoeffs, src/fmm/node.cpp:105-134).  One block per
// target box; threads stride over directions.
__global__ void k_m2l(const DevLevel* __restrict__ lvs, int level, const int* __restrict__ boxes,
                      int zero_empty) {
    const DevLevel lv = lvs[level];
    const int b = boxes[blockIdx.x];
    const int p0 = lv.m2l_ptr[b], p1 = lv.m2l_ptr[b + 1];
    const int ndir = lv.ndir;
    for (int d = threadIdx.x; d < ndir; d += blockDim.x) {
        double2* Bo = lv.B + (static_cast<size_t>(b) * ndir + d) * 2;
        if (p0 == p1) {
            if (zero_empty) { Bo[0] = z0(); Bo[1] = z0(); }
            continue;
        }
        double2 a0 = z0(), a1 = z0();
        for (int p = p0; p < p1; ++p) {
            const int s = lv.m2l_src[p], o = lv.m2l_off[p];
            const double2 t = lv.transl[static_cast<size_t>(o) * ndir + d];
            const double2* As = lv.A + (static_cast<size_t>(s) * ndir + d) * 2;
            a0 = cfma(t, As[0], a0);
            a1 = cfma(t, As[1], a1);
        }
        const double w = lv.w[d];
        Bo[0] = cscale(w, a0);
        Bo[1] = cscale(w, a1);
    }
}

// ------------------------------------------------------------ L2L
// child local += Anterp[shift(parent local)]: shift on the parent grid, then
// the transposed phi pass, then the transposed theta pass
// (Stem::getShiftedLocalCoeffs and addAnterpCoeffs, src/fmm/stem.cpp:109-244).
// In reference-compatible mode a parent with an empty list 2 passes nothing
// down (stem.cpp:115).
__global__ void k_l2l(const DevLevel* __restrict__ lvs, DevTrans T, int ref_compat) {
    extern __shared__ double2 sm[];
    const int par = blockIdx.x;
    if (ref_compat && !T.par_ilist[par]) return;
    const DevLevel P = lvs[T.plevel];
    const DevLevel C = lvs[T.plevel + 1];
    const int pth = P.nth, pph = P.nph, cth = C.nth, cph = C.nph, halfc = C.nph / 2;
    const double2* Bp = P.B + static_cast<size_t>(T.par_box[par]) * P.ndir * 2;
    for (int ci = T.child_ptr[par]; ci < T.child_ptr[par + 1]; ++ci) {
        const int cbox = T.child_box[ci], oct = T.child_oct[ci];
        const double2* sh = P.shift_down + static_cast<size_t>(oct) * P.ndir;
        for (int e = threadIdx.x; e < pth * cph; e += blockDim.x) {
            const int ith = e / cph, jph = e - ith * cph;
            double2 v0 = z0(), v1 = z0();
            for (int q = T.dn_ph.ptr[jph]; q < T.dn_ph.ptr[jph + 1]; ++q) {
                const int d = ith * pph + T.dn_ph.src[q];
                const double c = T.dn_ph.coef[q];
                const double2 ph = sh[d];
                v0 = cfma(make_double2(c, 0.0), cmul(ph, Bp[2 * d]), v0);
                v1 = cfma(make_double2(c, 0.0), cmul(ph, Bp[2 * d + 1]), v1);
            }
            sm[2 * e] = v0;
            sm[2 * e + 1] = v1;
        }
        __syncthreads();
        double2* Bc = C.B + static_cast<size_t>(cbox) * C.ndir * 2;
        for (int e = threadIdx.x; e < cth * cph; e += blockDim.x) {
            const int jth = e / cph, jph = e - jth * cph;
            double2 v0 = z0(), v1 = z0();
            for (int q = T.dn_th.ptr[jth]; q < T.dn_th.ptr[jth + 1]; ++q) {
                const bool rf = T.dn_th.refl[q];
                const int sp = rf ? (jph < halfc ? jph + halfc : jph - halfc) : jph;
                const double c = rf ? -T.dn_th.coef[q] : T.dn_th.coef[q];
                const double2* row = sm + (static_cast<size_t>(T.dn_th.src[q]) * cph + sp) * 2;
                v0 = cadd(v0, cscale(c, row[0]));
                v1 = cadd(v1, cscale(c, row[1]));
            }
            Bc[2 * e] = cadd(Bc[2 * e], v0);
            Bc[2 * e + 1] = cadd(Bc[2 * e + 1], v1);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ near field
// y_r += Z x_c and y_c += Z^T x_r for one stored block (Leaf::evalPairSols and
// evalSelfSols, src/fmm/leaf.cpp:329-383; C k applied in k_finish).  One
// block per near block: a warp per row (row sums by shuffle), lanes own
// columns (column sums reduced across warps in shared memory).
constexpr int kNearWarps = 4;
constexpr int kNearMaxC = 4;  // columns per lane per chunk

__global__ void __launch_bounds__(kNearWarps * 32)
k_near(const DevNearBlock* __restrict__ blocks, const double2* __restrict__ Z,
       const double2* __restrict__ x, double2* __restrict__ y) {
    __shared__ double2 colsum[kNearWarps][kNearMaxC * 32];
    const DevNearBlock b = blocks[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double2* zb = Z + b.off;
    for (int c0 = 0; c0 < b.ncol; c0 += 32 * kNearMaxC) {
        double2 cacc[kNearMaxC];
#pragma unroll
        for (int q = 0; q < kNearMaxC; ++q) cacc[q] = z0();
        for (int i = warp; i < b.nrow; i += kNearWarps) {
            const int rowlen = b.self ? i : b.ncol;
            if (c0 >= rowlen) continue;
            const double2* zr = zb + (b.self ? static_cast<long long>(i) * (i - 1) / 2
                                             : static_cast<long long>(i) * b.ncol);
            const double2 xi = x[b.row0 + i];
            double2 rs = z0();
#pragma unroll
            for (int q = 0; q < kNearMaxC; ++q) {
                const int j = c0 + lane + 32 * q;
                if (j < rowlen) {
                    const double2 z = zr[j];
                    rs = cfma(z, x[b.col0 + j], rs);
                    cacc[q] = cfma(z, xi, cacc[q]);
                }
            }
            rs = warp_sum(rs);
            if (lane == 0) atomic_add_z(&y[b.row0 + i], rs);
        }
#pragma unroll
        for (int q = 0; q < kNearMaxC; ++q) colsum[warp][lane + 32 * q] = cacc[q];
        __syncthreads();
        for (int t = threadIdx.x; t < 32 * kNearMaxC; t += blockDim.x) {
            const int j = c0 + t;
            if (j < b.ncol) {
                double2 s = z0();
#pragma unroll
                for (int w = 0; w < kNearWarps; ++w) s = cadd(s, colsum[w][t]);
                atomic_add_z(&y[b.col0 + j], s);
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ setup kernels
struct DevSources {
    int kind;
    double k;
    const double* pos;      // dipole positions (tree order)
    const double* phat;     // dipole unit moments
    const RwgGeom* rwg;     // RWG geometry (tree order)
    const TriGeom* tris;
    const double* tri_quad; // [tri][nq][3]
    const double* quad_w;   // [nq]
    int nq;
};

struct DevFarLeafGeom {
    double c[3];
};

// Radiation patterns R_n(dir) = T(dir) . e_n(dir) (Leaf::buildRadPats,
// src/fmm/leaf.cpp:185-207) with e_n = e^{ik khat.(c - r_n)} phat_n for a
// dipole (Dipole::getRadAlongDir, src/sources/dipole.h:47-51) and
// e^{ik khat.c} conj(I_n(k khat)) for an RWG (src/sources/rwg.h:23-25).
__global__ void k_patterns(const DevLevel* __restrict__ lvs, const DevFarLeaf* __restrict__ leaves,
                           const DevFarLeafGeom* __restrict__ geo, DevSources S, double2* __restrict__ pat) {
    const DevFarLeaf lf = leaves[blockIdx.x];
    const DevLevel lv = lvs[lf.level];
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

// Z_mn / (C k) for obs m, src n (Dipole/RWG::getIntegratedRad,
// src/sources/dipole.h:62-70, src/sources/rwg.cpp:92-140).  Coincident
// sources and coincident triangles contribute nothing.
__device__ zd near_entry(const DevSources& S, int m, int n) {
    if (S.kind == kDipole) {
        const double* a = S.pos + 3 * m;
        const double* b = S.pos + 3 * n;
        if (a[0] == b[0] && a[1] == b[1] && a[2] == b[2]) return mkz(0);
        const double X[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
        return dyadic_uv(X, S.k, S.phat + 3 * m, S.phat + 3 * n);
    }
    const RwgGeom& go = S.rwg[m];
    const RwgGeom& gs = S.rwg[n];
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

__global__ void k_near_assemble(const DevNearBlock* __restrict__ blocks, int nblocks, long long total,
                                DevSources S, double2* __restrict__ Z) {
    const long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= total) return;
    int lo = 0, hi = nblocks - 1;
    while (lo < hi) {  // last block with off <= e
        const int mid = (lo + hi + 1) >> 1;
        if (blocks[mid].off <= e) lo = mid; else hi = mid - 1;
    }
    const DevNearBlock b = blocks[lo];
    const long long loc = e - b.off;
    int i, j;
    if (b.self) {
        i = static_cast<int>((1.0 + sqrt(1.0 + 8.0 * static_cast<double>(loc))) / 2.0);
        while (static_cast<long long>(i) * (i - 1) / 2 > loc) --i;
        while (static_cast<long long>(i + 1) * i / 2 <= loc) ++i;
        j = static_cast<int>(loc - static_cast<long long>(i) * (i - 1) / 2);
    } else {
        i = static_cast<int>(loc / b.ncol);
        j = static_cast<int>(loc - static_cast<long long>(i) * b.ncol);
    }
    const zd z = near_entry(S, b.row0 + i, b.col0 + j);
    Z[e] = make_double2(z.x, z.y);
}

inline int blocks_for(long long n, int bs) { return static_cast<int>((n + bs - 1) / bs); }

}  // namespace

// ================================================================= DeviceOp

DeviceOp::~DeviceOp() {
    if (device_ >= 0) cudaSetDevice(device_);
    for (void* p : allocs_) cudaFree(p);
    if (ev_fork_) cudaEventDestroy(ev_fork_);
    if (ev_join_) cudaEventDestroy(ev_join_);
    if (stream_) cudaStreamDestroy(stream_);
    if (side_) cudaStreamDestroy(side_);
}

template <class T>
T* DeviceOp::alloc(size_t count) {
    void* p = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    if (cudaMalloc(&p, bytes) != cudaSuccess) throw std::runtime_error("cudaMalloc failed");
    allocs_.push_back(p);
    bytes_ += static_cast<long long>(bytes);
    return static_cast<T*>(p);
}

template <class T>
T* DeviceOp::upload(const std::vector<T>& v) {
    T* p = alloc<T>(v.size());
    if (!v.empty() && cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("cudaMemcpy failed");
    return p;
}

static std::vector<double2> to_d2(const std::vector<cplx>& v) {
    std::vector<double2> o(v.size());
    for (size_t i = 0; i < v.size(); ++i) o[i] = make_double2(v[i].real(), v[i].imag());
    return o;
}

std::string DeviceOp::setup(const Plan& plan, int device) {
    try {
        device_ = device;
        MLFMA_CK(cudaSetDevice(device));
        MLFMA_CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        MLFMA_CK(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
        MLFMA_CK(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
        MLFMA_CK(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming));
        n_ = plan.n;
        if (plan.max_level >= kMaxLevels) return "tree deeper than supported";
        const cplx ck = cplx(0, -kC0 * kMu0 / (4.0 * kPi)) * plan.pw.wavenum;
        ck_ = make_double2(ck.real(), ck.imag());
        perm_ = upload(plan.perm);
        xt_ = alloc<double2>(n_);
        yfar_ = alloc<double2>(n_);
        ynear_ = alloc<double2>(n_);
        yt_ = alloc<double2>(n_);

        // ---- levels
        std::memset(&lv_, 0, sizeof(lv_));
        lv_.lmin = plan.lmin;
        lv_.lmax = plan.max_level;
        lv_.k = plan.pw.wavenum;
        lv_.ref_compat = plan.cfg.ref_compat;
        traffic_ = Traffic{};
        for (int l = plan.lmin; l <= plan.max_level; ++l) {
            const Level& L = plan.levels[l];
            DevLevel& d = lv_.lv[l];
            d.nth = L.nth;
            d.nph = L.nph;
            d.ndir = L.ndir;
            d.nbox = static_cast<int>(L.boxes.size());
            const size_t cnt = static_cast<size_t>(d.nbox) * L.ndir * 2;
            d.A = alloc<double2>(cnt);
            d.B = alloc<double2>(cnt);
            MLFMA_CK(cudaMemset(d.A, 0, cnt * sizeof(double2)));
            MLFMA_CK(cudaMemset(d.B, 0, cnt * sizeof(double2)));
            d.transl = upload(to_d2(L.transl));
            d.w = upload(L.m2l_w);
            d.shift_up = upload(to_d2(L.shift_up));
            d.shift_down = upload(to_d2(L.shift_down));
            d.thph = upload(L.thph);
            d.khat = upload(L.khat);
            d.m2l_ptr = upload(L.m2l_ptr);
            d.m2l_src = upload(L.m2l_src);
            d.m2l_off = upload(L.m2l_off);
            max_ndir_ = std::max(max_ndir_, L.ndir);
            // M2L: read a_S and T per pair-direction (cached), write b once.
            traffic_.m2l += static_cast<double>(cnt) * 16.0 * 2.0 + 316.0 * L.ndir * 16.0;
        }
        DevLevel* d_lvs = upload(std::vector<DevLevel>(lv_.lv, lv_.lv + kMaxLevels));
        lv_dev_ = d_lvs;

        // ---- transitions
        trans_.assign(std::max(plan.max_level, 0) + 1, DevTrans{});
        for (int p = plan.lmin; p < plan.max_level; ++p) {
            const Transition& T = plan.trans[p];
            DevTrans& d = trans_[p];
            auto st = [&](const Stencil& s) {
                return DevStencil{upload(s.ptr), upload(s.src), upload(s.refl), upload(s.coef)};
            };
            d.up_th = st(T.up_th);
            d.up_ph = st(T.up_ph);
            d.dn_ph = st(T.dn_ph);
            d.dn_th = st(T.dn_th);
            d.plevel = p;
            d.npar = static_cast<int>(T.par_box.size());
            d.par_box = upload(T.par_box);
            d.par_ilist = upload(T.par_ilist);
            d.child_ptr = upload(T.child_ptr);
            d.child_box = upload(T.child_box);
            d.child_oct = upload(T.child_oct);
            const double nch = static_cast<double>(T.child_box.size());
            const double cdir = plan.levels[p + 1].ndir, pdir = plan.levels[p].ndir;
            traffic_.m2m += nch * cdir * 32.0 + d.npar * pdir * 32.0;
            traffic_.l2l += d.npar * pdir * 32.0 + nch * cdir * 32.0 * 2.0;
        }
        // M2L target lists per level.
        m2l_boxes_.assign(plan.max_level + 1, nullptr);
        m2l_nbox_.assign(plan.max_level + 1, 0);
        for (int l = plan.lmin; l <= plan.max_level; ++l) {
            const Level& L = plan.levels[l];
            std::vector<int> bl;
            for (int b = 0; b < static_cast<int>(L.boxes.size()); ++b)
                if (!plan.cfg.ref_compat || L.m2l_ptr[b + 1] > L.m2l_ptr[b]) bl.push_back(b);
            m2l_nbox_[l] = static_cast<int>(bl.size());
            m2l_boxes_[l] = upload(bl);
        }

        // ---- far leaves and radiation patterns
        h_leaves_.clear();
        std::vector<DevFarLeafGeom> geo;
        for (const FarLeaf& f : plan.far_leaves) {
            h_leaves_.push_back(DevFarLeaf{f.level, f.box, f.src0, f.nsrc, f.pat_off});
            const Node& nd = plan.nodes[plan.levels[f.level].boxes[f.box]];
            geo.push_back(DevFarLeafGeom{{nd.center[0], nd.center[1], nd.center[2]}});
        }
        n_leaves_ = static_cast<int>(h_leaves_.size());
        leaves_ = upload(h_leaves_);
        DevFarLeafGeom* d_geo = upload(geo);
        pat_ = alloc<double2>(static_cast<size_t>(plan.pat_elems) * 2);
        traffic_.s2m = plan.pat_elems * 32.0 + n_ * 16.0;
        traffic_.l2t = plan.pat_elems * 32.0 + n_ * 16.0;

        DevSources S{};
        S.kind = plan.kind;
        S.k = plan.pw.wavenum;
        if (plan.kind == kDipole) {
            S.pos = upload(plan.dip_pos);
            S.phat = upload(plan.dip_phat);
        } else {
            S.rwg = upload(plan.rwg);
            S.tris = upload(plan.tris);
            S.tri_quad = upload(plan.tri_quad);
            S.quad_w = upload(plan.quad_w);
            S.nq = plan.nq;
        }
        if (n_leaves_ > 0 && plan.kind == kRwg && plan.cfg.ref_compat) {
            // Reference-compatible RWG patterns: the closed-form integral is
            // ill-conditioned near alpha, beta, gamma = 0, so it is evaluated on
            // the host with the reference's exact rounding and uploaded.
            std::vector<cplx> hp;
            plan.rwg_patterns_host(hp);
            MLFMA_CK(cudaMemcpy(pat_, hp.data(), hp.size() * sizeof(cplx), cudaMemcpyHostToDevice));
        } else if (n_leaves_ > 0) {
            k_patterns<<<n_leaves_, 256, 0, stream_>>>(lv_dev_, leaves_, d_geo, S, pat_);
            MLFMA_CK(cudaGetLastError());
        }

        // ---- near field
        std::vector<DevNearBlock> nb;
        for (const NearBlock& b : plan.near_blocks)
            nb.push_back(DevNearBlock{b.row0, b.nrow, b.col0, b.ncol, b.off, b.self, 0});
        n_near_blocks_ = static_cast<int>(nb.size());
        near_blocks_ = upload(nb);
        near_entries_ = plan.near_entries;
        near_z_ = alloc<double2>(static_cast<size_t>(near_entries_));
        if (near_entries_ > 0) {
            k_near_assemble<<<blocks_for(near_entries_, 128), 128, 0, stream_>>>(
                near_blocks_, n_near_blocks_, near_entries_, S, near_z_);
            MLFMA_CK(cudaGetLastError());
        }
        traffic_.near = near_entries_ * 16.0 + n_ * 16.0 * 2.0;
        traffic_.total = traffic_.s2m + traffic_.m2m + traffic_.m2l + traffic_.l2l + traffic_.l2t + traffic_.near;

        // Shared-memory limits for the interpolation kernels.
        size_t m2m_smem = 0, l2l_smem = 0;
        for (int p = plan.lmin; p < plan.max_level; ++p) {
            const Level& Lp = plan.levels[p];
            const Level& Lc = plan.levels[p + 1];
            const int rows = m2m_rows(Lp.nth, Lp.nph);
            m2m_smem = std::max(m2m_smem, static_cast<size_t>(rows) * Lc.nph * 2 * sizeof(double2));
            l2l_smem = std::max(l2l_smem, static_cast<size_t>(Lp.nth) * Lc.nph * 2 * sizeof(double2));
        }
        int dev_smem = 0;
        MLFMA_CK(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
        if (m2m_smem > static_cast<size_t>(dev_smem) || l2l_smem > static_cast<size_t>(dev_smem))
            return "angular grid too large for the interpolation kernels' shared memory";
        MLFMA_CK(cudaFuncSetAttribute(k_m2m<kM2MOut>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(std::max<size_t>(m2m_smem, 1))));
        MLFMA_CK(cudaFuncSetAttribute(k_l2l, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(std::max<size_t>(l2l_smem, 1))));
        MLFMA_CK(cudaStreamSynchronize(stream_));
        MLFMA_CK(cudaGetLastError());
        ready_ = true;
        return {};
    } catch (const std::exception& e) {
        return e.what();
    }
}

int DeviceOp::launches_per_matvec() const {
    int n = 2;  // gather + finish
    if (n_leaves_) {
        n += 2;  // S2M + L2T
        for (int p = lv_.lmin; p < lv_.lmax; ++p)
            if (trans_[p].npar) n += 2;  // M2M + L2L
        for (int l = lv_.lmin; l <= lv_.lmax; ++l)
            if (m2l_nbox_[l]) n += 1;
    }
    if (n_near_blocks_) n += 1;
    return n;
}

int DeviceOp::m2m_rows(int nth, int nph) {
    const int rows = (kM2MThreads * kM2MOut) / std::max(nph, 1);
    return std::max(1, std::min(nth, rows));
}

void DeviceOp::run_far(const double2* xt, cudaStream_t s) {
    if (n_leaves_ == 0) return;
    k_s2m<<<n_leaves_, 128, 0, s>>>(lv_dev_, leaves_, pat_, xt);
    for (int p = lv_.lmax - 1; p >= lv_.lmin; --p) {
        const DevTrans& T = trans_[p];
        if (T.npar == 0) continue;
        const DevLevel& P = lv_.lv[p];
        const DevLevel& C = lv_.lv[p + 1];
        const int rows = m2m_rows(P.nth, P.nph);
        const dim3 grid(T.npar, (P.nth + rows - 1) / rows);
        const size_t smem = static_cast<size_t>(rows) * C.nph * 2 * sizeof(double2);
        k_m2m<kM2MOut><<<grid, kM2MThreads, smem, s>>>(lv_dev_, T, rows);
    }
    for (int l = lv_.lmin; l <= lv_.lmax; ++l) {
        if (m2l_nbox_[l] == 0) continue;
        const int bs = std::min(512, ((lv_.lv[l].ndir + 31) / 32) * 32);
        k_m2l<<<m2l_nbox_[l], bs, 0, s>>>(lv_dev_, l, m2l_boxes_[l], lv_.ref_compat ? 0 : 1);
    }
    for (int p = lv_.lmin; p < lv_.lmax; ++p) {
        const DevTrans& T = trans_[p];
        if (T.npar == 0) continue;
        const DevLevel& P = lv_.lv[p];
        const DevLevel& C = lv_.lv[p + 1];
        const size_t smem = static_cast<size_t>(P.nth) * C.nph * 2 * sizeof(double2);
        k_l2l<<<T.npar, 256, smem, s>>>(lv_dev_, T, lv_.ref_compat);
    }
    k_l2t<<<n_leaves_, 128, 0, s>>>(lv_dev_, leaves_, pat_, yfar_);
}

void DeviceOp::run_near(const double2* xt, cudaStream_t s) {
    if (n_near_blocks_ == 0) return;
    k_near<<<n_near_blocks_, kNearWarps * 32, 0, s>>>(near_blocks_, near_z_, xt, ynear_);
}

void DeviceOp::apply_tree(const double2* xt, double2* yt, cudaStream_t s) {
    cudaMemsetAsync(yfar_, 0, sizeof(double2) * n_, s);
    cudaMemsetAsync(ynear_, 0, sizeof(double2) * n_, s);
    cudaEventRecord(ev_fork_, s);
    cudaStreamWaitEvent(side_, ev_fork_, 0);
    run_near(xt, side_);
    cudaEventRecord(ev_join_, side_);
    run_far(xt, s);
    cudaStreamWaitEvent(s, ev_join_, 0);
    k_finish<<<blocks_for(n_, 256), 256, 0, s>>>(yfar_, ynear_, nullptr, yt, n_, ck_, 0);
}

std::string DeviceOp::matvec_device(const double2* x, double2* y, bool accumulate, cudaStream_t stream) {
    if (!ready_) return "operator not set up";
    cudaStream_t s = stream ? stream : stream_;
    MLFMA_CK(cudaSetDevice(device_));
    k_gather<<<blocks_for(n_, 256), 256, 0, s>>>(x, perm_, xt_, n_);
    cudaMemsetAsync(yfar_, 0, sizeof(double2) * n_, s);
    cudaMemsetAsync(ynear_, 0, sizeof(double2) * n_, s);
    cudaEventRecord(ev_fork_, s);
    cudaStreamWaitEvent(side_, ev_fork_, 0);
    run_near(xt_, side_);
    cudaEventRecord(ev_join_, side_);
    run_far(xt_, s);
    cudaStreamWaitEvent(s, ev_join_, 0);
    k_finish<<<blocks_for(n_, 256), 256, 0, s>>>(yfar_, ynear_, perm_, y, n_, ck_, accumulate ? 1 : 0);
    MLFMA_CK(cudaGetLastError());
    return {};
}

std::string DeviceOp::time_stages(StageTimes* out) {
    if (!ready_) return "operator not set up";
    MLFMA_CK(cudaSetDevice(device_));
    cudaEvent_t ev[9];
    for (auto& e : ev) MLFMA_CK(cudaEventCreate(&e));
    cudaStream_t s = stream_;
    cudaEventRecord(ev[0], s);
    cudaMemsetAsync(yfar_, 0, sizeof(double2) * n_, s);
    cudaMemsetAsync(ynear_, 0, sizeof(double2) * n_, s);
    cudaEventRecord(ev[1], s);
    if (n_leaves_) k_s2m<<<n_leaves_, 128, 0, s>>>(lv_dev_, leaves_, pat_, xt_);
    cudaEventRecord(ev[2], s);
    for (int p = lv_.lmax - 1; p >= lv_.lmin; --p) {
        const DevTrans& T = trans_[p];
        if (T.npar == 0) continue;
        const int rows = m2m_rows(lv_.lv[p].nth, lv_.lv[p].nph);
        const dim3 grid(T.npar, (lv_.lv[p].nth + rows - 1) / rows);
        k_m2m<kM2MOut><<<grid, kM2MThreads, static_cast<size_t>(rows) * lv_.lv[p + 1].nph * 32, s>>>(lv_dev_, T, rows);
    }
    cudaEventRecord(ev[3], s);
    for (int l = lv_.lmin; l <= lv_.lmax; ++l) {
        if (m2l_nbox_[l] == 0) continue;
        const int bs = std::min(512, ((lv_.lv[l].ndir + 31) / 32) * 32);
        k_m2l<<<m2l_nbox_[l], bs, 0, s>>>(lv_dev_, l, m2l_boxes_[l], lv_.ref_compat ? 0 : 1);
    }
    cudaEventRecord(ev[4], s);
    for (int p = lv_.lmin; p < lv_.lmax; ++p) {
        const DevTrans& T = trans_[p];
        if (T.npar == 0) continue;
        k_l2l<<<T.npar, 256, static_cast<size_t>(lv_.lv[p].nth) * lv_.lv[p + 1].nph * 32, s>>>(lv_dev_, T, lv_.ref_compat);
    }
    cudaEventRecord(ev[5], s);
    if (n_leaves_) k_l2t<<<n_leaves_, 128, 0, s>>>(lv_dev_, leaves_, pat_, yfar_);
    cudaEventRecord(ev[6], s);
    run_near(xt_, s);
    cudaEventRecord(ev[7], s);
    k_finish<<<blocks_for(n_, 256), 256, 0, s>>>(yfar_, ynear_, nullptr, yt_, n_, ck_, 0);
    cudaEventRecord(ev[8], s);
    MLFMA_CK(cudaEventSynchronize(ev[8]));
    float t[8];
    for (int i = 0; i < 8; ++i) cudaEventElapsedTime(&t[i], ev[i], ev[i + 1]);
    out->gather = t[0];
    out->s2m = t[1];
    out->m2m = t[2];
    out->m2l = t[3];
    out->l2l = t[4];
    out->l2t = t[5];
    out->near = t[6];
    out->finish = t[7];
    cudaEventElapsedTime(&out->total, ev[0], ev[8]);
    for (auto& e : ev) cudaEventDestroy(e);
    MLFMA_CK(cudaGetLastError());
    return {};
}

std::string DeviceOp::copy_level(int level, int which, double2* host, long long count) {
    if (level < lv_.lmin || level > lv_.lmax) return "level out of range";
    const DevLevel& d = lv_.lv[level];
    const long long cnt = static_cast<long long>(d.nbox) * d.ndir * 2;
    if (count < cnt) return "buffer too small";
    MLFMA_CK(cudaSetDevice(device_));
    MLFMA_CK(cudaStreamSynchronize(stream_));
    MLFMA_CK(cudaMemcpy(host, which ? d.B : d.A, cnt * sizeof(double2), cudaMemcpyDeviceToHost));
    return {};
}

}  // namespace mlfma
