// Far-field kernels of the MLFMA matvec: aggregation (S2M), interpolation
// (M2M), translation (M2L), anterpolation (L2L) and disaggregation (L2T).
// Templated on the real type R of the far field (double: FP64 path; float:
// mixed path, complex float storage with float accumulation).  Included once,
// by kernels.cu.
//
// Layout: per level, patterns are [box][direction][2 components] complex;
// element e = 2*direction + component runs contiguously, so a box's
// pattern is one contiguous run of 2*ndir values.
#pragma once

#include "device.cuh"
#include "zmath.cuh"
#include "bulk_copy.cuh"

namespace mlfma {
namespace {

// Programmatic dependent launch.  The far-field chain's kernels after the first
// are launched with programmatic stream serialization, so that a kernel's
// blocks are scheduled while its predecessor on the stream is still draining
// its last wave.  Every chain kernel therefore starts with griddepcontrol.wait,
// which returns once the predecessor grid has completed and its writes are
// visible (a no-op for a kernel launched without the attribute): nothing a
// predecessor writes is read, and nothing it reads is overwritten, before it.
// Only then does the kernel let its own successor launch, so at most one
// kernel's blocks wait ahead of the running one.
__device__ __forceinline__ void chain_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ------------------------------------------------------------ S2M
// a_B[e] = sum_n x_n R_n[e]  (Leaf::buildMpoleCoeffs, src/fmm/leaf.cpp:212-230).
// One block per work item (leaf, run of at most kS2MThreads elements), all leaf
// levels in one launch; one thread per element e (direction, component), so
// every pattern row is read once with coalesced loads; eight sources are in
// flight per thread.
constexpr int kS2MThreads = 352;
constexpr int kL2TThreads = 256;
constexpr int kL2TSrcPerBlock = kL2TThreads / 32;

// CJ: conjugated patterns, a_B[e] = sum_n x_n conj(R_n[e]) -- the transpose of
// L2T, first stage of the transposed product.
template <class R, bool CJ>
__global__ void __launch_bounds__(kS2MThreads)
k_s2m(const DevLevelT<R>* __restrict__ lvs, const int4* __restrict__ items, const DevFarLeaf* __restrict__ leaves,
      const typename Cx<R>::T* __restrict__ pat, const double2* __restrict__ x) {
    chain_wait();
    using C = typename Cx<R>::T;
    extern __shared__ unsigned char smraw[];
    C* xs = reinterpret_cast<C*>(smraw);
    const int4 it = items[blockIdx.x];  // leaf, first element, element count
    const DevFarLeaf lf = leaves[it.x];
    const int ne = 2 * lvs[lf.level].ndir;
    C* A = lvs[lf.level].A + static_cast<size_t>(lf.box) * ne;
    for (int i = threadIdx.x; i < lf.nsrc; i += blockDim.x) xs[i] = from_d2<C>(x[lf.src0 + i]);
    __syncthreads();
    if (static_cast<int>(threadIdx.x) >= it.z) return;
    const int e = it.y + threadIdx.x;
    const C* r = pat + lf.pat_off * 2 + e;
    C a0 = zero<C>(), a1 = zero<C>(), a2 = zero<C>(), a3 = zero<C>();
    int s = 0;
    for (; s + 8 <= lf.nsrc; s += 8) {
        C v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = ldg_stream(r + static_cast<size_t>(s + u) * ne);
        if (CJ) {
            a0 = cjfma(v[0], xs[s], a0);
            a1 = cjfma(v[1], xs[s + 1], a1);
            a2 = cjfma(v[2], xs[s + 2], a2);
            a3 = cjfma(v[3], xs[s + 3], a3);
            a0 = cjfma(v[4], xs[s + 4], a0);
            a1 = cjfma(v[5], xs[s + 5], a1);
            a2 = cjfma(v[6], xs[s + 6], a2);
            a3 = cjfma(v[7], xs[s + 7], a3);
        } else {
            a0 = cfma(xs[s], v[0], a0);
            a1 = cfma(xs[s + 1], v[1], a1);
            a2 = cfma(xs[s + 2], v[2], a2);
            a3 = cfma(xs[s + 3], v[3], a3);
            a0 = cfma(xs[s + 4], v[4], a0);
            a1 = cfma(xs[s + 5], v[5], a1);
            a2 = cfma(xs[s + 6], v[6], a2);
            a3 = cfma(xs[s + 7], v[7], a3);
        }
    }
    if (s < lf.nsrc) {  // the last sources: their loads in flight together
        C v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u)
            v[u] = s + u < lf.nsrc ? ldg_stream(r + static_cast<size_t>(s + u) * ne) : zero<C>();
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (s + u >= lf.nsrc) break;
            C& acc = (u & 3) == 0 ? a0 : (u & 3) == 1 ? a1 : (u & 3) == 2 ? a2 : a3;
            acc = CJ ? cjfma(v[u], xs[s + u], acc) : cfma(xs[s + u], v[u], acc);
        }
    }
    A[e] = cadd(cadd(a0, a1), cadd(a2, a3));
}

// ------------------------------------------------------------ L2T
// y_m = sum_e conj(R_m[e]) b_B[e]  (Leaf::evalFarSols, src/fmm/leaf.cpp:257-280;
// C k is applied when the result is written out).  One block per work item
// (leaf, run of up to eight sources), one warp per source, eight loads in
// flight per lane; the sum is widened to complex double on output.
// CJ = false: plain patterns, y_m = sum_e R_m[e] b_B[e] -- the transpose of S2M,
// last stage of the transposed product.
template <class R, bool CJ>
__global__ void __launch_bounds__(kL2TThreads)
k_l2t(const DevLevelT<R>* __restrict__ lvs, const int4* __restrict__ items, const DevFarLeaf* __restrict__ leaves,
      const typename Cx<R>::T* __restrict__ pat, double2* __restrict__ yfar) {
    chain_wait();
    using C = typename Cx<R>::T;
    const int4 it = items[blockIdx.x];  // leaf, first source, source count
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp >= it.z) return;
    const DevFarLeaf lf = leaves[it.x];
    const int ndir = lvs[lf.level].ndir, ne = 2 * ndir;
    const C* Bb = lvs[lf.level].B + static_cast<size_t>(lf.box) * ne;
    const int s = it.y + warp;
    const C* r = pat + (lf.pat_off + static_cast<long long>(s) * ndir) * 2;
    C a0 = zero<C>(), a1 = zero<C>(), a2 = zero<C>(), a3 = zero<C>();
    // eight loads in flight per lane, the last run of the row predicated (a
    // leaf-level row of 162-324 elements is one or two runs)
    for (int e = lane; e < ne; e += 256) {
        C v[8], bv[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const bool in = e + 32 * u < ne;
            v[u] = in ? ldg_stream(r + e + 32 * u) : zero<C>();
            bv[u] = in ? Bb[e + 32 * u] : zero<C>();
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            C& acc = (u & 3) == 0 ? a0 : (u & 3) == 1 ? a1 : (u & 3) == 2 ? a2 : a3;
            acc = CJ ? cjfma(v[u], bv[u], acc) : cfma(v[u], bv[u], acc);
        }
    }
    const C acc = warp_sum(cadd(cadd(a0, a1), cadd(a2, a3)));
    if (lane == 0) yfar[lf.src0 + s] = to_d2(acc);
}

// Half patterns (the complex-float far field of the mixed operator): patterns
// are kept for the first half of the directions only (d < ndir/2,
// `hpat`: per source, ndir elements (direction, component)).  The direction
// grid is symmetric under k -> -k (Gauss-Legendre theta rows in mirror pairs,
// an even number of phi columns), and for a real basis function
// R(-k) = conj(R(k)) as a vector; theta-hat is the same at -k and phi-hat flips,
// so the antipodal element anti[e] holds sgn(e) conj(R[e]), sgn = +1 for the
// theta component and -1 for the phi component.  S2M and L2T read each stored
// value once and use it for both directions: half the pattern bytes.  The
// closed-form RWG integrals are ill-conditioned enough that the derived
// antipodal values differ from directly computed ones by about 1e-8 relative:
// far below complex-float rounding, but above the 1e-10 agreement the FP64
// operator keeps with the reference, so the FP64 far field stores every
// direction and uses k_s2m / k_l2t.
// hpat from the full patterns: the first ndir elements of every source.
template <class R>
__global__ void k_half_patterns(const DevLevelT<R>* __restrict__ lvs, const DevFarLeaf* __restrict__ leaves,
                                const double2* __restrict__ pat, typename Cx<R>::T* __restrict__ hpat) {
    using C = typename Cx<R>::T;
    const DevFarLeaf lf = leaves[blockIdx.x];
    const int ne = lvs[lf.level].ndir;
    for (int i = threadIdx.x; i < lf.nsrc * ne; i += blockDim.x) {
        const int s = i / ne, e = i - s * ne;
        hpat[lf.pat_off + static_cast<long long>(s) * ne + e] =
            from_d2<C>(pat[(lf.pat_off + static_cast<long long>(s) * ne) * 2 + e]);
    }
}

// ------------------------------------------------------------ S2M, half patterns
// a_B[e] = sum_n x_n R_n[e]  (Leaf::buildMpoleCoeffs, src/fmm/leaf.cpp:212-230).
// One block per work item (leaf, run of at most kS2MThreads elements of the
// first half), all leaf levels in one launch; one thread per element e, which
// also forms the antipodal element a_B[anti[e]] = sgn sum_n x_n conj(R_n[e]);
// every stored pattern row is read once with coalesced loads; eight sources
// are in flight per thread.
// CJ: conjugated patterns, a_B[e] = sum_n x_n conj(R_n[e]) -- the transpose of
// L2T, first stage of the transposed product.
template <class R, bool CJ>
__global__ void __launch_bounds__(kS2MThreads)
k_s2m_half(const DevLevelT<R>* __restrict__ lvs, const int4* __restrict__ items, const DevFarLeaf* __restrict__ leaves,
      const typename Cx<R>::T* __restrict__ hpat, const double2* __restrict__ x) {
    chain_wait();
    using C = typename Cx<R>::T;
    extern __shared__ unsigned char smraw[];
    C* xs = reinterpret_cast<C*>(smraw);
    const int4 it = items[blockIdx.x];  // leaf, first element, element count
    const DevFarLeaf lf = leaves[it.x];
    const DevLevelT<R> lv = lvs[lf.level];
    const int ne = lv.ndir;  // stored elements per source
    C* A = lv.A + static_cast<size_t>(lf.box) * 2 * ne;
    for (int i = threadIdx.x; i < lf.nsrc; i += blockDim.x) xs[i] = from_d2<C>(x[lf.src0 + i]);
    __syncthreads();
    if (static_cast<int>(threadIdx.x) >= it.z) return;
    const int e = it.y + threadIdx.x;
    const C* r = hpat + lf.pat_off + e;
    // a: this element, b: sum of x conj(v) (or x v), the antipodal one up to its sign
    C a0 = zero<C>(), a1 = zero<C>(), a2 = zero<C>(), a3 = zero<C>();
    C b0 = zero<C>(), b1 = zero<C>(), b2 = zero<C>(), b3 = zero<C>();
    int s = 0;
    for (; s + 8 <= lf.nsrc; s += 8) {
        C v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = ldg_stream(r + static_cast<size_t>(s + u) * ne);
#pragma unroll
        for (int u = 0; u < 8; u += 4) {
            if (CJ) {
                a0 = cjfma(v[u], xs[s + u], a0);
                a1 = cjfma(v[u + 1], xs[s + u + 1], a1);
                a2 = cjfma(v[u + 2], xs[s + u + 2], a2);
                a3 = cjfma(v[u + 3], xs[s + u + 3], a3);
                b0 = cfma(xs[s + u], v[u], b0);
                b1 = cfma(xs[s + u + 1], v[u + 1], b1);
                b2 = cfma(xs[s + u + 2], v[u + 2], b2);
                b3 = cfma(xs[s + u + 3], v[u + 3], b3);
            } else {
                a0 = cfma(xs[s + u], v[u], a0);
                a1 = cfma(xs[s + u + 1], v[u + 1], a1);
                a2 = cfma(xs[s + u + 2], v[u + 2], a2);
                a3 = cfma(xs[s + u + 3], v[u + 3], a3);
                b0 = cjfma(v[u], xs[s + u], b0);
                b1 = cjfma(v[u + 1], xs[s + u + 1], b1);
                b2 = cjfma(v[u + 2], xs[s + u + 2], b2);
                b3 = cjfma(v[u + 3], xs[s + u + 3], b3);
            }
        }
    }
    if (s < lf.nsrc) {  // the last sources: their loads in flight together
        C v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u)
            v[u] = s + u < lf.nsrc ? ldg_stream(r + static_cast<size_t>(s + u) * ne) : zero<C>();
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (s + u >= lf.nsrc) break;
            C& a = (u & 3) == 0 ? a0 : (u & 3) == 1 ? a1 : (u & 3) == 2 ? a2 : a3;
            C& b = (u & 3) == 0 ? b0 : (u & 3) == 1 ? b1 : (u & 3) == 2 ? b2 : b3;
            a = CJ ? cjfma(v[u], xs[s + u], a) : cfma(xs[s + u], v[u], a);
            b = CJ ? cfma(xs[s + u], v[u], b) : cjfma(v[u], xs[s + u], b);
        }
    }
    A[e] = cadd(cadd(a0, a1), cadd(a2, a3));
    const C b = cadd(cadd(b0, b1), cadd(b2, b3));
    A[lv.anti[e]] = (e & 1) ? C{-b.x, -b.y} : b;
}

// ------------------------------------------------------------ L2T, half patterns
// y_m = sum_e conj(R_m[e]) b_B[e] over the stored half:
// y_m = sum_{e < ndir} conj(R_m[e]) b_B[e] + R_m[e] b'_B[e], b'_B[e] =
// sgn(e) b_B[anti[e]].  One block per work item (leaf, run of up to eight
// sources): the block first stages b_B and b'_B in shared memory, then one warp
// per source streams its stored patterns (eight loads in flight per lane).
// CJ = false: plain patterns (the transpose of S2M).
template <class R, bool CJ>
__global__ void __launch_bounds__(kL2TThreads)
k_l2t_half(const DevLevelT<R>* __restrict__ lvs, const int4* __restrict__ items, const DevFarLeaf* __restrict__ leaves,
           const typename Cx<R>::T* __restrict__ hpat, double2* __restrict__ yfar) {
    chain_wait();
    using C = typename Cx<R>::T;
    extern __shared__ unsigned char smraw[];
    const int4 it = items[blockIdx.x];  // leaf, first source, source count
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const DevFarLeaf lf = leaves[it.x];
    const DevLevelT<R> lv = lvs[lf.level];
    const int ne = lv.ndir;  // stored elements per source
    C* bs = reinterpret_cast<C*>(smraw);
    C* bp = bs + ne;
    {
        const C* Bb = lv.B + static_cast<size_t>(lf.box) * 2 * ne;
        for (int e = threadIdx.x; e < ne; e += blockDim.x) {
            bs[e] = Bb[e];
            const C q = Bb[lv.anti[e]];
            bp[e] = (e & 1) ? C{-q.x, -q.y} : q;
        }
    }
    __syncthreads();
    if (warp >= it.z) return;
    const int s = it.y + warp;
    const C* r = hpat + lf.pat_off + static_cast<long long>(s) * ne;
    C a0 = zero<C>(), a1 = zero<C>(), a2 = zero<C>(), a3 = zero<C>();
    // eight loads in flight per lane, the last run of the row predicated
    for (int e = lane; e < ne; e += 256) {
        C v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = e + 32 * u < ne ? ldg_stream(r + e + 32 * u) : zero<C>();
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int ee = e + 32 * u;
            if (ee >= ne) continue;
            C& acc = (u & 3) == 0 ? a0 : (u & 3) == 1 ? a1 : (u & 3) == 2 ? a2 : a3;
            if (CJ) {
                acc = cjfma(v[u], bs[ee], acc);
                acc = cfma(v[u], bp[ee], acc);
            } else {
                acc = cfma(v[u], bs[ee], acc);
                acc = cjfma(v[u], bp[ee], acc);
            }
        }
    }
    const C acc = warp_sum(cadd(cadd(a0, a1), cadd(a2, a3)));
    if (lane == 0) yfar[lf.src0 + s] = to_d2(acc);
}

// ------------------------------------------------------------ M2M
// Parent outgoing pattern = sum over non-empty children of Interp[shift(child)]:
// shift on the child grid, theta pass with pole reflection, periodic phi pass
// (Stem::buildMpoleCoeffs and addInterpCoeffs, src/fmm/stem.cpp:72-184).
// Block = (parent, tile of `rows` parent theta rows).  Phase 1 computes the
// theta pass of every child into shared memory at once (all loads
// independent); phase 2 forms each parent output from the children's rows.
// POST: the transposed L2L -- no shift before the theta pass; each child's
// interpolated pattern is multiplied by the parent-grid shift of its octant
// (shift_down of the parent level) before the sum over children.
template <class R, int W, bool POST>  // taps per row: 2 * interp_order (both passes)
__global__ void __launch_bounds__(128)
k_m2m(const DevLevelT<R>* __restrict__ lvs, DevTransT<R> T, int rows) {
    chain_wait();
    using C = typename Cx<R>::T;
    extern __shared__ unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int par = blockIdx.x;
    const DevLevelT<R> P = lvs[T.plevel];
    const DevLevelT<R> Cl = lvs[T.plevel + 1];
    const int nph = P.nph, mph = Cl.nph, halfm = Cl.nph / 2;
    const int r0 = blockIdx.y * rows;
    const int nrow = min(P.nth, r0 + rows) - r0;
    if (nrow <= 0) return;
    const int c0 = T.child_ptr[par], nch = T.child_ptr[par + 1] - c0;
    const int per_child = nrow * mph;
    for (int it = threadIdx.x; it < nch * per_child; it += blockDim.x) {
        const int c = it / per_child, e = it - c * per_child;
        const int jr = e / mph, iph = e - jr * mph;
        const int jth = r0 + jr;
        const C* Ac = Cl.A + static_cast<size_t>(T.child_box[c0 + c]) * Cl.ndir * 2;
        const C* sh = Cl.shift_up + static_cast<size_t>(T.child_oct[c0 + c]) * Cl.ndir;
        C v0 = zero<C>(), v1 = zero<C>();
#pragma unroll
        for (int k = 0; k < W; ++k) {
            const int q = jth * W + k;
            const bool rf = T.up_th.refl[q];
            const int sp = rf ? (iph < halfm ? iph + halfm : iph - halfm) : iph;
            const R cf = T.up_th.coef[q];
            const int d = T.up_th.src[q] * mph + sp;
            if (POST) {
                v0 = crfma(cf, Ac[2 * d], v0);
                v1 = crfma(cf, Ac[2 * d + 1], v1);
            } else {
                const C ph = sh[d];
                v0 = crfma(cf, cmul(ph, Ac[2 * d]), v0);
                v1 = crfma(cf, cmul(ph, Ac[2 * d + 1]), v1);
            }
        }
        sm[2 * it] = v0;
        sm[2 * it + 1] = v1;
    }
    __syncthreads();
    C* Ap = P.A + (static_cast<size_t>(T.par_box[par]) * P.ndir + static_cast<size_t>(r0) * nph) * 2;
    for (int o = threadIdx.x; o < nrow * nph; o += blockDim.x) {
        const int jr = o / nph, jph = o - jr * nph;
        C a0 = zero<C>(), a1 = zero<C>();
        for (int c = 0; c < nch; ++c) {
            const C* row = sm + (static_cast<size_t>(c) * per_child + static_cast<size_t>(jr) * mph) * 2;
            if (POST) {
                C t0 = zero<C>(), t1 = zero<C>();
#pragma unroll
                for (int k = 0; k < W; ++k) {
                    const int q = k * nph + jph;  // tap-major
                    const int s = T.up_ph.src_t[q];
                    const R cf = T.up_ph.coef_t[q];
                    t0 = crfma(cf, row[2 * s], t0);
                    t1 = crfma(cf, row[2 * s + 1], t1);
                }
                const C ph = P.shift_down[static_cast<size_t>(T.child_oct[c0 + c]) * P.ndir + (r0 + jr) * nph + jph];
                a0 = cfma(ph, t0, a0);
                a1 = cfma(ph, t1, a1);
            } else {
#pragma unroll
                for (int k = 0; k < W; ++k) {
                    const int q = k * nph + jph;  // tap-major
                    const int s = T.up_ph.src_t[q];
                    const R cf = T.up_ph.coef_t[q];
                    a0 = crfma(cf, row[2 * s], a0);
                    a1 = crfma(cf, row[2 * s + 1], a1);
                }
            }
        }
        Ap[2 * o] = a0;
        Ap[2 * o + 1] = a1;
    }
}

// ------------------------------------------------------------ M2L
// b_B = w_theta (2 pi / nph) sum_{S in list 2} T[c_B - c_S] a_S
// (Node::buildMpoleToLocalCoeffs, src/fmm/node.cpp:105-134).  One block per
// (level, box, direction chunk) item, all levels in one launch; four list
// entries in flight per thread.
// TR: the transposed translation, T(c_S - c_B) in place of T(c_B - c_S): the
// negated offset, id 315 - id in the order of Math::getINodeDistVecs (the
// offset set is symmetric and listed lexicographically).  Lists 2 are
// symmetric, so the same lists serve.
template <class R, bool TR>
__global__ void __launch_bounds__(128)
k_m2l(const DevLevelT<R>* __restrict__ lvs, const int4* __restrict__ items, int zero_empty) {
    chain_wait();
    using C = typename Cx<R>::T;
    const int4 it = items[blockIdx.x];  // level, box, first direction, count
    if (static_cast<int>(threadIdx.x) >= it.w) return;
    const DevLevelT<R> lv = lvs[it.x];
    const int b = it.y, d = it.z + threadIdx.x, ndir = lv.ndir;
    const int p0 = lv.m2l_ptr[b], p1 = lv.m2l_ptr[b + 1];
    C* Bo = lv.B + (static_cast<size_t>(b) * ndir + d) * 2;
    if (p0 == p1) {
        if (zero_empty) { Bo[0] = zero<C>(); Bo[1] = zero<C>(); }
        return;
    }
    C a0 = zero<C>(), a1 = zero<C>(), c0 = zero<C>(), c1 = zero<C>();
    int p = p0;
    for (; p + 4 <= p1; p += 4) {
        int sb[4], ob[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            sb[u] = lv.m2l_src[p + u];
            ob[u] = TR ? 315 - lv.m2l_off[p + u] : lv.m2l_off[p + u];
        }
        C t[4], xa[4], xb[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            t[u] = lv.transl[static_cast<size_t>(ob[u]) * ndir + d];
            const C* As = lv.A + (static_cast<size_t>(sb[u]) * ndir + d) * 2;
            xa[u] = As[0];
            xb[u] = As[1];
        }
        a0 = cfma(t[0], xa[0], a0);
        a1 = cfma(t[0], xb[0], a1);
        c0 = cfma(t[1], xa[1], c0);
        c1 = cfma(t[1], xb[1], c1);
        a0 = cfma(t[2], xa[2], a0);
        a1 = cfma(t[2], xb[2], a1);
        c0 = cfma(t[3], xa[3], c0);
        c1 = cfma(t[3], xb[3], c1);
    }
    for (; p < p1; ++p) {
        const int s0 = lv.m2l_src[p], o0 = TR ? 315 - lv.m2l_off[p] : lv.m2l_off[p];
        const C t0 = lv.transl[static_cast<size_t>(o0) * ndir + d];
        const C* A0 = lv.A + (static_cast<size_t>(s0) * ndir + d) * 2;
        a0 = cfma(t0, A0[0], a0);
        a1 = cfma(t0, A0[1], a1);
    }
    const R w = lv.w[d];
    Bo[0] = cscale(w, cadd(a0, c0));
    Bo[1] = cscale(w, cadd(a1, c1));
}

// The same translation with the box's list 2 (source boxes, offset ids)
// staged in shared memory first, so the inner loop's loads of patterns and
// transfer values depend on nothing but shared memory and U of them are in
// flight at once.
constexpr int kM2LStage = 256;  // list entries staged per round (list 2 holds at most 189)

template <class R, bool TR>
__global__ void __launch_bounds__(128)
k_m2l_staged(const DevLevelT<R>* __restrict__ lvs, const int4* __restrict__ items, int zero_empty) {
    chain_wait();
    using C = typename Cx<R>::T;
    constexpr int U = sizeof(R) == 4 ? 8 : 6;
    __shared__ int s_src[kM2LStage], s_off[kM2LStage];
    const int4 it = items[blockIdx.x];  // level, box, first direction, count
    const DevLevelT<R> lv = lvs[it.x];
    const int b = it.y, ndir = lv.ndir;
    const bool live = static_cast<int>(threadIdx.x) < it.w;
    const int d = it.z + (live ? threadIdx.x : 0);
    const int p0 = lv.m2l_ptr[b], p1 = lv.m2l_ptr[b + 1];
    C* Bo = lv.B + (static_cast<size_t>(b) * ndir + d) * 2;
    if (p0 == p1) {
        if (zero_empty && live) { Bo[0] = zero<C>(); Bo[1] = zero<C>(); }
        return;
    }
    C a0 = zero<C>(), a1 = zero<C>(), c0 = zero<C>(), c1 = zero<C>();
    for (int base = p0; base < p1; base += kM2LStage) {
        const int cnt = min(kM2LStage, p1 - base);
        __syncthreads();
        for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
            s_src[i] = lv.m2l_src[base + i];
            const int o = lv.m2l_off[base + i];
            s_off[i] = TR ? 315 - o : o;
        }
        __syncthreads();
        if (!live) continue;
        int p = 0;
        for (; p + U <= cnt; p += U) {
            C t[U], xa[U], xb[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                t[u] = lv.transl[static_cast<size_t>(s_off[p + u]) * ndir + d];
                const C* As = lv.A + (static_cast<size_t>(s_src[p + u]) * ndir + d) * 2;
                xa[u] = As[0];
                xb[u] = As[1];
            }
#pragma unroll
            for (int u = 0; u < U; u += 2) {
                a0 = cfma(t[u], xa[u], a0);
                a1 = cfma(t[u], xb[u], a1);
                c0 = cfma(t[u + 1], xa[u + 1], c0);
                c1 = cfma(t[u + 1], xb[u + 1], c1);
            }
        }
        for (; p < cnt; ++p) {
            const C t0 = lv.transl[static_cast<size_t>(s_off[p]) * ndir + d];
            const C* A0 = lv.A + (static_cast<size_t>(s_src[p]) * ndir + d) * 2;
            a0 = cfma(t0, A0[0], a0);
            a1 = cfma(t0, A0[1], a1);
        }
    }
    if (!live) return;
    const R w = lv.w[d];
    Bo[0] = cscale(w, cadd(a0, c0));
    Bo[1] = cscale(w, cadd(a1, c1));
}

// ------------------------------------------------------------ L2L
// child local += Anterp[shift(parent local)]: shift on the parent grid, then
// the transposed phi pass, then the transposed theta pass with pole
// reflection (Stem::getShiftedLocalCoeffs and addAnterpCoeffs,
// src/fmm/stem.cpp:109-244).  One block per (parent, child) pair; the
// pair list already omits parents that pass nothing down.
// POST: the transposed M2M -- no shift before the phi pass; the anterpolated
// pattern is multiplied by the child-grid shift of the child's octant
// (shift_up of the child level) as it is added to the child.
template <class R, int W, bool POST>  // both transposed stencils padded to W taps per row
__global__ void __launch_bounds__(256)
k_l2l(const DevLevelT<R>* __restrict__ lvs, DevTransT<R> T, const int2* __restrict__ pairs) {
    chain_wait();
    using C = typename Cx<R>::T;
    extern __shared__ unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int2 pc = pairs[blockIdx.x];  // parent index, child entry
    const DevLevelT<R> P = lvs[T.plevel];
    const DevLevelT<R> Cl = lvs[T.plevel + 1];
    const int pth = P.nth, pph = P.nph, cth = Cl.nth, cph = Cl.nph, halfc = Cl.nph / 2;
    const C* Bp = P.B + static_cast<size_t>(T.par_box[pc.x]) * P.ndir * 2;
    const C* sh = P.shift_down + static_cast<size_t>(T.child_oct[pc.y]) * P.ndir;
    for (int e = threadIdx.x; e < pth * cph; e += blockDim.x) {
        const int ith = e / cph, jph = e - ith * cph;
        C v0 = zero<C>(), v1 = zero<C>();
#pragma unroll
        for (int k = 0; k < W; ++k) {
            const int q = k * cph + jph;  // tap-major
            const int d = ith * pph + T.dn_ph.src_t[q];
            const R cf = T.dn_ph.coef_t[q];
            if (POST) {
                v0 = crfma(cf, Bp[2 * d], v0);
                v1 = crfma(cf, Bp[2 * d + 1], v1);
            } else {
                const C ph = sh[d];
                v0 = crfma(cf, cmul(ph, Bp[2 * d]), v0);
                v1 = crfma(cf, cmul(ph, Bp[2 * d + 1]), v1);
            }
        }
        sm[2 * e] = v0;
        sm[2 * e + 1] = v1;
    }
    __syncthreads();
    C* Bc = Cl.B + static_cast<size_t>(T.child_box[pc.y]) * Cl.ndir * 2;
    for (int e = threadIdx.x; e < cth * cph; e += blockDim.x) {
        const int jth = e / cph, jph = e - jth * cph;
        C v0 = zero<C>(), v1 = zero<C>();
#pragma unroll
        for (int k = 0; k < W; ++k) {
            const int q = jth * W + k;
            const bool rf = T.dn_th.refl[q];
            const int sp = rf ? (jph < halfc ? jph + halfc : jph - halfc) : jph;
            const R cf = T.dn_th.coef[q];
            const C* row = sm + (static_cast<size_t>(T.dn_th.src[q]) * cph + sp) * 2;
            v0 = crfma(cf, row[0], v0);
            v1 = crfma(cf, row[1], v1);
        }
        if (POST) {
            const C ph = Cl.shift_up[static_cast<size_t>(T.child_oct[pc.y]) * Cl.ndir + e];
            v0 = cmul(ph, v0);
            v1 = cmul(ph, v1);
        }
        Bc[2 * e] = cadd(Bc[2 * e], v0);
        Bc[2 * e + 1] = cadd(Bc[2 * e + 1], v1);
    }
}

// ------------------------------------------------------------ staged interpolation
// M2M with the children shifted and summed on the child grid first:
// U = sum_c shift_up(oct_c) A_c over the child theta rows the block's
// stencils read, then the theta pass (pole reflection as in k_m2m) into V,
// then the phi pass to the parent.  Interpolation is linear and the same for
// every child, so this is k_m2m's sum in another order (one interpolation per
// parent instead of one per child).  Block = (parent, tile of `rows` parent
// theta rows); each child value is read from global memory once per block and
// every stencil tap reads shared memory.
template <class R, int W, bool CS>  // taps per row: 2 * interp_order (both passes); CS: column-stationary phi pass
__global__ void __launch_bounds__(256)
k_m2m_sum(const DevLevelT<R>* __restrict__ lvs, DevTransT<R> T, int rows) {
    chain_wait();
    using C = typename Cx<R>::T;
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ int band[2];
    const int par = blockIdx.x;
    const DevLevelT<R> P = lvs[T.plevel];
    const DevLevelT<R> Cl = lvs[T.plevel + 1];
    const int nph = P.nph, mph = Cl.nph, halfm = Cl.nph / 2;
    const int r0 = blockIdx.y * rows;
    const int nrow = min(P.nth, r0 + rows) - r0;
    if (nrow <= 0) return;  // the whole block
    if (threadIdx.x == 0) {
        band[0] = Cl.nth;
        band[1] = -1;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nrow * W; q += blockDim.x) {
        const int src = T.up_th.src[r0 * W + q];
        atomicMin(&band[0], src);
        atomicMax(&band[1], src);
    }
    __syncthreads();
    const int lo = band[0], nb = band[1] - lo + 1;
    // component planes (theta, phi), so that neighbouring threads read
    // neighbouring 8- or 16-byte words of shared memory
    const size_t nu = static_cast<size_t>(nb) * mph, nv = static_cast<size_t>(nrow) * mph;
    C* U0 = reinterpret_cast<C*>(smraw);  // [nb * mph], child rows lo..lo+nb-1
    C* U1 = U0 + nu;
    C* V0 = U1 + nu;                      // [nrow * mph]
    C* V1 = V0 + nv;
    const int c0 = T.child_ptr[par], nch = T.child_ptr[par + 1] - c0;
    for (int e = threadIdx.x; e < nb * mph; e += blockDim.x) {
        const int d = lo * mph + e;
        C u0 = zero<C>(), u1 = zero<C>();
#pragma unroll 8
        for (int c = 0; c < nch; ++c) {
            const C* Ac = Cl.A + static_cast<size_t>(T.child_box[c0 + c]) * Cl.ndir * 2;
            const C ph = Cl.shift_up[static_cast<size_t>(T.child_oct[c0 + c]) * Cl.ndir + d];
            u0 = cfma(ph, Ac[2 * d], u0);
            u1 = cfma(ph, Ac[2 * d + 1], u1);
        }
        U0[e] = u0;
        U1[e] = u1;
    }
    __syncthreads();
    for (int it = threadIdx.x; it < nrow * mph; it += blockDim.x) {
        const int jr = it / mph, iph = it - jr * mph;
        const int jth = r0 + jr;
        C v0 = zero<C>(), v1 = zero<C>();
#pragma unroll
        for (int k = 0; k < W; ++k) {
            const int q = jth * W + k;
            const bool rf = T.up_th.refl[q];
            const int sp = rf ? (iph < halfm ? iph + halfm : iph - halfm) : iph;
            const R cf = T.up_th.coef[q];
            const int e = (T.up_th.src[q] - lo) * mph + sp;
            v0 = crfma(cf, U0[e], v0);
            v1 = crfma(cf, U1[e], v1);
        }
        V0[it] = v0;
        V1[it] = v1;
    }
    __syncthreads();
    C* Ap = P.A + (static_cast<size_t>(T.par_box[par]) * P.ndir + static_cast<size_t>(r0) * nph) * 2;
    if (!CS) {  // one output per thread, stencil read per tap (tap-major)
        for (int o = threadIdx.x; o < nrow * nph; o += blockDim.x) {
            const int jr = o / nph, jph = o - jr * nph;
            const C* row0 = V0 + static_cast<size_t>(jr) * mph;
            const C* row1 = V1 + static_cast<size_t>(jr) * mph;
            C a0 = zero<C>(), a1 = zero<C>();
#pragma unroll
            for (int k = 0; k < W; ++k) {
                const int q = k * nph + jph;
                const int s = T.up_ph.src_t[q];
                const R cf = T.up_ph.coef_t[q];
                a0 = crfma(cf, row0[s], a0);
                a1 = crfma(cf, row1[s], a1);
            }
            Ap[2 * o] = a0;
            Ap[2 * o + 1] = a1;
        }
        return;
    }
    // phi pass, column-stationary: a thread keeps one output column's stencil
    // in registers and walks the tile's rows (every row uses the same stencil)
    const int ng = max(1, static_cast<int>(blockDim.x) / nph);  // row groups
    for (int t = threadIdx.x; t < nph * ng; t += blockDim.x) {
        const int jph = t % nph, g = t / nph;
        int sk[W];
        R ck[W];
#pragma unroll
        for (int k = 0; k < W; ++k) {
            sk[k] = T.up_ph.src_t[k * nph + jph];
            ck[k] = T.up_ph.coef_t[k * nph + jph];
        }
        for (int jr = g; jr < nrow; jr += ng) {
            const C* row0 = V0 + static_cast<size_t>(jr) * mph;
            const C* row1 = V1 + static_cast<size_t>(jr) * mph;
            C a0 = zero<C>(), a1 = zero<C>();
#pragma unroll
            for (int k = 0; k < W; ++k) {
                a0 = crfma(ck[k], row0[sk[k]], a0);
                a1 = crfma(ck[k], row1[sk[k]], a1);
            }
            const int o = jr * nph + jph;
            Ap[2 * o] = a0;
            Ap[2 * o + 1] = a1;
        }
    }
}

// Shared memory of k_m2m_sum for a tile of `rows` parent rows (bound: every
// child row in the band).
inline size_t m2m_sum_smem(int child_nth, int child_nph, int rows, size_t csize) {
    return static_cast<size_t>(child_nth + rows) * child_nph * 2 * csize;
}

// L2L (and, POST, the transposed M2M) with the parent's local pattern, shifted
// to the child's octant, staged in shared memory once per block: the same
// arithmetic in the same order as k_l2l, every phi tap then reading shared
// memory instead of global memory.  One block per (parent, child) pair.
template <class R, int W, bool POST, bool CS>  // both transposed stencils padded to W taps per row
__global__ void __launch_bounds__(256)
k_l2l_st(const DevLevelT<R>* __restrict__ lvs, DevTransT<R> T, const int2* __restrict__ pairs) {
    chain_wait();
    using C = typename Cx<R>::T;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int2 pc = pairs[blockIdx.x];  // parent index, child entry
    const DevLevelT<R> P = lvs[T.plevel];
    const DevLevelT<R> Cl = lvs[T.plevel + 1];
    const int pth = P.nth, pph = P.nph, cth = Cl.nth, cph = Cl.nph, halfc = Cl.nph / 2;
    // component planes (theta, phi): neighbouring threads read neighbouring words
    const size_t np = static_cast<size_t>(pth) * pph, nq = static_cast<size_t>(pth) * cph;
    C* SB0 = reinterpret_cast<C*>(smraw);  // [pth * pph]
    C* SB1 = SB0 + np;
    C* S10 = SB1 + np;                     // [pth * cph]
    C* S11 = S10 + nq;
    const C* Bp = P.B + static_cast<size_t>(T.par_box[pc.x]) * P.ndir * 2;
    const C* sh = P.shift_down + static_cast<size_t>(T.child_oct[pc.y]) * P.ndir;
    for (int d = threadIdx.x; d < pth * pph; d += blockDim.x) {
        C b0 = Bp[2 * d], b1 = Bp[2 * d + 1];
        if (!POST) {
            const C ph = sh[d];
            b0 = cmul(ph, b0);
            b1 = cmul(ph, b1);
        }
        SB0[d] = b0;
        SB1[d] = b1;
    }
    __syncthreads();
    if (!CS) {  // one output per thread, stencil read per tap (tap-major)
        for (int e = threadIdx.x; e < pth * cph; e += blockDim.x) {
            const int ith = e / cph, jph = e - ith * cph;
            const C* row0 = SB0 + static_cast<size_t>(ith) * pph;
            const C* row1 = SB1 + static_cast<size_t>(ith) * pph;
            C v0 = zero<C>(), v1 = zero<C>();
#pragma unroll
            for (int k = 0; k < W; ++k) {
                const int q = k * cph + jph;
                const int d = T.dn_ph.src_t[q];
                const R cf = T.dn_ph.coef_t[q];
                v0 = crfma(cf, row0[d], v0);
                v1 = crfma(cf, row1[d], v1);
            }
            S10[e] = v0;
            S11[e] = v1;
        }
    }
    // phi pass, column-stationary: a thread keeps one child column's stencil in
    // registers and walks the parent's theta rows (the same stencil for each)
    const int ng = CS ? max(1, static_cast<int>(blockDim.x) / cph) : 0;  // row groups
    for (int t = threadIdx.x; t < cph * ng; t += blockDim.x) {
        const int jph = t % cph, g = t / cph;
        int sk[W];
        R ck[W];
#pragma unroll
        for (int k = 0; k < W; ++k) {
            sk[k] = T.dn_ph.src_t[k * cph + jph];
            ck[k] = T.dn_ph.coef_t[k * cph + jph];
        }
        for (int ith = g; ith < pth; ith += ng) {
            const C* row0 = SB0 + static_cast<size_t>(ith) * pph;
            const C* row1 = SB1 + static_cast<size_t>(ith) * pph;
            C v0 = zero<C>(), v1 = zero<C>();
#pragma unroll
            for (int k = 0; k < W; ++k) {
                v0 = crfma(ck[k], row0[sk[k]], v0);
                v1 = crfma(ck[k], row1[sk[k]], v1);
            }
            S10[ith * cph + jph] = v0;
            S11[ith * cph + jph] = v1;
        }
    }
    __syncthreads();
    C* Bc = Cl.B + static_cast<size_t>(T.child_box[pc.y]) * Cl.ndir * 2;
    for (int e = threadIdx.x; e < cth * cph; e += blockDim.x) {
        const int jth = e / cph, jph = e - jth * cph;
        C v0 = zero<C>(), v1 = zero<C>();
#pragma unroll
        for (int k = 0; k < W; ++k) {
            const int q = jth * W + k;
            const bool rf = T.dn_th.refl[q];
            const int sp = rf ? (jph < halfc ? jph + halfc : jph - halfc) : jph;
            const R cf = T.dn_th.coef[q];
            const size_t at = static_cast<size_t>(T.dn_th.src[q]) * cph + sp;
            v0 = crfma(cf, S10[at], v0);
            v1 = crfma(cf, S11[at], v1);
        }
        if (POST) {
            const C ph = Cl.shift_up[static_cast<size_t>(T.child_oct[pc.y]) * Cl.ndir + e];
            v0 = cmul(ph, v0);
            v1 = cmul(ph, v1);
        }
        Bc[2 * e] = cadd(Bc[2 * e], v0);
        Bc[2 * e + 1] = cadd(Bc[2 * e + 1], v1);
    }
}

// The staged L2L as a persistent, software-pipelined kernel: each block walks
// the pairs blockIdx.x, blockIdx.x + gridDim.x, ... and, while it computes one
// pair, the next pair's parent pattern, shift and child local pattern arrive by
// asynchronous copies (cp.async, 8 or 16 bytes per copy) into the other half of
// a double buffer; the child's updated local is written with plain stores.
// Same arithmetic in the same order as k_l2l_st<..., false>.
__device__ __forceinline__ void cp_async_elem(void* dst, const void* src, int bytes) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    if (bytes == 16)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

template <class R, int W, bool POST>
__global__ void __launch_bounds__(256)
k_l2l_pipe(const DevLevelT<R>* __restrict__ lvs, DevTransT<R> T, const int2* __restrict__ pairs, int npairs) {
    chain_wait();
    using C = typename Cx<R>::T;
    extern __shared__ __align__(16) unsigned char smraw[];
    const DevLevelT<R> P = lvs[T.plevel];
    const DevLevelT<R> Cl = lvs[T.plevel + 1];
    const int pth = P.nth, pph = P.nph, cth = Cl.nth, cph = Cl.nph, halfc = Cl.nph / 2;
    const int np = pth * pph, nq = pth * cph, nc = cth * cph;
    const int nsh = POST ? nc : np;  // shift values: parent grid (before) or child grid (after, POST)
    // per buffer: raw parent [2 np] (interleaved, as stored), shift [nsh], child [2 nc]
    const size_t per_buf = 2 * static_cast<size_t>(np) + nsh + 2 * static_cast<size_t>(nc);
    C* buf0 = reinterpret_cast<C*>(smraw);
    C* SB0 = buf0 + 2 * per_buf;  // planes [np] x 2, then S1 planes [nq] x 2
    C* SB1 = SB0 + np;
    C* S10 = SB1 + np;
    C* S11 = S10 + nq;
    auto issue = [&](int pi, int b) {
        const int2 pc = pairs[pi];
        C* raw = buf0 + b * per_buf;
        C* shv = raw + 2 * np;
        C* cl = shv + nsh;
        const C* Bp = P.B + static_cast<size_t>(T.par_box[pc.x]) * P.ndir * 2;
        const C* sh = POST ? Cl.shift_up + static_cast<size_t>(T.child_oct[pc.y]) * Cl.ndir
                           : P.shift_down + static_cast<size_t>(T.child_oct[pc.y]) * P.ndir;
        const C* Bc = Cl.B + static_cast<size_t>(T.child_box[pc.y]) * Cl.ndir * 2;
        for (int i = threadIdx.x; i < 2 * np; i += blockDim.x) cp_async_elem(raw + i, Bp + i, sizeof(C));
        for (int i = threadIdx.x; i < nsh; i += blockDim.x) cp_async_elem(shv + i, sh + i, sizeof(C));
        for (int i = threadIdx.x; i < 2 * nc; i += blockDim.x) cp_async_elem(cl + i, Bc + i, sizeof(C));
    };
    int b = 0;
    if (static_cast<int>(blockIdx.x) < npairs) issue(blockIdx.x, 0);
    cp_async_commit();
    for (int pi = blockIdx.x; pi < npairs; pi += gridDim.x, b ^= 1) {
        const int nxt = pi + gridDim.x;
        if (nxt < npairs) issue(nxt, b ^ 1);
        cp_async_commit();  // (possibly empty) group, so that wait_group 1 means "this pair"
        cp_async_wait1();
        __syncthreads();
        const C* raw = buf0 + b * per_buf;
        const C* shv = raw + 2 * np;
        const C* cl = shv + nsh;
        for (int d = threadIdx.x; d < np; d += blockDim.x) {
            C b0 = raw[2 * d], b1 = raw[2 * d + 1];
            if (!POST) {
                const C ph = shv[d];
                b0 = cmul(ph, b0);
                b1 = cmul(ph, b1);
            }
            SB0[d] = b0;
            SB1[d] = b1;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < nq; e += blockDim.x) {
            const int ith = e / cph, jph = e - ith * cph;
            const C* row0 = SB0 + static_cast<size_t>(ith) * pph;
            const C* row1 = SB1 + static_cast<size_t>(ith) * pph;
            C v0 = zero<C>(), v1 = zero<C>();
#pragma unroll
            for (int k = 0; k < W; ++k) {
                const int q = k * cph + jph;
                const int d = T.dn_ph.src_t[q];
                const R cf = T.dn_ph.coef_t[q];
                v0 = crfma(cf, row0[d], v0);
                v1 = crfma(cf, row1[d], v1);
            }
            S10[e] = v0;
            S11[e] = v1;
        }
        __syncthreads();
        const int2 pc = pairs[pi];
        C* Bc = Cl.B + static_cast<size_t>(T.child_box[pc.y]) * Cl.ndir * 2;
        for (int e = threadIdx.x; e < nc; e += blockDim.x) {
            const int jth = e / cph, jph = e - jth * cph;
            C v0 = zero<C>(), v1 = zero<C>();
#pragma unroll
            for (int k = 0; k < W; ++k) {
                const int q = jth * W + k;
                const bool rf = T.dn_th.refl[q];
                const int sp = rf ? (jph < halfc ? jph + halfc : jph - halfc) : jph;
                const R cf = T.dn_th.coef[q];
                const size_t at = static_cast<size_t>(T.dn_th.src[q]) * cph + sp;
                v0 = crfma(cf, S10[at], v0);
                v1 = crfma(cf, S11[at], v1);
            }
            if (POST) {
                const C ph = shv[e];
                v0 = cmul(ph, v0);
                v1 = cmul(ph, v1);
            }
            Bc[2 * e] = cadd(cl[2 * e], v0);
            Bc[2 * e + 1] = cadd(cl[2 * e + 1], v1);
        }
        __syncthreads();  // buffers and planes free for the next pair
    }
}

inline size_t l2l_pipe_smem(int pth, int pph, int cth, int cph, size_t csize) {
    const size_t np = static_cast<size_t>(pth) * pph, nc = static_cast<size_t>(cth) * cph;
    const size_t per_buf = 2 * np + std::max(np, nc) + 2 * nc;
    return (2 * per_buf + 2 * np + 2 * static_cast<size_t>(pth) * cph) * csize;
}

inline size_t l2l_st_smem(int parent_nth, int parent_nph, int child_nph, size_t csize) {
    return static_cast<size_t>(parent_nth) * (parent_nph + child_nph) * 2 * csize;
}

// Complex double -> far-field type (patterns, tables at setup).
template <class C>
__global__ void k_narrow(const double2* __restrict__ src, C* __restrict__ dst, long long n) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = from_d2<C>(src[i]);
}

}  // namespace
}  // namespace mlfma
