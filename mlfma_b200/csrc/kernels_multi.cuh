// Many right-hand sides in one product: the far-field stages and the near
// field applied to nr vectors at once.  Included once, by kernels.cu.
//
// Layout with the right-hand side innermost, so that every thread of a warp
// reads a different right-hand side of the same element (coalesced), and
// every coefficient (pattern, transfer function, stencil weight, near-field
// entry) is read once per product instead of once per right-hand side:
//   x, y (tree order)     [n][nr]
//   A_l, B_l per level     [box][direction][2 components][nr]
//
// S2M, L2T and the near field are small dense complex products per leaf
// (patterns x right-hand sides), done by one register-tiled complex GEMM
// device routine; M2L works on sibling groups (the children of one parent
// share their candidate source boxes), so each source pattern is read once per
// group rather than once per interaction pair; interpolation and
// anterpolation keep the single-product structure over chunks of right-hand
// sides.
#pragma once

#include "device.cuh"
#include "zmath.cuh"

namespace mlfma {
namespace {

// ------------------------------------------------------------ complex GEMM tile
// One thread block computes a BM x BN tile of
//   Cm[m][n] = sum_k opA(m, k) * B(k, n)
// with opA(m, k) = A[m * sam + k * sak] (conjugated when CONJ_A), B row k at
// B + (bidx ? bidx[k] : k) * ldb (entries n contiguous), output element (m, n)
// at out + m * ldc + n, converted to the output type.  K is walked in chunks of
// BK through shared memory; each of the 128 threads keeps a 4 x 4 register
// tile (16 complex products per 8 shared-memory loads).
constexpr int kGemmThreads = 128;
constexpr int kBM = 32, kBN = 64, kBK = 8;
constexpr int kLdA = kBM * kBK / kGemmThreads;  // A entries loaded per thread (2)
constexpr int kLdB = kBK * kBN / kGemmThreads;  // B entries loaded per thread (4)

template <class C> __device__ __forceinline__ C conj_c(C a) { a.y = -a.y; return a; }
template <class C, class S> __device__ __forceinline__ C to_c(S v);
template <> __device__ __forceinline__ double2 to_c<double2, double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 to_c<float2, float2>(float2 v) { return v; }
template <> __device__ __forceinline__ float2 to_c<float2, double2>(double2 v) {
    return make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
}
template <> __device__ __forceinline__ double2 to_c<double2, float2>(float2 v) { return make_double2(v.x, v.y); }

template <class C, class TA, class TB, class TO, bool CONJ_A, bool A_KMAJOR>
__device__ __forceinline__ void cgemm_tile(int M, int N, int K, int m0, int n0, const TA* __restrict__ A,
                                           long long sam, long long sak, const TB* __restrict__ B,
                                           const int* __restrict__ bidx, long long ldb, TO* __restrict__ out,
                                           long long ldc, C (*As)[kBM + 1], C (*Bs)[kBN]) {
    const int tid = threadIdx.x;
    const int ty = tid >> 4, tx = tid & 15;  // rows 4 ty .. 4 ty + 3, columns tx + 16 j
    C acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = zero<C>();
    // Registers of the next tile: its global loads are in flight while the
    // current tile is multiplied out of shared memory.
    C ra[kLdA], rb[kLdB];
    auto load = [&](int k0) {
#pragma unroll
        for (int u = 0; u < kLdA; ++u) {  // A tile: BM x BK
            const int idx = tid + u * kGemmThreads;
            int mm, kk;
            if (A_KMAJOR) { mm = idx / kBK; kk = idx % kBK; } else { kk = idx / kBM; mm = idx % kBM; }
            const int m = m0 + mm, k = k0 + kk;
            C v = zero<C>();
            if (m < M && k < K) {
                v = to_c<C, TA>(A[m * sam + k * sak]);
                if (CONJ_A) v = conj_c(v);
            }
            ra[u] = v;
        }
#pragma unroll
        for (int u = 0; u < kLdB; ++u) {  // B tile: BK x BN
            const int idx = tid + u * kGemmThreads;
            const int kk = idx / kBN, nn = idx % kBN;
            const int k = k0 + kk, n = n0 + nn;
            C v = zero<C>();
            if (k < K && n < N) {
                const long long row = bidx ? static_cast<long long>(bidx[k]) : static_cast<long long>(k);
                v = to_c<C, TB>(B[row * ldb + n]);
            }
            rb[u] = v;
        }
    };
    load(0);
    for (int k0 = 0; k0 < K; k0 += kBK) {
#pragma unroll
        for (int u = 0; u < kLdA; ++u) {
            const int idx = tid + u * kGemmThreads;
            if (A_KMAJOR) As[idx % kBK][idx / kBK] = ra[u]; else As[idx / kBM][idx % kBM] = ra[u];
        }
#pragma unroll
        for (int u = 0; u < kLdB; ++u) {
            const int idx = tid + u * kGemmThreads;
            Bs[idx / kBN][idx % kBN] = rb[u];
        }
        __syncthreads();
        if (k0 + kBK < K) load(k0 + kBK);
#pragma unroll
        for (int kk = 0; kk < kBK; ++kk) {
            C a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][4 * ty + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = cfma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = m0 + 4 * ty + i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = n0 + tx + 16 * j;
            if (n < N) out[m * ldc + n] = to_c<TO, C>(acc[i][j]);
        }
    }
}

// ------------------------------------------------------------ S2M (many)
// A_B[e][r] = sum_s R_s[e] x_s[r]  (Leaf::buildMpoleCoeffs, src/fmm/leaf.cpp:212-230,
// for nr vectors).  Work item: (leaf, first row e0 of a BM-row tile).
template <class R>
__global__ void __launch_bounds__(kGemmThreads)
k_s2m_m(const DevLevelT<R>* __restrict__ lvs, const int2* __restrict__ items, const DevFarLeaf* __restrict__ leaves,
        const typename Cx<R>::T* __restrict__ pat, const double2* __restrict__ x, int nr) {
    using C = typename Cx<R>::T;
    __shared__ C As[kBK][kBM + 1];
    __shared__ C Bs[kBK][kBN];
    const int2 it = items[blockIdx.x];
    const DevFarLeaf lf = leaves[it.x];
    const int ne = 2 * lvs[lf.level].ndir;
    C* Am = lvs[lf.level].Am + static_cast<size_t>(lf.box) * ne * nr;
    for (int n0 = 0; n0 < nr; n0 += kBN)
        cgemm_tile<C, C, double2, C, false, false>(ne, nr, lf.nsrc, it.y, n0, pat + lf.pat_off * 2, 1, ne,
                                                   x + static_cast<size_t>(lf.src0) * nr, nullptr, nr, Am, nr,
                                                   As, Bs);
}

// ------------------------------------------------------------ L2T (many)
// y_s[r] = sum_e conj(R_s[e]) b_B[e][r]  (Leaf::evalFarSols, src/fmm/leaf.cpp:257-280).
// Work item: (leaf, first source s0 of a BM-source tile).
template <class R>
__global__ void __launch_bounds__(kGemmThreads)
k_l2t_m(const DevLevelT<R>* __restrict__ lvs, const int2* __restrict__ items, const DevFarLeaf* __restrict__ leaves,
        const typename Cx<R>::T* __restrict__ pat, double2* __restrict__ yfar, int nr) {
    using C = typename Cx<R>::T;
    __shared__ C As[kBK][kBM + 1];
    __shared__ C Bs[kBK][kBN];
    const int2 it = items[blockIdx.x];
    const DevFarLeaf lf = leaves[it.x];
    const int ne = 2 * lvs[lf.level].ndir;
    const C* Bm = lvs[lf.level].Bm + static_cast<size_t>(lf.box) * ne * nr;
    for (int n0 = 0; n0 < nr; n0 += kBN)
        cgemm_tile<C, C, C, double2, true, true>(lf.nsrc, nr, ne, it.y, n0, pat + lf.pat_off * 2, ne, 1, Bm,
                                                 nullptr, nr, yfar + static_cast<size_t>(lf.src0) * nr, nr, As, Bs);
}

// ------------------------------------------------------------ near field (many)
// y_i[r] = sum_j Z_ij x_cols(j)[r] per block row (gather form, both
// orientations stored).  Work item: (row block, first row of a BM-row tile).
__global__ void __launch_bounds__(kGemmThreads)
k_near_m(const DevNearRow* __restrict__ rows, const int2* __restrict__ items, const double2* __restrict__ Z,
         const int* __restrict__ cols, const double2* __restrict__ x, double2* __restrict__ y, int nr) {
    __shared__ double2 As[kBK][kBM + 1];
    __shared__ double2 Bs[kBK][kBN];
    const int2 it = items[blockIdx.x];
    const DevNearRow Rw = rows[it.x];
    for (int n0 = 0; n0 < nr; n0 += kBN)
        cgemm_tile<double2, double2, double2, double2, false, true>(
            Rw.nrow, nr, Rw.ncol, it.y, n0, Z + Rw.off, Rw.ncol, 1, x, cols + Rw.col_off, nr,
            y + static_cast<size_t>(Rw.row0) * nr, nr, As, Bs);
}

// ------------------------------------------------------------ M2L (many)
// b_B = w (2 pi / nph) sum_{S in list 2 of B} T[c_B - c_S] a_S
// (Node::buildMpoleToLocalCoeffs, src/fmm/node.cpp:105-134).  One block per
// (sibling group, direction); thread = (component, rhs), blockDim = 2 nr
// rounded up to a warp.  The group's candidate sources are walked once; each
// loaded pattern value is used for every target of the group that has the
// source in its list 2.
constexpr int kM2LmThreads = 128;  // nr <= 64

// The transfer values are pre-gathered per group at setup, already scaled by
// the quadrature weight: t8[group][direction][candidate][target] (zero where
// the candidate is not in the target's list 2), so the inner loop has one
// dependent global load (the candidate's pattern) and reads the transfer
// values from shared memory.
constexpr int kCandChunk = 64;

template <class R>
__global__ void __launch_bounds__(kM2LmThreads)
k_m2l_m(const DevLevelT<R>* __restrict__ lvs, const int2* __restrict__ items, const DevM2LGroup* __restrict__ groups,
        const int* __restrict__ cand_src, const typename Cx<R>::T* __restrict__ t8, int nr, int zero_empty) {
    using C = typename Cx<R>::T;
    constexpr int U = sizeof(R) == 4 ? 8 : 4;  // candidates whose loads are in flight together
    __shared__ C tsm[kCandChunk][kMaxGroup];
    __shared__ int ssm[kCandChunk];
    const int2 it = items[blockIdx.x];  // group, direction
    const DevM2LGroup g = groups[it.x];
    const DevLevelT<R> lv = lvs[g.level];
    const int per_dir = 2 * nr;
    const int cr = threadIdx.x;  // component * nr + r
    const int d = it.y;
    const int ndir = lv.ndir;
    const bool live = cr < per_dir;
    C acc[kMaxGroup];
#pragma unroll
    for (int t = 0; t < kMaxGroup; ++t) acc[t] = zero<C>();
    const C* tg = t8 + g.t8_off + static_cast<long long>(d) * g.ncand * kMaxGroup;
    for (int c0 = 0; c0 < g.ncand; c0 += kCandChunk) {
        const int nc = min(kCandChunk, g.ncand - c0);
        for (int i = threadIdx.x; i < nc * kMaxGroup; i += blockDim.x)
            tsm[i / kMaxGroup][i % kMaxGroup] = tg[static_cast<long long>(c0) * kMaxGroup + i];
        for (int i = threadIdx.x; i < nc; i += blockDim.x) ssm[i] = cand_src[g.cand0 + c0 + i];
        __syncthreads();
        if (live)
            for (int i = 0; i < nc; i += U) {
                C a[U];
#pragma unroll
                for (int u = 0; u < U; ++u)
                    a[u] = (i + u < nc) ? lv.Am[(static_cast<size_t>(ssm[i + u]) * ndir + d) * per_dir + cr] : zero<C>();
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (i + u >= nc) break;
#pragma unroll
                    for (int t = 0; t < kMaxGroup; ++t) acc[t] = cfma(tsm[i + u][t], a[u], acc[t]);
                }
            }
        __syncthreads();
    }
    if (!live) return;
#pragma unroll
    for (int t = 0; t < kMaxGroup; ++t) {
        if (t >= g.ntgt) break;
        C* out = lv.Bm + (static_cast<size_t>(g.tgt[t]) * ndir + d) * per_dir + cr;
        if ((g.empty_mask >> t) & 1) {
            if (zero_empty) *out = zero<C>();
        } else {
            *out = acc[t];
        }
    }
}

// ------------------------------------------------------------ M2M (many)
// Interpolation and anterpolation on many right-hand sides work on chunks of
// 16 x RPL right-hand sides: lane = component * 16 + r, and each lane carries
// right-hand sides r, r + 16, ... of the chunk, so the 32 lanes of a warp read
// one pattern entry for the whole chunk and both components, while every
// stencil index, weight and shift is the same for the whole warp and is paid
// once per RPL values; warps stride over grid positions.  (kRc: the chunk of
// the anterpolation kernel, RPL = 2.)
constexpr int kRc = 32;
constexpr int kInterpThreads = 256;
constexpr int kInterpWarps = kInterpThreads / 32;
constexpr int kM2MOut = 16;  // most parent phi columns per warp held in registers

// Parent outgoing patterns = sum over children of Interp[shift(child)]
// (Stem::buildMpoleCoeffs and addInterpCoeffs, src/fmm/stem.cpp:72-184).
// Block = (parent, parent theta row, rhs chunk of 16 m2m_rpl right-hand
// sides).  Children one at a time: theta pass of the child into shared memory
// (one row of child phi columns), then the phi pass accumulated in registers
// over the children.  Complex double carries two right-hand sides per lane;
// complex float one (two measured slower: register pressure).
template <class R> __host__ __device__ constexpr int m2m_rpl() { return sizeof(R) == 4 ? 1 : 2; }
template <class R> __host__ __device__ constexpr bool m2m_rows_fast() { return sizeof(R) == 8; }

template <class R, int W, int OUT>  // OUT: parent phi columns per warp (nph <= OUT * 8)
__global__ void __launch_bounds__(kInterpThreads)
k_m2m_m(const DevLevelT<R>* __restrict__ lvs, DevTransT<R> T, int nr, int rows_fast) {
    using C = typename Cx<R>::T;
    constexpr int RPL = m2m_rpl<R>();
    extern __shared__ unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);  // [mph][32 lanes][RPL]
    // grid order: rows fastest (the blocks of one parent together, its
    // children read from DRAM about once; the FP64 default) or parents
    // fastest (the complex-float default); the autotuner may change it
    const int jth = rows_fast ? blockIdx.x : blockIdx.y;
    const int par = rows_fast ? blockIdx.z : blockIdx.x;
    const int r0 = (rows_fast ? blockIdx.y : blockIdx.z) * 16 * RPL;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int comp = lane >> 4, r = lane & 15;
    bool live[RPL];
#pragma unroll
    for (int j = 0; j < RPL; ++j) live[j] = r0 + r + 16 * j < nr;
    const int col = comp * nr + r0 + r;  // offset of (component, rhs) inside a direction
    const DevLevelT<R> P = lvs[T.plevel];
    const DevLevelT<R> Cl = lvs[T.plevel + 1];
    const int nph = P.nph, mph = Cl.nph, halfm = Cl.nph / 2;
    const int c0 = T.child_ptr[par], nch = T.child_ptr[par + 1] - c0;
    // Stencils in shared memory: this row's theta taps (sources; the weights
    // come with the shift from fold_up), every column's phi taps.
    __shared__ int th_src[W], th_refl[W];
    __shared__ int ph_src[OUT * kInterpWarps * W];
    __shared__ R ph_cf[OUT * kInterpWarps * W];
    if (threadIdx.x < W) {
        th_src[threadIdx.x] = T.up_th.src[jth * W + threadIdx.x];
        th_refl[threadIdx.x] = T.up_th.refl[jth * W + threadIdx.x];
    }
    for (int i = threadIdx.x; i < nph * W; i += blockDim.x) {
        ph_src[i] = T.up_ph.src[i];
        ph_cf[i] = T.up_ph.coef[i];
    }
    __syncthreads();
    C acc[OUT][RPL];
#pragma unroll
    for (int u = 0; u < OUT; ++u)
#pragma unroll
        for (int j = 0; j < RPL; ++j) acc[u][j] = zero<C>();
    if (nch == 0)  // (a listed parent has a child; kept well defined regardless)
        for (int iph = warp; iph < mph; iph += kInterpWarps)
#pragma unroll
            for (int j = 0; j < RPL; ++j) sm[(iph * 32 + lane) * RPL + j] = zero<C>();
    for (int c = 0; c < nch; ++c) {
        const C* Ac = Cl.Am + static_cast<size_t>(T.child_box[c0 + c]) * Cl.ndir * 2 * nr + col;
        // weights of this row with the child's octant shift folded in: [iph][k]
        const C* fu = T.fold_up + (static_cast<size_t>(T.child_oct[c0 + c]) * P.nth + jth) * mph * W;
        for (int iph = warp; iph < mph; iph += kInterpWarps) {
            const int iref = iph < halfm ? iph + halfm : iph - halfm;
            C v[RPL];
#pragma unroll
            for (int j = 0; j < RPL; ++j) v[j] = zero<C>();
#pragma unroll
            for (int k = 0; k < W; ++k) {
                const C* a = Ac + static_cast<size_t>(th_src[k] * mph + (th_refl[k] ? iref : iph)) * 2 * nr;
                const C f = fu[iph * W + k];
#pragma unroll
                for (int j = 0; j < RPL; ++j)
                    if (live[j]) v[j] = cfma(f, a[16 * j], v[j]);
            }
            // the phi pass is the same linear map for every child: sum the
            // children's theta passes first (each entry is this thread's own)
#pragma unroll
            for (int j = 0; j < RPL; ++j) {
                C& o = sm[(iph * 32 + lane) * RPL + j];
                o = c == 0 ? v[j] : cadd(o, v[j]);
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < OUT; ++u) {
        const int jph = warp + u * kInterpWarps;
        if (jph >= nph) break;
#pragma unroll
        for (int k = 0; k < W; ++k) {
            const R cf = ph_cf[jph * W + k];
            const C* v = sm + (ph_src[jph * W + k] * 32 + lane) * RPL;
#pragma unroll
            for (int j = 0; j < RPL; ++j) acc[u][j] = crfma(cf, v[j], acc[u][j]);
        }
    }
    C* Ap = P.Am + (static_cast<size_t>(T.par_box[par]) * P.ndir + static_cast<size_t>(jth) * nph) * 2 * nr + col;
#pragma unroll
    for (int u = 0; u < OUT; ++u) {
        const int jph = warp + u * kInterpWarps;
        if (jph >= nph) break;
#pragma unroll
        for (int j = 0; j < RPL; ++j)
            if (live[j]) Ap[static_cast<size_t>(jph) * 2 * nr + 16 * j] = acc[u][j];
    }
}

// ------------------------------------------------------------ L2L (many)
// child local += Anterp[shift(parent local)] (Stem::getShiftedLocalCoeffs and
// addAnterpCoeffs, src/fmm/stem.cpp:109-244).  Block = ((parent, child) pair,
// l2l_pairs child phi column pairs {j, j + cph/2}, rhs chunk): the transposed
// phi pass for those columns over all parent theta rows into shared memory
// (neighbouring columns share most of their parent taps, which then hit L1),
// then the transposed theta pass, whose pole reflection only moves between
// the two columns of a pair.
// (default: 2 column pairs for complex float; 1 for complex double, whose tile
// would otherwise hold occupancy to two blocks per SM; the autotuner may change
// it)
template <class R> __host__ __device__ constexpr int l2l_pairs() { return sizeof(R) == 4 ? 2 : 1; }

template <class R, int W, int kL2LPairs>
__global__ void __launch_bounds__(kInterpThreads)
k_l2l_m(const DevLevelT<R>* __restrict__ lvs, DevTransT<R> T, const int2* __restrict__ pairs, int nr) {
    using C = typename Cx<R>::T;
    constexpr int NC = 2 * kL2LPairs;  // columns of the block
    extern __shared__ unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);  // [pth][NC][32 lanes][2], then the theta taps
    const int2 pc = pairs[blockIdx.x];
    const int r0 = blockIdx.z * kRc;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int comp = lane >> 4, r = lane & 15;
    const bool live0 = r0 + r < nr, live1 = r0 + r + 16 < nr;
    const int col = comp * nr + r0 + r;
    const DevLevelT<R> P = lvs[T.plevel];
    const DevLevelT<R> Cl = lvs[T.plevel + 1];
    const int pth = P.nth, pph = P.nph, cth = Cl.nth, cph = Cl.nph, halfc = Cl.nph / 2;
    const int j0 = blockIdx.y * kL2LPairs, npair = min(kL2LPairs, halfc - j0);
    const C* Bp = P.Bm + static_cast<size_t>(T.par_box[pc.x]) * P.ndir * 2 * nr + col;
    // weights with the child's octant shift folded in: [ith][jph][k]
    const C* fd = T.fold_dn + static_cast<size_t>(T.child_oct[pc.y]) * pth * cph * W;
    // column c of the block: pair c % kL2LPairs, side c / kL2LPairs
    __shared__ int ph_src[NC * W];
    // dynamic shared memory: the tile, then cth x W theta taps (weight, source, reflection)
    R* th_cf = reinterpret_cast<R*>(sm + static_cast<size_t>(pth) * NC * 64);
    int* th_src = reinterpret_cast<int*>(th_cf + cth * W);
    int* th_refl = th_src + cth * W;
    for (int i = threadIdx.x; i < NC * W; i += blockDim.x) {
        const int c = i / W, k = i - c * W;
        const int pr = c % kL2LPairs;
        const int jph = j0 + min(pr, npair - 1) + (c / kL2LPairs) * halfc;
        ph_src[i] = T.dn_ph.src[jph * W + k];
    }
    for (int i = threadIdx.x; i < cth * W; i += blockDim.x) {
        th_src[i] = T.dn_th.src[i];
        th_refl[i] = T.dn_th.refl[i];
        th_cf[i] = T.dn_th.coef[i];
    }
    __syncthreads();
    for (int pos = warp; pos < pth * NC; pos += kInterpWarps) {
        const int ith = pos / NC, c = pos - ith * NC;
        const int jph = j0 + min(c % kL2LPairs, npair - 1) + (c / kL2LPairs) * halfc;
        const C* f = fd + (static_cast<size_t>(ith) * cph + jph) * W;
        C v0 = zero<C>(), v1 = zero<C>();
#pragma unroll
        for (int k = 0; k < W; ++k) {
            const C* b = Bp + static_cast<size_t>(ith * pph + ph_src[c * W + k]) * 2 * nr;
            const C fk = f[k];
            if (live0) v0 = cfma(fk, b[0], v0);
            if (live1) v1 = cfma(fk, b[16], v1);
        }
        sm[(pos * 32 + lane) * 2] = v0;
        sm[(pos * 32 + lane) * 2 + 1] = v1;
    }
    __syncthreads();
    C* Bc = Cl.Bm + static_cast<size_t>(T.child_box[pc.y]) * Cl.ndir * 2 * nr + col;
    for (int pos = warp; pos < cth * NC; pos += kInterpWarps) {
        const int jth = pos / NC, c = pos - jth * NC;
        const int pr = c % kL2LPairs, side = c / kL2LPairs;
        if (pr >= npair) continue;
        C v0 = zero<C>(), v1 = zero<C>();
#pragma unroll
        for (int k = 0; k < W; ++k) {
            const int q = jth * W + k;
            const int c2 = th_refl[q] ? pr + (1 - side) * kL2LPairs : c;
            const C* v = sm + ((th_src[q] * NC + c2) * 32 + lane) * 2;
            v0 = crfma(th_cf[q], v[0], v0);
            v1 = crfma(th_cf[q], v[1], v1);
        }
        C* o = Bc + static_cast<size_t>(jth * cph + j0 + pr + side * halfc) * 2 * nr;
        if (live0) o[0] = cadd(o[0], v0);
        if (live1) o[16] = cadd(o[16], v1);
    }
}

// ------------------------------------------------------------ boundary (many)
// xt[t][r] = x[r][perm[t]]: caller layout (one vector after another, caller
// order) to tree order with the right-hand side innermost.
__global__ void k_gather_m(const double2* __restrict__ x, const int* __restrict__ perm, double2* __restrict__ xt,
                           int n, int nr) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<long long>(n) * nr) return;
    const int t = static_cast<int>(i / nr), r = static_cast<int>(i - static_cast<long long>(t) * nr);
    xt[i] = x[static_cast<size_t>(r) * n + perm[t]];
}

// y[r][perm[t]] (+)= ck (yfar[t][r] + ynear[t][r]) + loads[t] xt[t][r] (loads may
// be null); perm == nullptr: tree order, rhs innermost.
__global__ void k_finish_m(const double2* __restrict__ yfar, const double2* __restrict__ ynear,
                           const int* __restrict__ perm, double2* __restrict__ y, int n, int nr, double2 ck,
                           int accumulate, const double2* __restrict__ xt, const double2* __restrict__ loads) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<long long>(n) * nr) return;
    const int t = static_cast<int>(i / nr), r = static_cast<int>(i - static_cast<long long>(t) * nr);
    double2 v = cmul(ck, cadd(yfar[i], ynear[i]));
    if (loads) v = cfma(loads[t], xt[i], v);
    const size_t o = perm ? static_cast<size_t>(r) * n + perm[t] : static_cast<size_t>(i);
    y[o] = accumulate ? cadd(y[o], v) : v;
}

}  // namespace
}  // namespace mlfma
