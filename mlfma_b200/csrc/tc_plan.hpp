// Index arithmetic of the tensor-core interpolation passes (kernels_tc.cuh),
// shared by the kernels and by host code: the pass arguments, the row ->
// (item, position, float) decomposition, the input each row contracts and the
// output it writes, the MMA operand layouts in shared memory, and the dense
// interpolation weights built from the stencils.  Plain C++ when compiled by a
// host compiler (tests/cpp/tc_check.cpp runs the same functions on the CPU).
#pragma once

#include <vector_types.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "plan.hpp"

#if defined(__CUDACC__)
#define MLFMA_HD __host__ __device__ __forceinline__
#else
#define MLFMA_HD inline
#endif

namespace mlfma {

enum TcKind { kTcTheta = 0, kTcPhi = 1, kTcPhiT = 2, kTcThetaT = 3 };
constexpr int kTcRows = 128;           // rows of a tile (MMA M)
constexpr int kTcKChunk = 64;          // contraction values staged at once
constexpr int kTcShiftFlag = 1 << 30;  // krow entry: source read at phi + pi
constexpr int kTcMaxChildren = 8;

// One pass over a chunk of items (parents for M2M, (parent, child) pairs for L2L).
struct TcArgs {
    int item0, nitems;   // items of this launch
    int J, Q;            // rows per item: J positions on the other axis x Q floats
    int K, Kpad;         // contraction length (reflected rows included), padded to 8
    int N, Npad;         // outputs per row, padded to 16
    int nr;              // right-hand sides in the pattern layout ([dir][2][nr] complex)
    int mth, mph, nth, nph;  // child and parent grids
    const float* w;      // weights: hi then lo, each Npad x Kpad in the canonical K-major layout
    const int* krow;     // [K] source row of each contraction index (theta passes), | kTcShiftFlag
    const float2* pat_in;     // child A (THETA) or parent B (PHI_T)
    float2* pat_out;          // parent A (PHI) or child B (THETA_T)
    const float2* shift;      // child-level shift_up (THETA) / parent-level shift_down (PHI_T): [8][ndir]
    const float* scr_in;      // intermediate written by the first pass of the stage
    float* scr_out;
    const int* child_ptr;
    const int* child_box;
    const int* child_oct;
    const int* par_box;
    const int2* pairs;        // (parent, child entry)
};

// Row f of a pass: item b, position j on the other axis, float q of the
// (component, right-hand side, re/im) entries of one direction.
struct TcRow {
    int b, j, q;
    bool live;
};

MLFMA_HD TcRow tc_row(const TcArgs& a, long long f) {
    const long long per_item = static_cast<long long>(a.J) * a.Q;
    TcRow r{0, 0, 0, f < per_item * a.nitems};
    if (r.live) {
        r.b = static_cast<int>(f / per_item);
        const int rem = static_cast<int>(f - static_cast<long long>(r.b) * per_item);
        r.j = rem / a.Q;
        r.q = rem - r.j * a.Q;
    }
    return r;
}

// Real part (q even) or imaginary part (q odd) of s * x.
MLFMA_HD float tc_cmul_part(float2 s, float2 x, int q) {
    return (q & 1) ? (s.x * x.y + s.y * x.x) : (s.x * x.x - s.y * x.y);
}

// Item context of a row: for THETA the children of the parent (boxes and
// octants, at most 8), for PHI the parent box, for PHI_T the parent box and the
// child's octant, for THETA_T the child box.
struct TcItem {
    int box, oct, nch;
    int cbox[kTcMaxChildren], coct[kTcMaxChildren];
};

template <int KIND>
MLFMA_HD TcItem tc_item(const TcArgs& a, const TcRow& r) {
    TcItem it{};
    const int item = a.item0 + (r.live ? r.b : 0);
    if (KIND == kTcTheta) {
        const int c0 = a.child_ptr[item];
        it.nch = a.child_ptr[item + 1] - c0;
        if (it.nch > kTcMaxChildren) it.nch = kTcMaxChildren;
        for (int c = 0; c < it.nch; ++c) {
            it.cbox[c] = a.child_box[c0 + c];
            it.coct[c] = a.child_oct[c0 + c];
        }
    } else if (KIND == kTcPhi) {
        it.box = a.par_box[item];
    } else if (KIND == kTcPhiT) {
        const int2 pc = a.pairs[item];
        it.box = a.par_box[pc.x];
        it.oct = a.child_oct[pc.y];
    } else {
        it.box = a.child_box[a.pairs[item].y];
    }
    return it;
}

// Input of row r at contraction index k (0 beyond K or past the last row).
template <int KIND>
MLFMA_HD float tc_load(const TcArgs& a, const TcRow& r, int k, const int* krow, const TcItem& it) {
    if (!r.live || k >= a.K) return 0.f;
    const int cq = r.q >> 1;  // complex value (component, rhs) within a direction
    if (KIND == kTcTheta) {
        // sum over the children of shift_up .* A_child at (source row, phi or phi + pi)
        const int kr = krow[k];
        const int th = kr & (kTcShiftFlag - 1);
        const int ph = (kr & kTcShiftFlag) ? (r.j + (a.mph >> 1)) % a.mph : r.j;
        const int ndir = a.mth * a.mph;
        const int d = th * a.mph + ph;
        float v = 0.f;
        for (int c = 0; c < it.nch; ++c) {
            const float2 s = a.shift[static_cast<size_t>(it.coct[c]) * ndir + d];
            const float2 x = a.pat_in[(static_cast<size_t>(it.cbox[c]) * ndir + d) * 2 * a.nr + cq];
            v += tc_cmul_part(s, x, r.q);
        }
        return v;
    } else if (KIND == kTcPhi) {
        // intermediate [item][parent theta row][child phi][Q]
        return a.scr_in[((static_cast<size_t>(r.b) * a.nth + r.j) * a.mph + k) * a.Q + r.q];
    } else if (KIND == kTcPhiT) {
        // shift_down .* B_parent at (parent theta row j, parent phi k)
        const int ndir = a.nth * a.nph;
        const int d = r.j * a.nph + k;
        const float2 s = a.shift[static_cast<size_t>(it.oct) * ndir + d];
        const float2 x = a.pat_in[(static_cast<size_t>(it.box) * ndir + d) * 2 * a.nr + cq];
        return tc_cmul_part(s, x, r.q);
    } else {
        // intermediate [item][parent theta row][child phi][Q] at (source row, phi or phi + pi)
        const int kr = krow[k];
        const int th = kr & (kTcShiftFlag - 1);
        const int ph = (kr & kTcShiftFlag) ? (r.j + (a.mph >> 1)) % a.mph : r.j;
        return a.scr_in[((static_cast<size_t>(r.b) * a.nth + th) * a.mph + ph) * a.Q + r.q];
    }
}

// Output (row r, i) of a pass.
template <int KIND>
MLFMA_HD void tc_store(const TcArgs& a, const TcRow& r, int i, float v, const TcItem& it) {
    if (KIND == kTcTheta) {  // intermediate [item][parent theta i][child phi j][Q]
        a.scr_out[((static_cast<size_t>(r.b) * a.nth + i) * a.mph + r.j) * a.Q + r.q] = v;
    } else if (KIND == kTcPhi) {  // parent A at (theta j, phi i)
        float* o = reinterpret_cast<float*>(a.pat_out);
        o[(static_cast<size_t>(it.box) * a.nth * a.nph + static_cast<size_t>(r.j) * a.nph + i) * 4 * a.nr + r.q] = v;
    } else if (KIND == kTcPhiT) {  // intermediate [item][parent theta j][child phi i][Q]
        a.scr_out[((static_cast<size_t>(r.b) * a.nth + r.j) * a.mph + i) * a.Q + r.q] = v;
    } else {  // child B at (theta i, phi j), accumulated
        float* o = reinterpret_cast<float*>(a.pat_out);
        o[(static_cast<size_t>(it.box) * a.mth * a.mph + static_cast<size_t>(i) * a.mph + r.j) * 4 * a.nr + r.q] += v;
    }
}

// THETA_T's output (child B at theta i, phi j), read and written separately
// so that a row's loads can all be in flight before its stores.
MLFMA_HD size_t tc_out_index_thetaT(const TcArgs& a, const TcRow& r, int i, const TcItem& it) {
    return (static_cast<size_t>(it.box) * a.mth * a.mph + static_cast<size_t>(i) * a.mph + r.j) * 4 * a.nr + r.q;
}
MLFMA_HD float tc_peek_out(const TcArgs& a, const TcRow& r, int i, const TcItem& it) {
    return reinterpret_cast<const float*>(a.pat_out)[tc_out_index_thetaT(a, r, i, it)];
}
MLFMA_HD void tc_put_out(const TcArgs& a, const TcRow& r, int i, float v, const TcItem& it) {
    reinterpret_cast<float*>(a.pat_out)[tc_out_index_thetaT(a, r, i, it)] = v;
}

// Shared-memory byte offset of the four contraction values [4 kq, 4 kq + 4)
// of tile row m within the staged chunk: K-major without swizzle, core
// matrices of 8 rows x 16 bytes, the chunk's 16-byte K pieces of one 8-row
// group 128 bytes apart (the descriptor's leading offset), 8-row groups
// kc_max * 32 bytes apart (its stride offset; kc_max = the largest chunk).
MLFMA_HD uint32_t tc_a_offset(int m, int kq, int kc_max) {
    return static_cast<uint32_t>((m >> 3) * (kc_max * 32) + kq * 128 + (m & 7) * 16);
}
// Element (output n, contraction k) of a weight matrix with Kpad columns in the
// K-major layout without swizzle: 8-row groups Kpad * 32 bytes apart (stride
// offset), 16-byte K chunks 128 bytes apart (leading offset); as a float index.
MLFMA_HD size_t tc_w_index(int n, int k, int Kpad) {
    return static_cast<size_t>(n / 8) * (Kpad * 8) + (k / 4) * 32 + (n % 8) * 4 + (k % 4);
}

// Bytes of one A tile half (hi or lo): 128 rows x kc_max values, at least
// 16 KB, so that the region exceeds any span an operand descriptor over it
// could cover.
MLFMA_HD size_t tc_a_bytes(int Kpad) {
    const size_t b = static_cast<size_t>(Kpad < kTcKChunk ? Kpad : kTcKChunk) * 512;
    return b > 16384 ? b : 16384;
}
MLFMA_HD size_t tc_w_bytes(int Npad, int Kpad) { return static_cast<size_t>(Npad) * Kpad * 4; }
// Dynamic shared memory of a pass: alignment slack, weights (hi, lo) rounded to
// 1 KB, the A tile (hi, lo), the contraction table.
inline size_t tc_smem_bytes(int Npad, int Kpad, int K) {
    return 1024 + ((2 * tc_w_bytes(Npad, Kpad) + 1023) & ~static_cast<size_t>(1023)) + 2 * tc_a_bytes(Kpad) +
           4 * static_cast<size_t>(K);
}

// ---------------------------------------------------------------- host side

// Round to the nearest TF32 value, ties away from zero (cvt.rna.tf32.f32).
inline float tf32_host(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) != 0x7f800000u) u += 0x1000u;
    u &= 0xffffe000u;
    std::memcpy(&x, &u, 4);
    return x;
}

// Dense weights of one pass from its stencil: rows = outputs, columns =
// contraction indices, the nsrc source rows first, then (theta passes) each
// source row that a tap reads reflected, at phi + pi; the reflection sign is
// folded into the weight.  krow: source row of each column (| kTcShiftFlag).
struct TcDense {
    int N = 0, K = 0;
    std::vector<double> w;
    std::vector<int> krow;
};

inline std::string tc_dense_weights(const Stencil& st, int nsrc, bool theta, TcDense& d) {
    const int rows = static_cast<int>(st.ptr.size()) - 1;
    std::vector<int> refl_rows;
    for (int r = 0; r < rows; ++r)
        for (int q = st.ptr[r]; q < st.ptr[r + 1]; ++q)
            if (st.refl[q]) {
                if (!theta) return "reflected tap in a phi stencil";
                if (std::find(refl_rows.begin(), refl_rows.end(), st.src[q]) == refl_rows.end())
                    refl_rows.push_back(st.src[q]);
            }
    d.N = rows;
    d.K = nsrc + static_cast<int>(refl_rows.size());
    d.w.assign(static_cast<size_t>(d.N) * d.K, 0.0);
    d.krow.resize(d.K);
    for (int i = 0; i < nsrc; ++i) d.krow[i] = i;
    for (size_t t = 0; t < refl_rows.size(); ++t) d.krow[nsrc + t] = refl_rows[t] | kTcShiftFlag;
    for (int r = 0; r < rows; ++r)
        for (int q = st.ptr[r]; q < st.ptr[r + 1]; ++q) {
            int k = st.src[q];
            if (k < 0 || k >= nsrc) return "stencil source out of range";
            if (st.refl[q])
                k = nsrc + static_cast<int>(std::find(refl_rows.begin(), refl_rows.end(), st.src[q]) -
                                            refl_rows.begin());
            d.w[static_cast<size_t>(r) * d.K + k] += st.refl[q] ? -st.coef[q] : st.coef[q];
        }
    return {};
}

// hi then lo halves (w = hi + lo to about 2^-22), each Npad x Kpad, zero padded.
inline std::vector<float> tc_pack_weights(const TcDense& d, int Npad, int Kpad) {
    std::vector<float> out(static_cast<size_t>(2) * Npad * Kpad, 0.f);
    const size_t half = static_cast<size_t>(Npad) * Kpad;
    for (int n = 0; n < d.N; ++n)
        for (int k = 0; k < d.K; ++k) {
            const double w = d.w[static_cast<size_t>(n) * d.K + k];
            const float hi = tf32_host(static_cast<float>(w));
            const float lo = tf32_host(static_cast<float>(w - static_cast<double>(hi)));
            const size_t at = tc_w_index(n, k, Kpad);
            out[at] = hi;
            out[half + at] = lo;
        }
    return out;
}

}  // namespace mlfma
