// CPU check of the near-field tiling (Plan::build_near_plan, plan.cpp) and of
// the index arithmetic the near-field kernels apply to it (kernels_near.cuh):
// k_near_blocks_assemble's decoding of packed self blocks, k_near_sym's bulk
// copies (source and destination ranges, expected byte counts), its row and
// column sums over the stage, the partial slots, and k_near_reduce's sums per
// target.  Every stored entry must land in exactly one tile, every read must hit
// a copied value, every partial must be written once, and the result must equal
// the block-row form (each leaf's rows against all the sources it meets) on a
// symmetric synthetic entry.  Run by tests/test_near_tiles.py.
#include "plan.hpp"
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <random>
using namespace mlfma;
using C = std::complex<double>;
// A symmetric synthetic near-field entry (diagonal distinct).
static C f(int m, int n) {
    const double a = m + n, b = double(m) * n;
    return C(std::cos(0.37 * a + 1e-3 * b), std::sin(0.11 * a - 2e-4 * b)) * (m == n ? 5.0 : 1.0);
}
static long long prow(int i, int kind) { return kind == 1 ? (long long)i * (i - 1) / 2 : (long long)i * (i + 1) / 2; }
// n dipoles, half of them in a small ball (uneven leaves, list-3/4 pairs),
// boxes split above maxsrc sources.
int run(int n, int maxsrc, int self_terms, double side, int seed) {
    std::mt19937 g(seed);
    std::uniform_real_distribution<double> u(-side / 2 * 0.999, side / 2 * 0.999);
    std::vector<double> pos(3 * n), mom(3 * n);
    for (int i = 0; i < n; ++i) {
        // clustered: half the sources in a small ball (uneven leaves, list 3/4)
        const double s = (i % 2) ? 1.0 : 0.1;
        for (int k = 0; k < 3; ++k) { pos[3 * i + k] = u(g) * s; mom[3 * i + k] = (k == 0); }
    }
    Config cfg; cfg.max_node_srcs = maxsrc; cfg.root_leng = side; cfg.self_terms = self_terms; cfg.ref_compat = 0;
    PlaneWave pw; pw.wavenum = 2 * M_PI;
    Plan p;
    std::string e = p.build_dipoles(cfg, pw, n, pos.data(), mom.data());
    if (!e.empty()) { printf("plan error %s\n", e.c_str()); return 1; }
    // assemble (decode as k_near_blocks_assemble)
    std::vector<C> Z(p.near_entries);
    std::vector<int> kinds;
    for (auto& b : p.near_blocks) kinds.push_back(b.self ? (self_terms ? 2 : 1) : 0);
    for (long long e2 = 0; e2 < p.near_entries; ++e2) {
        int lo = 0, hi = (int)p.near_blocks.size() - 1;
        while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (p.near_blocks[mid].off <= e2) lo = mid; else hi = mid - 1; }
        const NearBlock& B = p.near_blocks[lo]; const int kind = kinds[lo];
        long long loc = e2 - B.off; int i, j;
        if (kind == 0) { i = loc / B.ncol; j = loc - (long long)i * B.ncol; }
        else {
            double q = std::sqrt(1.0 + 8.0 * (double)loc);
            i = (int)(kind == 1 ? (1.0 + q) * 0.5 : (q - 1.0) * 0.5);
            while (i > 0 && prow(i, kind) > loc) --i;
            while (prow(i + 1, kind) <= loc) ++i;
            j = loc - prow(i, kind);
            if (!(kind == 1 ? j < i : j <= i)) { printf("bad self decode\n"); return 1; }
        }
        if (i < 0 || i >= B.nrow || j < 0 || j >= B.ncol) { printf("decode out of block\n"); return 1; }
        Z[e2] = f(B.row0 + i, B.col0 + j);
    }
    std::vector<C> x(n);
    for (int i = 0; i < n; ++i) x[i] = C(std::sin(1.3 * i), std::cos(0.7 * i));
    std::vector<C> part(p.near_parts, C(0));
    std::vector<int> written(p.near_parts, 0);
    const int XC = kNearTileEntries, XR = XC + kNearTileCols, SL = XR + kNearTileRows;
    const int SE = SL + (kNearTileRows + kNearTileCols) * 4 / 16;
    std::vector<C> st(SE); std::vector<char> ok(SE); std::vector<int> slotmem(kNearTileRows + kNearTileCols); std::vector<char> slotok(kNearTileRows + kNearTileCols);
    auto rowlen = [&](const NearTile& T, int r) { if (T.kind == 0) return T.nj; return std::max(0, std::min(T.nj, T.i0 + r + (T.kind == 2 ? 1 : 0) - T.j0)); };
    auto rowstart = [&](const NearTile& T, int r) { return T.mode == 1 ? (int)(prow(T.i0 + r, T.kind) - prow(T.i0, T.kind)) : r * T.nj; };
    auto colstart = [&](const NearTile& T, int c) { return T.kind == 0 ? 0 : std::max(0, T.j0 + c - T.i0 + 1); };
    int modes[3] = {0, 0, 0}; long long tile_entries_sum = 0;
    for (const NearTile& T : p.near_tiles) {
        modes[T.mode]++;
        if (T.ni < 1 || T.nj < 1 || T.ni > kNearTileRows || T.nj > kNearTileCols) { printf("tile size\n"); return 1; }
        if (T.mode == 2 && T.ni > kNearTileRowsSplit) { printf("mode 2 rows\n"); return 1; }
        if (T.slot % 4) { printf("slot align\n"); return 1; }
        std::fill(ok.begin(), ok.end(), 0); std::fill(slotok.begin(), slotok.end(), 0);
        long long total = 0, copied = 0;
        if (T.mode == 2) {
            for (int lane = 0; lane < T.ni; ++lane) {
                const int il = T.i0 + lane, nv = rowlen(T, lane);
                const long long off = T.z + (T.kind == 0 ? (long long)il * T.ld : prow(il, T.kind)) + T.j0;
                total += nv;
                for (int j = 0; j < nv; ++j) {
                    if (off + j < 0 || off + j >= p.near_entries) { printf("copy src out of range\n"); return 1; }
                    const int d = lane * T.nj + j; if (d >= XC) { printf("dst\n"); return 1; }
                    st[d] = Z[off + j]; ok[d] = 1; copied++;
                }
            }
        } else {
            total = T.mode == 0 ? T.ni * T.nj : prow(T.i0 + T.ni, T.kind) - prow(T.i0, T.kind);
            if (total > kNearTileEntries || total <= 0) { printf("tile entries %lld\n", total); return 1; }
            for (long long e2 = 0; e2 < total; ++e2) {
                if (T.z + e2 >= p.near_entries) { printf("span out of range\n"); return 1; }
                st[e2] = Z[T.z + e2]; ok[e2] = 1; copied++;
            }
            // every row's entries lie in the span
            for (int r = 0; r < T.ni; ++r) if (rowstart(T, r) + rowlen(T, r) > total) { printf("row past span\n"); return 1; }
            if (T.mode == 1 && rowlen(T, T.ni - 1) != T.nj) { printf("mode 1 nj\n"); return 1; }
        }
        tile_entries_sum += total;
        const int nslot = (T.ni + T.nj + 3) & ~3;
        if (T.c0 + T.j0 + T.nj > n || T.r0 + T.i0 + T.ni > n) { printf("x copy range\n"); return 1; }
        if (T.slot + nslot > (int)p.near_slot.size()) { printf("slot copy range\n"); return 1; }
        for (int j = 0; j < T.nj; ++j) { st[XC + j] = x[T.c0 + T.j0 + j]; ok[XC + j] = 1; }
        for (int i = 0; i < T.ni; ++i) { st[XR + i] = x[T.r0 + T.i0 + i]; ok[XR + i] = 1; }
        for (int q = 0; q < nslot; ++q) { slotmem[q] = p.near_slot[T.slot + q]; slotok[q] = 1; }
        if (total != copied || (total + T.ni + T.nj) * 16 + nslot * 4 >= (1 << 20)) { printf("tx bytes\n"); return 1; }
        auto rd = [&](int a) -> C { if (a < 0 || a >= SE || !ok[a]) { printf("read of uncopied slot %d\n", a); exit(1); } return st[a]; };
        auto rs = [&](int a) -> int { if (!slotok[a]) { printf("slot read\n"); exit(1); } return slotmem[a]; };
        // k_near_sym's consumers: G adjacent lanes per row (column), each a
        // segment; the lane with h == 0 writes the group's sum
        C gsum[128]; int myslot[128];
        for (int ct = 0; ct < 128; ++ct) {
            myslot[ct] = -1;
            C a(0);
            if (ct < 64) {
                const int G = T.ni <= 8 ? 8 : T.ni <= 16 ? 4 : T.ni <= 32 ? 2 : 1;
                const int r = ct / G, h = ct & (G - 1);
                if (r < T.ni) {
                    const int len = rowlen(T, r);
                    const int seg = (len + G - 1) / G;
                    const int k0 = std::min(len, h * seg), k1 = std::min(len, k0 + seg), L = k1 - k0;
                    int q = (T.mode != 1 && !(T.nj & 1) && L > 0) ? r % L : 0;
                    for (int m = 0; m < L; ++m) { a += rd(rowstart(T, r) + k0 + q) * rd(XC + k0 + q); if (++q == L) q = 0; }
                    if (h == 0) myslot[ct] = rs(r);
                }
            } else {
                const int cc = ct - 64;
                const int G = T.nj <= 8 ? 8 : T.nj <= 16 ? 4 : T.nj <= 32 ? 2 : 1;
                const int c = cc / G, h = cc & (G - 1);
                if (c < T.nj) {
                    const int r0s = colstart(T, c);
                    const int seg = (std::max(0, T.ni - r0s) + G - 1) / G;
                    const int ra = std::min(T.ni, r0s + h * seg), rb = std::min(T.ni, ra + seg);
                    for (int r = ra; r < rb; ++r) a += rd(rowstart(T, r) + c) * rd(XR + r);
                    if (h == 0) myslot[ct] = rs(T.ni + c);
                }
            }
            gsum[ct] = a;
        }
        for (int ct = 0; ct < 128; ++ct) {
            if (myslot[ct] < 0) continue;
            if (myslot[ct] >= p.near_parts) { printf("slot value range\n"); return 1; }
            const int G = ct < 64 ? (T.ni <= 8 ? 8 : T.ni <= 16 ? 4 : T.ni <= 32 ? 2 : 1)
                                  : (T.nj <= 8 ? 8 : T.nj <= 16 ? 4 : T.nj <= 32 ? 2 : 1);
            C a(0);
            for (int h = 0; h < G; ++h) a += gsum[ct + h];  // the group's lanes
            part[myslot[ct]] = a;
            written[myslot[ct]]++;
        }
    }
    if (tile_entries_sum != p.near_entries) { printf("tiles hold %lld of %lld entries\n", tile_entries_sum, p.near_entries); return 1; }
    printf("  modes %d %d %d\n", modes[0], modes[1], modes[2]);
    for (int q = 0; q < p.near_parts; ++q) if (written[q] != 1) { printf("partial %d written %d times\n", q, written[q]); return 1; }
    std::vector<C> y(n);
    for (int t = 0; t < n; ++t) { C a(0); for (int q = p.near_red_ptr[t]; q < p.near_red_ptr[t + 1]; ++q) a += part[q]; y[t] = a; }
    // block-row form
    double err = 0, nrm = 0;
    for (const NearRow& r : p.near_rows)
        for (int i = 0; i < r.nrow; ++i) {
            C a(0);
            for (int k = 0; k < r.ncol; ++k) {
                const int c = p.near_cols[r.col_off + k];
                C v = f(r.row0 + i, c);
                if (c == r.row0 + i && !self_terms) v = 0;
                a += v * x[c];
            }
            err = std::max(err, std::abs(a - y[r.row0 + i])); nrm = std::max(nrm, std::abs(a));
        }
    size_t maxnc = 0;
    for (auto& b : p.near_blocks) { maxnc = std::max<size_t>(maxnc, b.ncol); }
    printf("n=%d maxsrc=%d self=%d blocks=%zu tiles=%zu parts=%d entries=%lld row_entries=%lld maxncol=%zu err=%.3g (|y| %.3g)\n",
           n, maxsrc, self_terms, p.near_blocks.size(), p.near_tiles.size(), p.near_parts, p.near_entries,
           p.near_row_entries, maxnc, err, nrm);
    return err > 1e-9 * nrm ? 1 : 0;
}
int main() {
    int bad = 0;
    bad |= run(3000, 16, 0, 4.0, 1);
    bad |= run(3000, 16, 1, 4.0, 2);
    bad |= run(5000, 150, 1, 4.0, 3);
    bad |= run(5000, 100, 0, 4.0, 4);
    bad |= run(40, 64, 1, 0.5, 5);
    bad |= run(1, 64, 1, 0.5, 6);
    bad |= run(2, 64, 0, 0.5, 7);
    printf(bad ? "FAIL\n" : "ALL OK\n");
    return bad;
}
