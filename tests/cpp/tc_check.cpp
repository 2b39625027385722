// CPU check of the tensor-core interpolation passes (kernels_tc.cuh) through
// their shared index arithmetic (tc_plan.hpp): for real plans, every pass's
// dense weights, contraction table, row decomposition, loads and stores are run
// on the CPU exactly as the kernels run them (chunks of items included) and
// compared with a direct application of the stencils in double, in the order
// of the CUDA-core kernels k_m2m / k_l2l (per child: shift, theta pass with
// pole reflection, phi pass; per (parent, child): shift, transposed phi pass,
// transposed theta pass).  Built with AddressSanitizer, so every load and
// store is bounds-checked.  Also checks that the shared-memory layout of every
// pass fits a CTA and that every offset the kernel writes, and every span its
// MMA descriptors cover, stays inside the region it belongs to.
// Run by tests/test_tc_plan.py.
#include "plan.hpp"
#include "tc_plan.hpp"

#include <vector_functions.h>

#include <cmath>
#include <complex>
#include <cstdio>
#include <random>

using namespace mlfma;
using C = std::complex<double>;

static float2 f2(C v) { return make_float2(static_cast<float>(v.real()), static_cast<float>(v.imag())); }
static C cd(float2 v) { return C(v.x, v.y); }

// Effective weight the MMA sees: hi + lo at the canonical position.
static double weff(const std::vector<float>& w, int n, int k, int Npad, int Kpad) {
    const size_t at = tc_w_index(n, k, Kpad);
    return static_cast<double>(w[at]) + static_cast<double>(w[static_cast<size_t>(Npad) * Kpad + at]);
}

// One pass over items [i0, i0 + ni): every row and output, as the kernel's
// threads do (the contraction in double here; on the GPU in FP32 from 3xTF32).
template <int KIND>
static void run_pass(TcArgs a, const std::vector<float>& w, const std::vector<int>& krow) {
    const long long rows = static_cast<long long>(a.J) * a.Q * a.nitems;
    const long long tiles = (rows + kTcRows - 1) / kTcRows;
    for (long long t = 0; t < tiles; ++t)
        for (int m = 0; m < kTcRows; ++m) {
            const TcRow r = tc_row(a, t * kTcRows + m);
            const TcItem it = tc_item<KIND>(a, r);
            std::vector<double> x(a.Kpad);
            for (int k0 = 0; k0 < a.Kpad; k0 += kTcKChunk) {
                const int kc = std::min(kTcKChunk, a.Kpad - k0);
                for (int k = 0; k < kc; ++k) x[k0 + k] = tc_load<KIND>(a, r, k0 + k, krow.data(), it);
            }
            if (!r.live) continue;
            for (int i = 0; i < a.N; ++i) {
                double acc = 0;
                for (int k = 0; k < a.Kpad; ++k) acc += x[k] * weff(w, i, k, a.Npad, a.Kpad);
                tc_store<KIND>(a, r, i, static_cast<float>(acc), it);
            }
        }
}

static int check_layout(const TcDense& d, int Npad, int Kpad, const char* what) {
    const size_t smem = tc_smem_bytes(Npad, Kpad, d.K);
    if (smem > 232448) { printf("%s: shared memory %zu too large\n", what, smem); return 1; }
    const size_t ab = tc_a_bytes(Kpad);
    const int kc = std::min(Kpad, kTcKChunk);
    // every 16-byte piece written once, all inside the tile
    std::vector<int> hit(ab / 16, 0);
    for (int m = 0; m < kTcRows; ++m)
        for (int kq = 0; kq < kc / 4; ++kq) {
            const uint32_t o = tc_a_offset(m, kq, kc);
            if (o % 16 || o + 16 > ab || hit[o / 16]++) {
                printf("%s: A tile piece (%d, %d) at %u outside the tile or written twice\n", what, m, kq, o);
                return 1;
            }
        }
    // an MMA reads K step kk: 16 row groups (stride kc * 32) of two 16-byte
    // pieces (leading offset 128) from kk * 256; with the offsets swapped it
    // would reach 15 * 128 + 128 + kk * 256 + kc * 32 -- both inside the region
    const size_t span1 = static_cast<size_t>(15) * kc * 32 + (kc / 8 - 1) * 256 + 256;
    const size_t span2 = static_cast<size_t>(15) * 128 + (kc / 8 - 1) * 256 + static_cast<size_t>(kc) * 32 + 128;
    if (span1 > ab || span2 > ab) {
        printf("%s: A descriptor spans exceed the tile (%zu, %zu, %zu)\n", what, span1, span2, ab);
        return 1;
    }
    size_t wmax = 0;
    for (int n = 0; n < Npad; ++n)
        for (int k = 0; k < Kpad; ++k) wmax = std::max(wmax, tc_w_index(n, k, Kpad) + 1);
    if (wmax != static_cast<size_t>(Npad) * Kpad) { printf("%s: weight layout not dense\n", what); return 1; }
    return 0;
}

static int run(Plan& p, int nr, size_t scratch_cap, const char* name) {
    std::mt19937 g(7 + nr);
    std::normal_distribution<double> nd;
    int bad = 0;
    double worst = 0;
    for (int pl = p.lmin; pl < p.max_level; ++pl) {
        const Level& PL = p.levels[pl];
        const Level& CL = p.levels[pl + 1];
        const Transition& T = p.trans[pl];
        const int nth = PL.nth, nph = PL.nph, mth = CL.nth, mph = CL.nph, halfm = mph / 2;
        const int npb = static_cast<int>(PL.boxes.size()), ncb = static_cast<int>(CL.boxes.size());
        const int npar = static_cast<int>(T.par_box.size());
        TcDense d[4];
        std::string e;
        if ((e = tc_dense_weights(T.up_th, mth, true, d[0])).size() || (e = tc_dense_weights(T.up_ph, mph, false, d[1])).size() ||
            (e = tc_dense_weights(T.dn_ph, nph, false, d[2])).size() || (e = tc_dense_weights(T.dn_th, nth, true, d[3])).size()) {
            printf("%s: weights: %s\n", name, e.c_str());
            return 1;
        }
        std::vector<float> w[4];
        int Kp[4], Np[4];
        for (int k = 0; k < 4; ++k) {
            Kp[k] = (d[k].K + 7) / 8 * 8;
            Np[k] = (d[k].N + 15) / 16 * 16;
            w[k] = tc_pack_weights(d[k], Np[k], Kp[k]);
            if (check_layout(d[k], Np[k], Kp[k], name)) return 1;
        }
        // patterns and shifts (complex float, [box][dir][2][nr])
        auto rnd = [&](size_t n) { std::vector<float2> v(n); for (auto& x : v) x = make_float2(nd(g), nd(g)); return v; };
        std::vector<float2> Ac = rnd(static_cast<size_t>(ncb) * CL.ndir * 2 * nr);
        std::vector<float2> Bp = rnd(static_cast<size_t>(npb) * PL.ndir * 2 * nr);
        std::vector<float2> Bc0 = rnd(static_cast<size_t>(ncb) * CL.ndir * 2 * nr);
        std::vector<float2> Ap(static_cast<size_t>(npb) * PL.ndir * 2 * nr, make_float2(0, 0));
        std::vector<float2> Bc = Bc0;
        std::vector<float2> shu(CL.shift_up.size()), shd(PL.shift_down.size());
        for (size_t i = 0; i < shu.size(); ++i) shu[i] = f2(CL.shift_up[i]);
        for (size_t i = 0; i < shd.size(); ++i) shd[i] = f2(PL.shift_down[i]);
        std::vector<int2> pairs;
        for (int q = 0; q < npar; ++q)
            for (int c = T.child_ptr[q]; c < T.child_ptr[q + 1]; ++c) pairs.push_back(make_int2(q, c));
        const int npairs = static_cast<int>(pairs.size());
        // ---- reference M2M and L2L (double, stencils as the CUDA-core kernels apply them)
        std::vector<C> Aref(Ap.size(), 0.0), Bref(Bc.size());
        for (size_t i = 0; i < Bc.size(); ++i) Bref[i] = cd(Bc0[i]);
        for (int q = 0; q < npar; ++q)
            for (int c = T.child_ptr[q]; c < T.child_ptr[q + 1]; ++c)
                for (int cq = 0; cq < 2 * nr; ++cq) {
                    std::vector<C> th(static_cast<size_t>(nth) * mph);
                    for (int jt = 0; jt < nth; ++jt)
                        for (int ip = 0; ip < mph; ++ip) {
                            C v = 0;
                            for (int t = T.up_th.ptr[jt]; t < T.up_th.ptr[jt + 1]; ++t) {
                                const bool rf = T.up_th.refl[t];
                                const int sp = rf ? (ip < halfm ? ip + halfm : ip - halfm) : ip;
                                const int dd = T.up_th.src[t] * mph + sp;
                                const double cf = rf ? -T.up_th.coef[t] : T.up_th.coef[t];
                                v += cf * cd(shu[static_cast<size_t>(T.child_oct[c]) * CL.ndir + dd]) *
                                     cd(Ac[(static_cast<size_t>(T.child_box[c]) * CL.ndir + dd) * 2 * nr + cq]);
                            }
                            th[static_cast<size_t>(jt) * mph + ip] = v;
                        }
                    for (int jt = 0; jt < nth; ++jt)
                        for (int jp = 0; jp < nph; ++jp) {
                            C v = 0;
                            for (int t = T.up_ph.ptr[jp]; t < T.up_ph.ptr[jp + 1]; ++t)
                                v += T.up_ph.coef[t] * th[static_cast<size_t>(jt) * mph + T.up_ph.src[t]];
                            Aref[(static_cast<size_t>(T.par_box[q]) * PL.ndir + jt * nph + jp) * 2 * nr + cq] += v;
                        }
                }
        for (const int2 pc : pairs)
            for (int cq = 0; cq < 2 * nr; ++cq) {
                std::vector<C> ph(static_cast<size_t>(nth) * mph);
                for (int it = 0; it < nth; ++it)
                    for (int jp = 0; jp < mph; ++jp) {
                        C v = 0;
                        for (int t = T.dn_ph.ptr[jp]; t < T.dn_ph.ptr[jp + 1]; ++t) {
                            const int dd = it * nph + T.dn_ph.src[t];
                            v += T.dn_ph.coef[t] * cd(shd[static_cast<size_t>(T.child_oct[pc.y]) * PL.ndir + dd]) *
                                 cd(Bp[(static_cast<size_t>(T.par_box[pc.x]) * PL.ndir + dd) * 2 * nr + cq]);
                        }
                        ph[static_cast<size_t>(it) * mph + jp] = v;
                    }
                for (int jt = 0; jt < mth; ++jt)
                    for (int jp = 0; jp < mph; ++jp) {
                        C v = 0;
                        for (int t = T.dn_th.ptr[jt]; t < T.dn_th.ptr[jt + 1]; ++t) {
                            const bool rf = T.dn_th.refl[t];
                            const int sp = rf ? (jp < halfm ? jp + halfm : jp - halfm) : jp;
                            v += (rf ? -T.dn_th.coef[t] : T.dn_th.coef[t]) * ph[static_cast<size_t>(T.dn_th.src[t]) * mph + sp];
                        }
                        Bref[(static_cast<size_t>(T.child_box[pc.y]) * CL.ndir + jt * mph + jp) * 2 * nr + cq] += v;
                    }
            }
        // ---- the tensor-core passes, in chunks of items as the host launches them
        std::vector<float> scr(scratch_cap);
        const size_t per_item = static_cast<size_t>(nth) * mph * 4 * nr;
        auto base = [&](int kind) {
            TcArgs a{};
            a.K = d[kind].K; a.Kpad = Kp[kind]; a.N = d[kind].N; a.Npad = Np[kind];
            a.nr = nr; a.Q = 4 * nr; a.mth = mth; a.mph = mph; a.nth = nth; a.nph = nph;
            a.child_ptr = T.child_ptr.data(); a.child_box = T.child_box.data(); a.child_oct = T.child_oct.data();
            a.par_box = T.par_box.data(); a.pairs = pairs.data();
            a.scr_in = scr.data(); a.scr_out = scr.data();
            return a;
        };
        const int chunk_m = static_cast<int>(std::max<size_t>(1, std::min<size_t>(npar, scratch_cap / per_item)));
        for (int i0 = 0; i0 < npar; i0 += chunk_m) {
            TcArgs a = base(kTcTheta);
            a.item0 = i0; a.nitems = std::min(chunk_m, npar - i0); a.J = mph; a.pat_in = Ac.data(); a.shift = shu.data();
            run_pass<kTcTheta>(a, w[0], d[0].krow);
            TcArgs b = base(kTcPhi);
            b.item0 = i0; b.nitems = a.nitems; b.J = nth; b.pat_out = Ap.data();
            run_pass<kTcPhi>(b, w[1], d[1].krow);
        }
        const int chunk_l = static_cast<int>(std::max<size_t>(1, std::min<size_t>(npairs, scratch_cap / per_item)));
        for (int i0 = 0; i0 < npairs; i0 += chunk_l) {
            TcArgs a = base(kTcPhiT);
            a.item0 = i0; a.nitems = std::min(chunk_l, npairs - i0); a.J = nth; a.pat_in = Bp.data(); a.shift = shd.data();
            run_pass<kTcPhiT>(a, w[2], d[2].krow);
            TcArgs b = base(kTcThetaT);
            b.item0 = i0; b.nitems = a.nitems; b.J = mph; b.pat_out = Bc.data();
            run_pass<kTcThetaT>(b, w[3], d[3].krow);
        }
        double num = 0, den = 0, num2 = 0, den2 = 0;
        for (size_t i = 0; i < Ap.size(); ++i) { num += std::norm(cd(Ap[i]) - Aref[i]); den += std::norm(Aref[i]); }
        for (size_t i = 0; i < Bc.size(); ++i) {
            num2 += std::norm(cd(Bc[i]) - Bref[i]);
            den2 += std::norm(Bref[i] - cd(Bc0[i]));
        }
        const double e1 = std::sqrt(num / den), e2 = std::sqrt(num2 / den2);
        worst = std::max(worst, std::max(e1, e2));
        printf("%s nr=%d transition %d->%d: grids %dx%d -> %dx%d, K %d/%d/%d/%d, M2M err %.2e, L2L err %.2e\n", name,
               nr, pl + 1, pl, mth, mph, nth, nph, d[0].K, d[1].K, d[2].K, d[3].K, e1, e2);
        if (!(e1 < 1e-6) || !(e2 < 1e-6)) bad = 1;
    }
    return bad;
}

int main() {
    int bad = 0;
    {  // dipoles in a 4-wavelength cube, leaves 0.25 wavelength (levels 2-4)
        const int n = 3000;
        std::mt19937 g(3);
        std::uniform_real_distribution<double> u(-1.99, 1.99);
        std::vector<double> pos(3 * n), mom(3 * n);
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) { pos[3 * i + k] = u(g); mom[3 * i + k] = (k == 0); }
        Config cfg; cfg.max_node_srcs = 4; cfg.max_level = 4; cfg.root_leng = 4.0; cfg.ref_compat = 0;
        PlaneWave pw; pw.wavenum = 2 * M_PI;
        Plan p;
        std::string e = p.build_dipoles(cfg, pw, n, pos.data(), mom.data());
        if (!e.empty()) { printf("plan: %s\n", e.c_str()); return 1; }
        bad |= run(p, 1, 1 << 22, "cube4");
        bad |= run(p, 3, 20000, "cube4-chunked");  // small buffer: many chunks
    }
    {  // sources on a sphere of radius 8 in a 16-wavelength root box, leaves
       // 0.25 wavelength (levels 2-6): the grids of the largest benchmark
        const int n = 4000;
        std::mt19937 g(5);
        std::normal_distribution<double> nd;
        std::vector<double> pos(3 * n), mom(3 * n);
        for (int i = 0; i < n; ++i) {
            double v[3] = {nd(g), nd(g), nd(g)};
            const double r = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            for (int k = 0; k < 3; ++k) { pos[3 * i + k] = 7.99 * v[k] / r; mom[3 * i + k] = (k == 1); }
        }
        Config cfg; cfg.max_node_srcs = 1; cfg.max_level = 6; cfg.root_leng = 16.0; cfg.ref_compat = 0;
        PlaneWave pw; pw.wavenum = 2 * M_PI;
        Plan p;
        std::string e = p.build_dipoles(cfg, pw, n, pos.data(), mom.data());
        if (!e.empty()) { printf("plan: %s\n", e.c_str()); return 1; }
        bad |= run(p, 1, 1 << 24, "sphere16");
    }
    if (!bad) printf("ALL OK\n");
    return bad;
}
