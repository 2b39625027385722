// Host setup of the MLFMA operator.  See plan.hpp.
#include "plan.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <deque>
#include <thread>
#include <functional>
#include <limits>
#include <stdexcept>
#include <unordered_map>

namespace mlfma {

namespace {

// ------------------------------------------------------------ special functions
// P_n(x) and P_n'(x) by the three-term recurrence (Math::legendreP, src/math.cpp:25-42).
void legendre_p(double x, int n, double* p, double* dp) {
    double pnm = 1.0;
    if (!n) { *p = pnm; *dp = 0.0; return; }
    double pn = x;
    for (int i = 1; i < n; ++i) {
        const double pnp = ((2.0 * i + 1) * x * pn - i * pnm) / static_cast<double>(i + 1);
        pnm = pn;
        pn = pnp;
    }
    *p = pn;
    *dp = n * (x * pn - pnm) / (x * x - 1.0);
}

// Gauss-Legendre nodes/weights on [a,b] by Newton iteration from Chebyshev-like
// guesses, stopping when the step is <= eps; the weight uses P' from the last
// evaluation (Interp::gaussLegendre, src/interp.cpp:12-52).
void gauss_legendre(int l, double eps, double a, double b, std::vector<double>& nodes,
                    std::vector<double>& weights) {
    const double leng = b - a, mid = (a + b) / 2.0;
    nodes.assign(l, 0.0);
    weights.assign(l, 0.0);
    const int kmax = l / 2;
    if (l % 2) {
        nodes[kmax] = mid;
        double p, dp;
        legendre_p(0.0, l, &p, &dp);
        weights[kmax] = leng / (dp * dp);
    }
    for (int k = 0; k < kmax; ++k) {
        double xk = std::cos(kPi * (4.0 * (kmax - k) - 1) / (4.0 * l + 2.0));
        double dpk;
        for (int it = 0;; ++it) {
            double p, dp;
            legendre_p(xk, l, &p, &dp);
            xk -= p / dp;
            if (std::fabs(p / dp) <= eps || it > 200) { dpk = dp; break; }
        }
        const int kplus = l % 2 ? kmax + 1 + k : kmax + k;
        const int kminus = kmax - 1 - k;
        nodes[kplus] = leng / 2.0 * xk + mid;
        nodes[kminus] = -leng / 2.0 * xk + mid;
        weights[kplus] = leng / ((1.0 - xk * xk) * dpk * dpk);
        weights[kminus] = weights[kplus];
    }
}

// Index of the order-m Gauss-Legendre node nearest below x on [a,b]
// (Interp::getNearGLNodeIdx, src/interp.cpp:63-77).
int near_gl_node_idx(double xi, int m, double a, double b) {
    const double leng = b - a, mid = (a + b) / 2.0;
    const double x = 2.0 * (xi - mid) / leng;
    return static_cast<int>(m - std::floor(((4.0 * m + 2.0) * std::acos(x) / kPi + 1.0) / 4.0) - 1);
}

// Lagrange basis polynomial k on nodes xs at x (Interp::evalLagrangeBasis, src/interp.cpp:86-100).
double lagrange(double x, const double* xs, int n, int k) {
    double prod = 1.0;
    for (int j = 0; j < n; ++j) {
        if (j == k) continue;
        prod *= (x - xs[j]) / (xs[k] - xs[j]);
    }
    return prod;
}

// One reflection into [0,size) (Math::flipIdxToRange, src/math.h:144-154).
int flip_idx(int i, int size) {
    if (i < 0) return -i - 1;
    if (i >= size) return 2 * size - i - 1;
    return i;
}
// One period into [0,size) (Math::wrapIdxToRange, src/math.h:156-166).
int wrap_idx(int i, int size) {
    if (i < 0) return i + size;
    if (i >= size) return i - size;
    return i;
}

// h_n^(1)(x) for n = 0..nmax by upward recurrence (Math::sphericalHankel1,
// src/math.cpp:66-81); the n-th value equals the reference's call with order n.
void spherical_hankel1_all(double x, int nmax, std::vector<cplx>& h) {
    const cplx iu(0, 1);
    h.assign(nmax + 1, cplx(0));
    cplx hnm = -iu * std::exp(iu * x) / x;
    h[0] = hnm;
    if (nmax == 0) return;
    cplx hn = -std::exp(iu * x) * (1.0 / x + iu / (x * x));
    h[1] = hn;
    for (int i = 1; i < nmax; ++i) {
        const cplx hnp = (2.0 * i + 1.0) / x * hn - hnm;
        hnm = hn;
        hn = hnp;
        h[i + 1] = hn;
    }
}

// P_l(x) for l = 0..lmax (same recurrence as legendre_p, value only).
void legendre_all(double x, int lmax, std::vector<double>& P) {
    P.assign(lmax + 1, 0.0);
    P[0] = 1.0;
    if (lmax == 0) return;
    double pnm = 1.0, pn = x;
    P[1] = pn;
    for (int i = 1; i < lmax; ++i) {
        const double pnp = ((2.0 * i + 1) * x * pn - i * pnm) / static_cast<double>(i + 1);
        pnm = pn;
        pn = pnp;
        P[i + 1] = pn;
    }
}

cplx pow_i(int m) {  // Math::powI, src/math.h:26-33
    switch (m % 4) {
        case 0: return 1.0;
        case 1: return cplx(0, 1);
        case 2: return -1.0;
        default: return cplx(0, -1);
    }
}

// Reference direction order (FMM::Dir, src/fmm/fmm.h:13-17) as (dx, dy, dz).
const int kDirs[26][3] = {
    {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1},
    {-1, -1, 0}, {1, -1, 0}, {-1, 1, 0}, {1, 1, 0},
    {-1, 0, -1}, {1, 0, -1}, {-1, 0, 1}, {1, 0, 1},
    {0, -1, -1}, {0, 1, -1}, {0, -1, 1}, {0, 1, 1},
    {-1, -1, -1}, {1, -1, -1}, {-1, 1, -1}, {1, 1, -1},
    {-1, -1, 1}, {1, -1, 1}, {-1, 1, 1}, {1, 1, 1}};

// Triangle quadrature rules in barycentric form (Triangle::buildQuads,
// src/sources/triangle.cpp:45-130): rows of (w0, w1, w2, weight).
void quad_rule(int prec, std::vector<double>& rule) {
    rule.clear();
    auto add = [&](double a, double b, double c, double w) { rule.insert(rule.end(), {a, b, c, w}); };
    switch (prec) {
        case 0:
            add(-1, -1, -1, 0.5);  // centroid
            break;
        case 1: {
            const double w = 1.0 / 6.0;
            add(2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0, w);
            add(1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0, w);
            add(1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0, w);
            break;
        }
        case 2: {
            add(-1, -1, -1, 0.1125);
            const double w1 = 0.066197076394253, a = 0.059715871789770, b = 0.470142064105115;
            add(a, b, b, w1); add(b, a, b, w1); add(b, b, a, w1);
            const double w2 = 0.0629695902724135, g = 0.797426985353087, d = 0.101286507323456;
            add(g, d, d, w2); add(d, g, d, w2); add(d, d, g, w2);
            break;
        }
        case 3: {
            add(-1, -1, -1, -0.074785022233841);
            const double w1 = 0.087807628716604, a = 0.479308067841920, b = 0.260345966079040;
            add(a, b, b, w1); add(b, a, b, w1); add(b, b, a, w1);
            const double w2 = 0.026673617804419, g = 0.869739794195568, d = 0.065130102902216;
            add(g, d, d, w2); add(d, g, d, w2); add(d, d, g, w2);
            const double w3 = 0.0385568804451285, e = 0.048690315425316, z = 0.312865496004874,
                         t = 0.638444188569810;
            add(e, z, t, w3); add(t, e, z, w3); add(z, t, e, w3);
            add(e, t, z, w3); add(z, e, t, w3); add(t, z, e, w3);
            break;
        }
        default:
            throw std::runtime_error("quad_prec must be 0..3");
    }
}

double dot3_seq(const double* a, const double* b) {
    // ((0 + a0 b0) + a1 b1) + a2 b2: the accumulation order of a 3-vector dot.
    double s = 0.0;
    for (int i = 0; i < 3; ++i) s += a[i] * b[i];
    return s;
}

}  // namespace

const int* plan_directions() { return &kDirs[0][0]; }

// Weak, so that host-only programs built from this file alone still link; the
// CUDA library defines it.
std::string build_tree_lists_device(Plan& P, const std::vector<double>& centers) __attribute__((weak));

// I(k) of one RWG in the closed form of RWG::getIntegratedPlaneWave
// (src/sources/rwg.cpp:46-86), written operation for operation with
// std::complex<double> so that, built without floating-point contraction,
// it rounds exactly as the reference does.  The closed form cancels badly
// when alpha, beta or gamma is small ((1 - e^{ia})/a^2 and the like), so any
// other evaluation order differs from the reference well above 1e-10.
void rwg_integral_exact(const RwgGeom& g, const TriGeom* tris, const double* kvec, cplx* out) {
    const cplx iu(0, 1);
    cplx rad[3] = {cplx(0), cplx(0), cplx(0)};
    for (int t = 0; t < 2; ++t) {
        const TriGeom& T = tris[g.tri[t]];
        const double alpha = dot3_seq(kvec, T.D0);
        const double beta = -dot3_seq(kvec, T.D2);
        const double gamma = alpha - beta;
        const double alphasq = alpha * alpha, betasq = beta * beta;
        const cplx expI_alpha = std::exp(iu * alpha), expI_beta = std::exp(iu * beta);
        const cplx f0_alpha = approx_zero(alpha) ? -iu : (1.0 - expI_alpha) / alpha;
        const cplx f0_beta = approx_zero(beta) ? -iu : (1.0 - expI_beta) / beta;
        const cplx f1_alpha = approx_zero(alpha) ? cplx(-0.5) : (1.0 - (1.0 - iu * alpha) * expI_alpha) / alphasq;
        const cplx f1_beta = approx_zero(beta) ? cplx(-0.5) : (1.0 - (1.0 - iu * beta) * expI_beta) / betasq;
        cplx radVec[3];
        if (approx_zero(gamma)) {
            const cplx f2 = (expI_alpha * (alphasq + 2.0 * iu * alpha - 2.0) + 2.0) / (2.0 * alpha * alphasq);
            for (int c = 0; c < 3; ++c)
                radVec[c] = -f1_alpha * (T.X0[c] - g.xpm[t][c]) - iu * f2 * (T.D0[c] - T.D2[c]);
        } else {
            const cplx I0 = (f0_alpha - f0_beta) / gamma;
            const cplx I1 = iu * (I0 + f1_alpha);
            const cplx I2 = -iu * (I0 + f1_beta);
            for (int c = 0; c < 3; ++c)
                radVec[c] = I0 * (T.X0[c] - g.xpm[t][c]) + (I1 * T.D0[c] - I2 * T.D2[c]) / gamma;
        }
        const cplx ph = std::exp(iu * dot3_seq(kvec, T.X0));
        const double sgn = t ? -1.0 : 1.0;
        for (int c = 0; c < 3; ++c) rad[c] += ph * radVec[c] * sgn;
    }
    for (int c = 0; c < 3; ++c) out[c] = g.leng * rad[c];
}

void Plan::rwg_patterns_host(std::vector<cplx>& pat) const {
    pat.assign(static_cast<size_t>(pat_elems) * 2, cplx(0));
    const int nthreads = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::atomic<int> next{0};
    auto work = [&]() {
        for (int i = next++; i < static_cast<int>(far_leaves.size()); i = next++) {
            const FarLeaf& f = far_leaves[i];
            const Level& L = levels[f.level];
            const Node& nd = nodes[L.boxes[f.box]];
            const cplx iu(0, 1);
            for (int d = 0; d < L.ndir; ++d) {
                // kvec = khat * wavenum (Leaf::buildRadPats, src/fmm/leaf.cpp:194)
                const double kv[3] = {L.khat[3 * d] * pw.wavenum, L.khat[3 * d + 1] * pw.wavenum,
                                      L.khat[3 * d + 2] * pw.wavenum};
                const cplx ph = std::exp(iu * dot3_seq(kv, nd.center));
                const double* T = &L.thph[6 * d];
                for (int s = 0; s < f.nsrc; ++s) {
                    cplx I[3];
                    rwg_integral_exact(rwg[f.src0 + s], tris.data(), kv, I);
                    // RWG::getRadAlongDir (rwg.h:23-25), then the 2x3 projection.
                    cplx v[3];
                    for (int c = 0; c < 3; ++c) v[c] = ph * std::conj(I[c]);
                    cplx o[2];
                    for (int r = 0; r < 2; ++r) {
                        cplx acc(0);
                        for (int c = 0; c < 3; ++c) acc += T[3 * r + c] * v[c];
                        o[r] = acc;
                    }
                    const size_t at = (static_cast<size_t>(f.pat_off) + static_cast<size_t>(s) * L.ndir + d) * 2;
                    pat[at] = o[0];
                    pat[at + 1] = o[1];
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; ++t) pool.emplace_back(work);
    for (auto& th : pool) th.join();
}

int offset_id(int dx, int dy, int dz) {
    static int table[7][7][7];
    static bool init = false;
    if (!init) {
        int idx = 0;
        for (int z = -3; z <= 3; ++z)
            for (int y = -3; y <= 3; ++y)
                for (int x = -3; x <= 3; ++x) {
                    const int inf = std::max({std::abs(x), std::abs(y), std::abs(z)});
                    table[z + 3][y + 3][x + 3] = inf > 1 ? idx++ : -1;
                }
        init = true;
    }
    if (std::abs(dx) > 3 || std::abs(dy) > 3 || std::abs(dz) > 3) return -1;
    return table[dz + 3][dy + 3][dx + 3];
}

// ---------------------------------------------------------------- sources

std::string Plan::build_dipoles(const Config& c, const PlaneWave& p, int n_, const double* pos,
                                const double* mom) {
    kind = kDipole;
    cfg = c;
    pw = p;
    n = n_;
    if (n <= 0) return "no sources";
    std::vector<double> centers(pos, pos + 3 * static_cast<size_t>(n));
    std::string err = build_common(centers);
    if (!err.empty()) return err;
    dip_pos.resize(3 * static_cast<size_t>(n));
    dip_phat.resize(3 * static_cast<size_t>(n));
    for (int t = 0; t < n; ++t) {
        const int s = perm[t];
        const double* P = mom + 3 * s;
        const double pm = std::sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2]);
        if (!(pm > 0)) return "dipole moment must be non-zero";
        for (int k = 0; k < 3; ++k) {
            dip_pos[3 * t + k] = pos[3 * s + k];
            dip_phat[3 * t + k] = P[k] / pm;  // Dipole ctor, src/sources/dipole.h:21-24
        }
    }
    dip_mom.assign(mom, mom + 3 * static_cast<size_t>(n));
    return {};
}

std::string Plan::build_rwg(const Config& c, const PlaneWave& p, int nv, const double* verts, int nf,
                            const int* faces, int ne, const int* rwgs) {
    kind = kRwg;
    cfg = c;
    pw = p;
    n = ne;
    if (ne <= 0 || nf <= 0 || nv <= 0) return "empty mesh";
    std::vector<double> rule;
    try { quad_rule(cfg.quad_prec, rule); } catch (const std::exception& e) { return e.what(); }
    nq = static_cast<int>(rule.size() / 4);
    quad_w.resize(nq);
    for (int q = 0; q < nq; ++q) quad_w[q] = rule[4 * q + 3];
    // Triangles (Triangle ctor, src/sources/triangle.cpp:5-21).
    tris.resize(nf);
    tri_quad.resize(static_cast<size_t>(nf) * nq * 3);
    tri_v.resize(static_cast<size_t>(nf) * 3);
    tri_p.resize(static_cast<size_t>(nf) * 9);
    for (int f = 0; f < nf; ++f) {
        const double* X[3];
        for (int v = 0; v < 3; ++v) {
            const int vi = faces[3 * f + v];
            if (vi < 0 || vi >= nv) return "face vertex index out of range";
            X[v] = verts + 3 * vi;
            tri_v[3 * f + v] = vi;
            for (int k = 0; k < 3; ++k) tri_p[9 * f + 3 * v + k] = X[v][k];
        }
        TriGeom& T = tris[f];
        double cen[3];
        for (int k = 0; k < 3; ++k) {
            T.X0[k] = X[0][k];
            T.D0[k] = X[1][k] - X[0][k];
            T.D2[k] = X[0][k] - X[2][k];
            cen[k] = (X[0][k] + X[1][k] + X[2][k]) / 3.0;
        }
        for (int q = 0; q < nq; ++q) {
            double* out = &tri_quad[(static_cast<size_t>(f) * nq + q) * 3];
            if (rule[4 * q] < 0) {
                for (int k = 0; k < 3; ++k) out[k] = cen[k];
            } else {
                for (int k = 0; k < 3; ++k)
                    out[k] = rule[4 * q] * X[0][k] + rule[4 * q + 1] * X[1][k] + rule[4 * q + 2] * X[2][k];
            }
        }
    }
    // RWGs (RWG ctor, src/sources/rwg.cpp:3-26).
    std::vector<RwgGeom> g(ne);
    std::vector<double> centers(3 * static_cast<size_t>(ne));
    for (int e = 0; e < ne; ++e) {
        const int* r = rwgs + 4 * e;
        for (int k = 0; k < 2; ++k)
            if (r[k] < 0 || r[k] >= nv) return "rwg vertex index out of range";
        for (int k = 2; k < 4; ++k)
            if (r[k] < 0 || r[k] >= nf) return "rwg triangle index out of range";
        RwgGeom& G = g[e];
        const double* X0 = verts + 3 * r[0];
        const double* X1 = verts + 3 * r[1];
        double d2 = 0;
        for (int k = 0; k < 3; ++k) {
            G.center[k] = (X0[k] + X1[k]) / 2.0;
            d2 += (X0[k] - X1[k]) * (X0[k] - X1[k]);
            centers[3 * e + k] = G.center[k];
        }
        G.leng = std::sqrt(d2);
        G.tri[0] = r[2];
        G.tri[1] = r[3];
        for (int t = 0; t < 2; ++t) {
            bool found = false;
            for (int v = 0; v < 3; ++v) {
                const int vi = faces[3 * r[2 + t] + v];
                if (vi != r[0] && vi != r[1]) {
                    for (int k = 0; k < 3; ++k) G.xpm[t][k] = verts[3 * vi + k];
                    found = true;
                }
            }
            if (!found) return "rwg triangle does not have a free vertex";
        }
    }
    std::string err = build_common(centers);
    if (!err.empty()) return err;
    rwg.resize(ne);
    for (int t = 0; t < ne; ++t) rwg[t] = g[perm[t]];
    return {};
}

void Plan::rhs(cplx* b) const { rhs_for(pw, b); }

void Plan::rhs_for(const PlaneWave& pw, cplx* b) const {
    const cplx iu(0, 1);
    const double* kin = pw.khat;
    double kvec[3] = {pw.wavenum * kin[0], pw.wavenum * kin[1], pw.wavenum * kin[2]};
    for (int t = 0; t < n; ++t) {
        cplx V;
        if (kind == kDipole) {
            // Dipole::buildVoltage, src/sources/dipole.h:29-32.  The reference
            // evaluates it inside the delegated constructor, before the given
            // moment replaces the default (Phys::p0, 0, 0) (dipole.h:10-24), so
            // in reference-compatible mode the voltage uses that default moment.
            const int s = perm[t];
            const double p0[3] = {1.0E-8, 0.0, 0.0};  // Phys::p0, src/phys.h:8
            const double* P = cfg.ref_compat ? p0 : &dip_mom[3 * s];
            const double* r = &dip_pos[3 * t];
            V = -pw.amplitude * std::exp(iu * dot3(kvec, r)) * dot3(P, pw.pol);
        } else {
            // RWG::buildVoltage, src/sources/rwg.h:18-21: -amp conj(I . pol), the
            // dot conjugating I.
            cplx I[3];
            const double wv[3] = {pw.wavenum * kin[0], pw.wavenum * kin[1], pw.wavenum * kin[2]};
            rwg_integral_exact(rwg[t], tris.data(), wv, I);
            cplx s(0);
            for (int k = 0; k < 3; ++k) s += std::conj(I[k]) * pw.pol[k];
            V = -pw.amplitude * std::conj(s);
        }
        b[perm[t]] = -V;
    }
}

// ---------------------------------------------------------------- tree

std::string Plan::build_common(const std::vector<double>& centers) {
    if (!(cfg.root_leng > 0)) return "root_leng must be positive";
    if (cfg.max_node_srcs < 1) return "max_node_srcs must be >= 1";
    if (cfg.interp_order < 1) return "interp_order must be >= 1";
    if (cfg.digits < 1) return "digits must be >= 1";
    if (!(pw.wavenum > 0)) return "wavenumber must be positive";
    const double h = cfg.root_leng / 2.0;
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k)
            if (!(std::fabs(centers[3 * i + k]) <= h)) return "source outside the root box";
    bool host_tree = true;
    if (cfg.device_tree) {
        if (!&build_tree_lists_device) return "device_tree needs the CUDA library";
        const std::string e = build_tree_lists_device(*this, centers);
        if (e.empty()) host_tree = false;
        else if (e.rfind("host:", 0) != 0) return e;
    }
    if (host_tree) {
        build_tree(centers);
        build_lists();
    }
    build_levels();
    build_far_plan();
    build_near_plan();
    return {};
}

// Octree by recursive bucketing: a box with more than max_node_srcs sources
// splits into 8 children by the strict test src > centre per axis, keeping the
// input order inside each child (Stem ctor, src/fmm/stem.cpp:3-26; node
// geometry from the Node ctor, src/fmm/node.cpp:33-44).
void Plan::build_tree(const std::vector<double>& centers) {
    nodes.clear();
    perm.clear();
    leaves.clear();
    max_level = 0;
    const int hard_cap = 30;
    std::function<int(std::vector<int>&&, int, int, int)> make =
        [&](std::vector<int>&& srcs, int level, int parent, int branch) -> int {
        const int id = static_cast<int>(nodes.size());
        nodes.emplace_back();
        {
            Node& nd = nodes[id];
            nd.level = level;
            nd.parent = parent;
            nd.branch = branch;
            if (parent < 0) {
                nd.leng = cfg.root_leng;
            } else {
                const Node& P = nodes[parent];
                nd.leng = P.leng / 2.0;
                const double pm[3] = {(branch & 1) ? 1.0 : -1.0, (branch & 2) ? 1.0 : -1.0,
                                      (branch & 4) ? 1.0 : -1.0};
                for (int k = 0; k < 3; ++k) nd.center[k] = P.center[k] + nd.leng / 2.0 * pm[k];
                nd.ix = 2 * P.ix + (branch & 1);
                nd.iy = 2 * P.iy + ((branch >> 1) & 1);
                nd.iz = 2 * P.iz + ((branch >> 2) & 1);
            }
        }
        const bool split = static_cast<int>(srcs.size()) > cfg.max_node_srcs &&
                           (cfg.max_level <= 0 || level < cfg.max_level) && level < hard_cap;
        if (!split) {
            Node& nd = nodes[id];
            nd.leaf = true;
            nd.src_begin = static_cast<int>(perm.size());
            nd.src_count = static_cast<int>(srcs.size());
            perm.insert(perm.end(), srcs.begin(), srcs.end());
            max_level = std::max(max_level, level);  // Leaf ctor, src/fmm/leaf.cpp:13
            return id;
        }
        std::vector<int> bucket[8];
        const double c[3] = {nodes[id].center[0], nodes[id].center[1], nodes[id].center[2]};
        for (int s : srcs) {
            const double* x = &centers[3 * s];
            const int b = (x[0] > c[0]) + 2 * (x[1] > c[1]) + 4 * (x[2] > c[2]);
            bucket[b].push_back(s);
        }
        srcs.clear();
        srcs.shrink_to_fit();
        nodes[id].leaf = false;
        nodes[id].src_begin = static_cast<int>(perm.size());
        for (int b = 0; b < 8; ++b) {
            const int ch = make(std::move(bucket[b]), level + 1, id, b);
            nodes[id].child[b] = ch;
        }
        nodes[id].src_count = static_cast<int>(perm.size()) - nodes[id].src_begin;
        return id;
    };
    std::vector<int> all(n);
    for (int i = 0; i < n; ++i) all[i] = i;
    make(std::move(all), 0, -1, 0);
    for (size_t i = 0; i < nodes.size(); ++i)
        if (nodes[i].leaf) leaves.push_back(static_cast<int>(i));
    src_center.resize(3 * static_cast<size_t>(n));
    for (int t = 0; t < n; ++t)
        for (int k = 0; k < 3; ++k) src_center[3 * t + k] = centers[3 * perm[t] + k];
}

// ---------------------------------------------------------------- lists

// Neighbour of equal or greater size along d, or -1.  A coarser leaf is
// reported only along the direction that reaches it without passing through
// another face/edge neighbour, so each neighbour appears once
// (Node::getNeighborGeqSize, src/fmm/nbor.cpp:10-483, written per axis).
static int nbr_geq(const std::vector<Node>& nodes, int id, const int* d) {
    const Node& nd = nodes[id];
    if (nd.parent < 0) return -1;
    const int b[3] = {nd.branch & 1, (nd.branch >> 1) & 1, (nd.branch >> 2) & 1};
    int dout[3] = {0, 0, 0};
    bool any_out = false, all_out = true;
    int mask = 0;
    for (int a = 0; a < 3; ++a) {
        if (!d[a]) continue;
        mask |= 1 << a;
        const bool out = (d[a] > 0 && b[a] == 1) || (d[a] < 0 && b[a] == 0);
        if (out) { dout[a] = d[a]; any_out = true; } else { all_out = false; }
    }
    const int target = nd.branch ^ mask;
    if (!any_out) return nodes[nd.parent].child[target];
    const int nb = nbr_geq(nodes, nd.parent, dout);
    if (nb < 0) return -1;
    if (nodes[nb].leaf) return all_out ? nb : -1;
    return nodes[nb].child[target];
}

// Leaves inside nb touching the current box across direction d, breadth first
// (Node::getNeighborsLeqSize, src/fmm/nbor.cpp:490-643).
static void nbrs_leq(const std::vector<Node>& nodes, int nb, const int* d, std::vector<int>& out) {
    std::deque<int> q{nb};
    while (!q.empty()) {
        const int cur = q.front();
        q.pop_front();
        if (nodes[cur].leaf) { out.push_back(cur); continue; }
        for (int c = 0; c < 8; ++c) {
            const int cb[3] = {c & 1, (c >> 1) & 1, (c >> 2) & 1};
            bool ok = true;
            for (int a = 0; a < 3; ++a)
                if ((d[a] > 0 && cb[a] != 0) || (d[a] < 0 && cb[a] != 1)) ok = false;
            if (ok) q.push_back(nodes[cur].child[c]);
        }
    }
}

void Plan::build_lists() {
    // Pre-order over the tree, as Stem/Leaf::buildLists (src/fmm/stem.cpp:48-57,
    // src/fmm/leaf.cpp:50-58).
    n_list2 = n_list4 = 0;
    for (size_t id = 0; id < nodes.size(); ++id) {
        Node& nd = nodes[id];
        if (nd.parent < 0) continue;
        for (int i = 0; i < 26; ++i) {
            const int nb = nbr_geq(nodes, static_cast<int>(id), kDirs[i]);
            if (nb < 0) continue;
            nd.nbors.push_back(nb);
            if (nd.leaf) nbrs_leq(nodes, nb, kDirs[i], nd.near_nbors);
        }
    }
    // Interaction lists (Node::buildInteractionList, src/fmm/node.cpp:61-84).
    for (size_t id = 0; id < nodes.size(); ++id) {
        Node& nd = nodes[id];
        if (nd.parent < 0) continue;
        auto contains = [&](int v) { return std::find(nd.nbors.begin(), nd.nbors.end(), v) != nd.nbors.end(); };
        for (int bn : nodes[nd.parent].nbors) {
            const Node& B = nodes[bn];
            if (B.src_count == 0) continue;
            if (B.leaf && !contains(bn)) { nd.leaf_ilist.push_back(bn); continue; }
            if (B.leaf) continue;
            for (int c = 0; c < 8; ++c) {
                const int ch = B.child[c];
                if (!contains(ch) && nodes[ch].src_count > 0) nd.ilist.push_back(ch);
            }
        }
        n_list2 += static_cast<long long>(nd.ilist.size());
        n_list4 += static_cast<long long>(nd.leaf_ilist.size());
    }
}

// ---------------------------------------------------------------- levels

void Plan::build_levels() {
    levels.assign(max_level + 1, Level{});
    const double k = pw.wavenum;
    const int order = cfg.interp_order;
    for (int l = lmin; l <= max_level; ++l) {
        Level& L = levels[l];
        L.level = l;
        // Angles::buildAngularSamples, src/fmm/angles.cpp:3-31.
        L.leng = cfg.root_leng / std::pow(2.0, l);
        const int tau = static_cast<int>(std::ceil(
            (1.73 * k * L.leng + 2.16 * std::pow(cfg.digits, 2.0 / 3.0) * std::pow(k * L.leng, 1.0 / 3.0))));
        L.L = static_cast<int>(std::floor(0.50 * tau));
        L.nth = tau + 1;
        gauss_legendre(L.nth, 1.0E-9, 0.0, kPi, L.thetas, L.weights);
        for (int i = 0; i < L.nth; ++i) L.weights[i] = L.weights[i] * std::sin(L.thetas[i]);
        L.nph = 2 * L.nth;
        L.phis.resize(L.nph);
        for (int i = 0; i < L.nph; ++i) L.phis[i] = 2.0 * kPi * i / static_cast<double>(L.nph);
        L.ndir = L.nth * L.nph;
        L.nps = static_cast<int>(std::floor(cfg.over_interp * (L.nth - 1)));
        // Angles::buildAngularMatrices, src/fmm/angles.cpp:33-55.
        L.khat.resize(3 * L.ndir);
        L.thph.resize(6 * L.ndir);
        L.m2l_w.resize(L.ndir);
        const double phi_w = 2.0 * kPi / static_cast<double>(L.nph);
        for (int ith = 0, d = 0; ith < L.nth; ++ith) {
            const double th = L.thetas[ith];
            for (int iph = 0; iph < L.nph; ++iph, ++d) {
                const double ph = L.phis[iph];
                L.khat[3 * d + 0] = std::sin(th) * std::cos(ph);
                L.khat[3 * d + 1] = std::sin(th) * std::sin(ph);
                L.khat[3 * d + 2] = std::cos(th);
                double* T = &L.thph[6 * d];
                T[0] = std::cos(th) * std::cos(ph);
                T[1] = std::cos(th) * std::sin(ph);
                T[2] = -std::sin(th);
                T[3] = -std::sin(ph);
                T[4] = std::cos(ph);
                T[5] = 0.0;
                L.m2l_w[d] = L.weights[ith] * phi_w;  // Node::buildMpoleToLocalCoeffs, node.cpp:124-132
            }
        }
        // Translation table (Tables::getAlpha / getInterpPsi / buildTranslationTable,
        // src/fmm/tables.cpp:90-220).
        const int nps = L.nps;
        if (nps < 2 * order || nps < 2) throw std::runtime_error("over_interp too small for interp_order");
        // The interpolation stencils reflect an index once at each pole and
        // wrap it once in phi: a grid needs at least interp_order thetas.
        if (L.nth < order)
            throw std::runtime_error("level " + std::to_string(l) + " has " + std::to_string(L.nth) +
                                     " thetas, fewer than interp_order: boxes too small for the wavelength "
                                     "(lower max_level or raise max_node_srcs)");
        std::unordered_map<long long, std::vector<cplx>> alpha;  // key: r^2 (integer)
        std::vector<cplx> h;
        std::vector<double> P;
        const cplx iu(0, 1);
        for (int dz = 0; dz <= 3; ++dz)
            for (int dy = 0; dy <= 3; ++dy)
                for (int dx = 0; dx <= 3; ++dx) {
                    if (std::max({dx, dy, dz}) <= 1) continue;
                    const long long r2 = dx * dx + dy * dy + dz * dz;
                    if (alpha.count(r2)) continue;
                    const double dist = std::sqrt(static_cast<double>(r2));
                    const double kr = k * dist * L.leng;
                    spherical_hankel1_all(kr, L.L, h);
                    std::vector<cplx> a(nps);
                    for (int ips = 0; ips < nps; ++ips) {
                        const double xi = std::cos(kPi * ips / static_cast<double>(nps - 1));
                        legendre_all(xi, L.L, P);
                        cplx coeff = 0.0;
                        for (int l2 = 0; l2 <= L.L; ++l2) coeff += pow_i(l2) * (2.0 * l2 + 1.0) * h[l2] * P[l2];
                        a[ips] = iu * k / (4.0 * kPi) * coeff;
                    }
                    alpha.emplace(r2, std::move(a));
                }
        L.transl.assign(static_cast<size_t>(316) * L.ndir, cplx(0));
        std::vector<double> psis(2 * order);
        int oid = 0;
        for (int dz = -3; dz <= 3; ++dz)
            for (int dy = -3; dy <= 3; ++dy)
                for (int dx = -3; dx <= 3; ++dx) {
                    if (std::max({std::abs(dx), std::abs(dy), std::abs(dz)}) <= 1) continue;
                    const double X[3] = {double(dx), double(dy), double(dz)};
                    const double r = std::sqrt(X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
                    const double rh[3] = {X[0] / r, X[1] / r, X[2] / r};
                    const auto& a = alpha.at(static_cast<long long>(dx * dx + dy * dy + dz * dz));
                    for (int d = 0; d < L.ndir; ++d) {
                        const double* kh = &L.khat[3 * d];
                        double c = kh[0] * rh[0] + kh[1] * rh[1] + kh[2] * rh[2];
                        c = std::min(1.0, std::max(-1.0, c));
                        const double psi = std::acos(c);
                        const int near = static_cast<int>(std::floor((nps - 1) * psi / kPi));
                        for (int ips = near + 1 - order, kk = 0; ips <= near + order; ++ips, ++kk)
                            psis[kk] = kPi * ips / static_cast<double>(nps - 1);
                        cplx t = 0.0;
                        for (int ips = near + 1 - order, kk = 0; kk < 2 * order; ++ips, ++kk)
                            t += a[flip_idx(ips, nps)] * lagrange(psi, psis.data(), 2 * order, kk);
                        L.transl[static_cast<size_t>(oid) * L.ndir + d] = t;
                    }
                    ++oid;
                }
        // Child/parent phase shifts on this level's grid (Stem::buildMpoleCoeffs
        // and getShiftedLocalCoeffs, src/fmm/stem.cpp:89-96,118-125).
        L.shift_up.resize(8 * static_cast<size_t>(L.ndir));
        L.shift_down.resize(8 * static_cast<size_t>(L.ndir));
        for (int b = 0; b < 8; ++b) {
            const double pm[3] = {(b & 1) ? 1.0 : -1.0, (b & 2) ? 1.0 : -1.0, (b & 4) ? 1.0 : -1.0};
            double up[3], dn[3];
            for (int a = 0; a < 3; ++a) {
                up[a] = -(L.leng / 2.0 * pm[a]);        // c_parent - c_child, child at this level
                dn[a] = (L.leng / 2.0) / 2.0 * pm[a];  // c_child - c_this, child one level down
            }
            for (int d = 0; d < L.ndir; ++d) {
                const double kv[3] = {L.khat[3 * d] * k, L.khat[3 * d + 1] * k, L.khat[3 * d + 2] * k};
                L.shift_up[static_cast<size_t>(b) * L.ndir + d] = std::exp(iu * dot3(kv, up));
                L.shift_down[static_cast<size_t>(b) * L.ndir + d] = std::exp(iu * dot3(kv, dn));
            }
        }
    }
}

// ---------------------------------------------------------------- far plan

void Plan::build_far_plan() {
    const int order = cfg.interp_order, o2 = 2 * order;
    for (size_t id = 0; id < nodes.size(); ++id) nodes[id].box = -1;
    for (int l = lmin; l <= max_level; ++l) levels[l].boxes.clear();
    for (size_t id = 0; id < nodes.size(); ++id) {
        Node& nd = nodes[id];
        if (nd.level < lmin || nd.src_count == 0) continue;
        Level& L = levels[nd.level];
        nd.box = static_cast<int>(L.boxes.size());
        L.boxes.push_back(static_cast<int>(id));
    }
    for (int l = lmin; l <= max_level; ++l) {
        Level& L = levels[l];
        L.m2l_ptr.assign(1, 0);
        L.m2l_src.clear();
        L.m2l_off.clear();
        for (int id : L.boxes) {
            const Node& B = nodes[id];
            for (int s : B.ilist) {
                const Node& S = nodes[s];
                L.m2l_src.push_back(S.box);
                L.m2l_off.push_back(offset_id(B.ix - S.ix, B.iy - S.iy, B.iz - S.iz));
            }
            L.m2l_ptr.push_back(static_cast<int>(L.m2l_src.size()));
        }
    }
    // Transitions parent level p -> child level p+1.
    trans.assign(std::max(max_level, 0) + 1, Transition{});
    for (int p = lmin; p < max_level; ++p) {
        Transition& T = trans[p];
        T.plevel = p;
        const Level& Lp = levels[p];
        const Level& Lc = levels[p + 1];
        const int mth = Lc.nth, mph = Lc.nph;  // child grid
        const int nth = Lp.nth, nph = Lp.nph;  // parent grid
        // Tables::getInterpTheta(p+1 -> p), src/fmm/tables.cpp:7-47.
        std::vector<double> th_coef(static_cast<size_t>(nth) * o2), ph_coef(static_cast<size_t>(nph) * o2);
        std::vector<int> th_near(nth), ph_near(nph);
        std::vector<double> xs(o2);
        for (int j = 0; j < nth; ++j) {
            const double tgt = Lp.thetas[j];
            const int near = near_gl_node_idx(tgt, mth, 0.0, kPi);
            for (int i = near + 1 - order, kk = 0; i <= near + order; ++i, ++kk) {
                double s = Lc.thetas[flip_idx(i, mth)];
                if (i < 0) s *= -1.0;
                else if (i >= mth) s = 2.0 * kPi - s;
                xs[kk] = s;
            }
            for (int kk = 0; kk < o2; ++kk) th_coef[j * o2 + kk] = lagrange(tgt, xs.data(), o2, kk);
            th_near[j] = near;
        }
        // Tables::getInterpPhi(p+1 -> p), src/fmm/tables.cpp:49-78.
        for (int j = 0; j < nph; ++j) {
            const double tgt = Lp.phis[j];
            const int near = static_cast<int>(std::floor(mph * tgt / (2.0 * kPi)));
            for (int i = near + 1 - order, kk = 0; i <= near + order; ++i, ++kk)
                xs[kk] = 2.0 * kPi * i / static_cast<double>(mph);
            for (int kk = 0; kk < o2; ++kk) ph_coef[j * o2 + kk] = lagrange(tgt, xs.data(), o2, kk);
            ph_near[j] = near;
        }
        // M2M stencils (Stem::addInterpCoeffs, src/fmm/stem.cpp:133-184).
        auto reset = [](Stencil& s, int rows) {
            s.ptr.assign(rows + 1, 0);
            s.src.clear();
            s.refl.clear();
            s.coef.clear();
        };
        reset(T.up_th, nth);
        for (int j = 0; j < nth; ++j) {
            for (int i = th_near[j] + 1 - order, kk = 0; i <= th_near[j] + order; ++i, ++kk) {
                const int f = flip_idx(i, mth);
                T.up_th.src.push_back(f);
                T.up_th.refl.push_back(f != i);
                T.up_th.coef.push_back(th_coef[j * o2 + kk]);
            }
            T.up_th.ptr[j + 1] = static_cast<int>(T.up_th.src.size());
        }
        reset(T.up_ph, nph);
        for (int j = 0; j < nph; ++j) {
            for (int i = ph_near[j] + 1 - order, kk = 0; i <= ph_near[j] + order; ++i, ++kk) {
                T.up_ph.src.push_back(wrap_idx(i, mph));
                T.up_ph.refl.push_back(0);
                T.up_ph.coef.push_back(ph_coef[j * o2 + kk]);
            }
            T.up_ph.ptr[j + 1] = static_cast<int>(T.up_ph.src.size());
        }
        // L2L stencils: exact transposes, in gather form (Stem::addAnterpCoeffs,
        // src/fmm/stem.cpp:186-244).  Rows are child indices.
        {
            std::vector<std::vector<std::pair<int, double>>> rows(mph);
            for (int ip = 0; ip < nph; ++ip)
                for (int j = ph_near[ip] + 1 - order, kk = 0; j <= ph_near[ip] + order; ++j, ++kk)
                    rows[wrap_idx(j, mph)].emplace_back(ip, ph_coef[ip * o2 + kk]);
            reset(T.dn_ph, mph);
            for (int r = 0; r < mph; ++r) {
                for (auto& e : rows[r]) {
                    T.dn_ph.src.push_back(e.first);
                    T.dn_ph.refl.push_back(0);
                    T.dn_ph.coef.push_back(e.second);
                }
                T.dn_ph.ptr[r + 1] = static_cast<int>(T.dn_ph.src.size());
            }
        }
        {
            struct E { int src, refl; double c; };
            std::vector<std::vector<E>> rows(mth);
            for (int it = 0; it < nth; ++it)
                for (int j = th_near[it] + 1 - order, kk = 0; j <= th_near[it] + order; ++j, ++kk) {
                    const int f = flip_idx(j, mth);
                    rows[f].push_back(E{it, f != j, th_coef[it * o2 + kk]});
                }
            reset(T.dn_th, mth);
            for (int r = 0; r < mth; ++r) {
                for (auto& e : rows[r]) {
                    T.dn_th.src.push_back(e.src);
                    T.dn_th.refl.push_back(e.refl);
                    T.dn_th.coef.push_back(e.c);
                }
                T.dn_th.ptr[r + 1] = static_cast<int>(T.dn_th.src.size());
            }
        }
        // Parent/child box lists.
        T.par_box.clear();
        T.par_ilist.clear();
        T.child_ptr.assign(1, 0);
        T.child_box.clear();
        T.child_oct.clear();
        for (int id : Lp.boxes) {
            const Node& P = nodes[id];
            if (P.leaf) continue;
            T.par_box.push_back(P.box);
            T.par_ilist.push_back(P.ilist.empty() ? 0 : 1);
            for (int b = 0; b < 8; ++b) {
                const Node& C = nodes[P.child[b]];
                if (C.src_count == 0) continue;
                T.child_box.push_back(C.box);
                T.child_oct.push_back(b);
            }
            T.child_ptr.push_back(static_cast<int>(T.child_box.size()));
        }
    }
    // Far leaves and pattern storage.
    far_leaves.clear();
    pat_elems = 0;
    for (int id : leaves) {
        const Node& nd = nodes[id];
        if (nd.level < lmin || nd.src_count == 0) continue;
        FarLeaf f;
        f.level = nd.level;
        f.box = nd.box;
        f.src0 = nd.src_begin;
        f.nsrc = nd.src_count;
        f.pat_off = pat_elems;
        pat_elems += static_cast<long long>(nd.src_count) * levels[nd.level].ndir;
        far_leaves.push_back(f);
    }
}

// ---------------------------------------------------------------- near plan

// Near-field blocks: every list-1 leaf pair once, every list-3/4 (leaf, node)
// pair, and the strict lower triangle of every leaf (Leaf::findNearNborPairs and
// Leaf::buildNearRads, src/fmm/leaf.cpp:70-163; Node::pushSelfToNearNonNbors,
// src/fmm/node.cpp:90-99).  Each stored block is applied as Z and Z^T.
void Plan::build_near_plan() {
    near_blocks.clear();
    near_entries = 0;
    n_near_pairs = 0;
    auto add = [&](int r0, int nr, int c0, int nc, int self) {
        if (nr <= 0 || nc <= 0) return;
        NearBlock b{r0, nr, c0, nc, near_entries, self};
        // a self block is strict-lower in the reference; with self terms it
        // also holds the diagonal
        const long long cnt = self ? static_cast<long long>(nr) * (nr - 1) / 2 + (cfg.self_terms ? nr : 0)
                                   : static_cast<long long>(nr) * nc;
        if (cnt == 0) return;
        near_entries += cnt;
        near_blocks.push_back(b);
    };
    for (int a : leaves) {
        const Node& A = nodes[a];
        for (int b : A.near_nbors) {
            if (!(a < b)) continue;
            const Node& B = nodes[b];
            if (A.src_count == 0 || B.src_count == 0) continue;
            ++n_near_pairs;
            add(A.src_begin, A.src_count, B.src_begin, B.src_count, 0);
        }
    }
    for (size_t id = 0; id < nodes.size(); ++id) {
        const Node& B = nodes[id];
        for (int lf : B.leaf_ilist) {
            const Node& Lf = nodes[lf];
            add(Lf.src_begin, Lf.src_count, B.src_begin, B.src_count, 0);
        }
    }
    for (int a : leaves) {
        const Node& A = nodes[a];
        add(A.src_begin, A.src_count, A.src_begin, A.src_count, 1);
    }

    // Tiles of the stored blocks and the partial sums they write.  A self block
    // is packed lower-triangular (row i holds columns 0..i-1, or 0..i with the
    // diagonal).  Partials are numbered tile by tile (rows, then columns), then
    // given slots sorted by target, ties in that order.
    near_tiles.clear();
    long long parts = 0;
    std::vector<int> part_tgt;
    auto tri = [](long long i, int kind) { return kind == 1 ? i * (i - 1) / 2 : i * (i + 1) / 2; };
    auto push = [&](const NearBlock& b, int kind, int mode, long long z, int i0, int ni, int j0, int nj) {
        NearTile t;
        t.z = z;
        t.r0 = b.row0;
        t.c0 = b.col0;
        t.i0 = i0;
        t.ni = ni;
        t.j0 = j0;
        t.nj = nj;
        t.ld = kind == 0 ? b.ncol : 0;
        t.kind = kind;
        t.slot = 0;
        t.mode = mode;
        parts += ni + nj;
        if (parts > std::numeric_limits<int>::max() / 2) throw std::runtime_error("near field: too many partial sums");
        for (int i = 0; i < ni; ++i) part_tgt.push_back(b.row0 + i0 + i);
        for (int j = 0; j < nj; ++j) part_tgt.push_back(b.col0 + j0 + j);
        near_tiles.push_back(t);
    };
    for (const NearBlock& b : near_blocks) {
        const int kind = b.self ? (cfg.self_terms ? 2 : 1) : 0;
        const int d = kind == 2 ? 1 : 0;
        if (kind == 0 && b.ncol <= kNearTileCols) {  // whole rows
            const int rows = std::min(kNearTileRows, kNearTileEntries / b.ncol);
            for (int i0 = 0; i0 < b.nrow; i0 += rows)
                push(b, 0, 0, b.off + static_cast<long long>(i0) * b.ncol, i0, std::min(rows, b.nrow - i0), 0, b.ncol);
        } else if (kind != 0 && b.nrow <= kNearTileCols) {  // whole packed rows
            for (int i0 = 0; i0 < b.nrow;) {
                int ni = 1;
                while (i0 + ni < b.nrow && ni < kNearTileRows && tri(i0 + ni + 1, kind) - tri(i0, kind) <= kNearTileEntries)
                    ++ni;
                const int nj = i0 + ni - 1 + d;  // columns 0 .. nj - 1
                if (nj > 0) push(b, kind, 1, b.off + tri(i0, kind), i0, ni, 0, nj);
                i0 += ni;
            }
        } else {  // column ranges, row by row
            for (int i0 = 0; i0 < b.nrow; i0 += kNearTileRowsSplit) {
                const int ni = std::min(kNearTileRowsSplit, b.nrow - i0);
                for (int j0 = 0; j0 < b.ncol; j0 += kNearTileCols) {
                    if (kind != 0 && j0 >= i0 + ni - 1 + d) break;  // no entries from here on
                    push(b, kind, 2, b.off, i0, ni, j0, std::min(kNearTileCols, b.ncol - j0));
                }
            }
        }
    }
    near_parts = static_cast<int>(parts);
    near_red_ptr.assign(n + 1, 0);
    for (int t : part_tgt) ++near_red_ptr[t + 1];
    for (int t = 0; t < n; ++t) near_red_ptr[t + 1] += near_red_ptr[t];
    {
        std::vector<int> fill(near_red_ptr.begin(), near_red_ptr.end() - 1);
        near_slot.clear();
        int p = 0;
        for (NearTile& t : near_tiles) {
            t.slot = static_cast<int>(near_slot.size());
            const int cnt = t.ni + t.nj;
            for (int q = 0; q < cnt; ++q) near_slot.push_back(fill[part_tgt[p + q]]++);
            while (near_slot.size() % 4) near_slot.push_back(0);
            p += cnt;
        }
    }

    // Block rows: every stored block in both orientations.
    std::vector<int> leaf_of(n, -1);  // tree slot -> leaf node
    for (int a : leaves)
        for (int s = 0; s < nodes[a].src_count; ++s) leaf_of[nodes[a].src_begin + s] = a;
    std::unordered_map<int, std::vector<std::pair<int, int>>> ranges;  // leaf -> column ranges
    for (const NearBlock& b : near_blocks) {
        const int ra = leaf_of[b.row0];
        ranges[ra].emplace_back(b.col0, b.ncol);
        if (b.self) continue;
        // transpose: every leaf holding rows of the column range sees the row range
        for (int s = b.col0; s < b.col0 + b.ncol;) {
            const int lb = leaf_of[s];
            ranges[lb].emplace_back(b.row0, b.nrow);
            s = nodes[lb].src_begin + nodes[lb].src_count;
        }
    }
    near_rows.clear();
    near_cols.clear();
    near_row_entries = 0;
    for (int a : leaves) {
        const Node& A = nodes[a];
        if (A.src_count == 0) continue;
        auto it = ranges.find(a);
        if (it == ranges.end()) continue;
        NearRow r{A.src_begin, A.src_count, 0, near_row_entries, static_cast<long long>(near_cols.size())};
        for (const auto& rg : it->second)
            for (int c = 0; c < rg.second; ++c) near_cols.push_back(rg.first + c);
        r.ncol = static_cast<int>(near_cols.size() - r.col_off);
        near_row_entries += static_cast<long long>(r.nrow) * r.ncol;
        near_rows.push_back(r);
    }
}

}  // namespace mlfma
