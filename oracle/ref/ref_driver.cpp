// Oracle driver: the reference MLFMA (ellilu11/MLFMA, src/) compiled from its
// own sources and exposed through a small C API so that tests can feed it the
// same seeded inputs as the CUDA implementation.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product library links or calls this.
//
// The driver repeats the reference's own setup and solve sequence
// (src/mlfma.cpp:16-76) without its hard-wired config files, building the
// sources the way src/fileio.h:110-131 (dipoles) and src/fileio.h:174-202
// (RWG) do.  The reference keeps all state in class statics (src/fmm/node.h:93-105),
// so one problem exists at a time; ref_create_* resets those statics first.
//
// White-box access: the reference's tree, lists and tables are private or
// protected members.  After every standard header is in, `private` and
// `protected` are redefined to `public` for the reference headers only, so
// the driver can read them (list sizes, tables, leaf membership) for
// cross-checking.  Layout is unaffected.

#include <Eigen/Dense>
#include <algorithm>
#include <array>
#include <cassert>
#include <cctype>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <numeric>
#include <queue>
#include <random>
#include <sstream>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <utility>
#include <vector>

#define private public
#define protected public
#include "mlfma.h"
#include "config.h"
#include "fileio.h"
#include "fmm/fmm.h"
#undef private
#undef protected

// The reference defines its stage timer in its main translation unit
// (src/mlfma.cpp:10); the driver is that unit here.
ClockTimes t;

using namespace FMM;

namespace {

struct RefState {
    std::shared_ptr<Excitation::PlaneWave> einc;
    SrcVec srcs;
    std::vector<vec3d> vertices;
    TriVec triangles;
    std::shared_ptr<Node> root;
    bool ready = false;
};
RefState g;

void reset_statics() {
    Node::angles.clear();
    Node::tables.clear();
    Node::nonNearPairs.clear();
    Node::maxLevel = 0;
    Node::numNodes = 0;
    Leaf::resetLeaves();
    g = RefState{};
}

Config make_config(int quad_prec, int digits, int interp_order, double over_interp,
                   double root_leng, int max_node_srcs, int nsrcs) {
    Config c;
    c.mode = Mode::READ;
    c.pdist = Dist::UNIFORM;
    c.qdist = QDist::UNIFORM;
    c.quadPrec = static_cast<Precision>(quad_prec);
    c.digits = digits;
    c.interpOrder = interp_order;
    c.overInterp = over_interp;
    c.rootLeng = root_leng;
    c.maxNodeSrcs = max_node_srcs;
    c.evalDirect = false;
    c.nsrcs = nsrcs;
    return c;
}

// Setup sequence of src/mlfma.cpp:21-64.
void build_operator(const Config& config) {
    const auto nsrcs = g.srcs.size();
    Node::initStatic(config, g.einc, static_cast<int>(nsrcs));
    if (nsrcs > static_cast<size_t>(config.maxNodeSrcs))
        g.root = std::make_shared<Stem>(g.srcs, 0, nullptr);
    else
        g.root = std::make_shared<Leaf>(g.srcs, 0, nullptr);
    g.root->buildLists();
    Leaf::buildNearRads();
    Node::buildTables();
    g.root->resizeCoeffs();
    Leaf::buildRadPats();
    g.ready = true;
}

// Silence the reference's console banners while it runs.
struct QuietCout {
    std::ostringstream sink;
    std::streambuf* old;
    QuietCout() : old(std::cout.rdbuf(sink.rdbuf())) {}
    ~QuietCout() { std::cout.rdbuf(old); }
};

}  // namespace

extern "C" {

// plane wave: [amplitude, pol(3), khat(3), wavenum]
int ref_create_dipoles(const double* pos, const double* mom, int n, const double* pw,
                       int digits, int interp_order, double over_interp,
                       double root_leng, int max_node_srcs) {
    QuietCout q;
    try {
        reset_statics();
        g.einc = std::make_shared<Excitation::PlaneWave>(
            vec3d(pw[1], pw[2], pw[3]), vec3d(pw[4], pw[5], pw[6]), pw[7], pw[0]);
        for (int i = 0; i < n; ++i)
            g.srcs.emplace_back(std::make_shared<Dipole>(
                g.einc, i, vec3d(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]),
                vec3d(mom[3 * i], mom[3 * i + 1], mom[3 * i + 2])));
        build_operator(make_config(0, digits, interp_order, over_interp, root_leng, max_node_srcs, n));
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "ref_create_dipoles: " << e.what() << '\n';
        return 1;
    }
}

// faces: nf x 3 vertex indices; rwgs: ne x 4 (v0, v1, t+, t-), all 0-based.
int ref_create_rwg(const double* verts, int nv, const int* faces, int nf, const int* rwgs, int ne,
                   const double* pw, int quad_prec, int digits, int interp_order,
                   double over_interp, double root_leng, int max_node_srcs) {
    QuietCout q;
    try {
        reset_statics();
        g.einc = std::make_shared<Excitation::PlaneWave>(
            vec3d(pw[1], pw[2], pw[3]), vec3d(pw[4], pw[5], pw[6]), pw[7], pw[0]);
        for (int i = 0; i < nv; ++i)
            g.vertices.emplace_back(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]);
        const auto prec = static_cast<Precision>(quad_prec);
        for (int i = 0; i < nf; ++i)
            g.triangles.emplace_back(std::make_shared<Triangle>(
                vec3i(faces[3 * i], faces[3 * i + 1], faces[3 * i + 2]), g.vertices, prec));
        for (int i = 0; i < ne; ++i)
            g.srcs.emplace_back(std::make_shared<RWG>(
                g.einc, i,
                Eigen::Vector4i(rwgs[4 * i], rwgs[4 * i + 1], rwgs[4 * i + 2], rwgs[4 * i + 3]),
                g.vertices, g.triangles));
        build_operator(make_config(quad_prec, digits, interp_order, over_interp, root_leng,
                                   max_node_srcs, ne));
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "ref_create_rwg: " << e.what() << '\n';
        return 1;
    }
}

// From the reference's text files, read by its own importers
// (importPlaneWave, src/fileio.h:8-27; importDipoles, fileio.h:110-131;
// importRWG, fileio.h:174-202).  Returns 1 when an importer throws.
int ref_create_dipoles_file(const char* path, const char* pw_path, int digits, int interp_order,
                            double over_interp, double root_leng, int max_node_srcs) {
    QuietCout q;
    try {
        reset_statics();
        g.einc = importPlaneWave(pw_path);
        g.srcs = importDipoles(path, g.einc);
        build_operator(make_config(0, digits, interp_order, over_interp, root_leng, max_node_srcs,
                                   static_cast<int>(g.srcs.size())));
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "ref_create_dipoles_file: " << e.what() << '\n';
        return 1;
    }
}

int ref_create_rwg_files(const char* vpath, const char* fpath, const char* rpath, const char* pw_path,
                         int quad_prec, int digits, int interp_order, double over_interp, double root_leng,
                         int max_node_srcs) {
    QuietCout q;
    try {
        reset_statics();
        g.einc = importPlaneWave(pw_path);
        g.srcs = importRWG(vpath, fpath, rpath, static_cast<Precision>(quad_prec), g.einc);
        build_operator(make_config(quad_prec, digits, interp_order, over_interp, root_leng, max_node_srcs,
                                   static_cast<int>(g.srcs.size())));
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "ref_create_rwg_files: " << e.what() << '\n';
        return 1;
    }
}

int ref_num_srcs() { return static_cast<int>(g.srcs.size()); }

// [numNodes, numLeaves, maxLevel]
void ref_info(int* out) {
    out[0] = Node::getNumNodes();
    out[1] = Leaf::getNumLeaves();
    out[2] = Node::getMaxLvl();
}

// b = -V, interleaved complex (src/solver.cpp:31-32).
int ref_rhs(double* b) {
    if (!g.ready) return 1;
    for (size_t i = 0; i < g.srcs.size(); ++i) {
        const cmplx v = -g.srcs[i]->getVoltage();
        b[2 * i] = v.real();
        b[2 * i + 1] = v.imag();
    }
    return 0;
}

// y = A x: the body of Solver::evalRvec (src/solver.cpp:41-48) on a fresh rvec.
// The FMM coefficient state persists across calls exactly as in the reference.
int ref_matvec(const double* x, double* y) {
    if (!g.ready) return 1;
    QuietCout q;
    const size_t n = g.srcs.size();
    for (size_t i = 0; i < n; ++i) (*Node::lvec)[i] = cmplx(x[2 * i], x[2 * i + 1]);
    *Node::rvec = vecXcd::Zero(static_cast<long>(n));
    if (g.root->isNodeType<Stem>()) {
        g.root->buildMpoleCoeffs();
        g.root->buildLocalCoeffs();
    }
    Leaf::evaluateSols();
    for (size_t i = 0; i < n; ++i) {
        y[2 * i] = (*Node::rvec)[i].real();
        y[2 * i + 1] = (*Node::rvec)[i].imag();
    }
    return 0;
}

// Solver(...).solve() (src/mlfma.cpp:72-76); returns the iteration count.
int ref_solve(int max_iter, double eps, double* currents, int* iters) {
    if (!g.ready) return 1;
    std::ostringstream sink;
    std::streambuf* old = std::cout.rdbuf(sink.rdbuf());
    // main() reaches the solve with rvec zero from Node::initStatic
    // (src/fmm/node.cpp:21-22); earlier ref_matvec calls leave a result there.
    *Node::rvec = vecXcd::Zero(static_cast<long>(g.srcs.size()));
    Solver solver(g.srcs, g.root, max_iter, eps, Node::lvec, Node::rvec, Node::currents);
    solver.solve();
    std::cout.rdbuf(old);
    const std::string log = sink.str();
    int count = 0;
    for (size_t p = log.find("Do iteration"); p != std::string::npos; p = log.find("Do iteration", p + 1))
        ++count;
    *iters = count;
    for (size_t i = 0; i < g.srcs.size(); ++i) {
        currents[2 * i] = (*Node::currents)[i].real();
        currents[2 * i + 1] = (*Node::currents)[i].imag();
    }
    return 0;
}

// Angular grid of one level: sizes first (nth, nph, L), then optional arrays.
int ref_angles(int level, int* sizes, double* thetas, double* weights, double* phis) {
    if (level < 0 || level >= static_cast<int>(Node::angles.size())) return 1;
    const auto& a = Node::angles[level];
    sizes[0] = static_cast<int>(a.thetas.size());
    sizes[1] = static_cast<int>(a.phis.size());
    sizes[2] = a.L;
    if (thetas) std::copy(a.thetas.begin(), a.thetas.end(), thetas);
    if (weights) std::copy(a.weights.begin(), a.weights.end(), weights);
    if (phis) std::copy(a.phis.begin(), a.phis.end(), phis);
    return 0;
}

// Interpolation tables (level+1 -> level): per target row 2*order coefficients
// and the near index (src/fmm/tables.cpp:7-78).
int ref_interp(int level, double* th_coef, int* th_near, double* ph_coef, int* ph_near) {
    if (level < 0 || level >= static_cast<int>(Node::tables.size())) return 1;
    const auto& tb = Node::tables[level];
    if (tb.interpTheta.empty()) return 2;
    const int o2 = 2 * Node::config.interpOrder;
    for (size_t j = 0; j < tb.interpTheta.size(); ++j) {
        for (int k = 0; k < o2; ++k) th_coef[j * o2 + k] = tb.interpTheta[j].first[k];
        th_near[j] = tb.interpTheta[j].second;
    }
    for (size_t j = 0; j < tb.interpPhi.size(); ++j) {
        for (int k = 0; k < o2; ++k) ph_coef[j * o2 + k] = tb.interpPhi[j].first[k];
        ph_near[j] = tb.interpPhi[j].second;
    }
    return 0;
}

// Translation table of one level, 316 offsets in the order of
// Math::getINodeDistVecs (src/math.cpp:106-122), interleaved complex.
int ref_transl(int level, double* out) {
    if (level < 0 || level >= static_cast<int>(Node::tables.size())) return 1;
    const auto& tb = Node::tables[level];
    const auto dvecs = Math::getINodeDistVecs();
    const size_t ndir = Node::angles[level].getNumAllAngles();
    for (size_t o = 0; o < dvecs.size(); ++o) {
        const auto& row = tb.transl.at(dvecs[o]);
        for (size_t d = 0; d < ndir; ++d) {
            out[2 * (o * ndir + d)] = row[d].real();
            out[2 * (o * ndir + d) + 1] = row[d].imag();
        }
    }
    return 0;
}

// Leaves in the reference's DFS order: level, centre, source count.
int ref_num_leaves() { return Leaf::getNumLeaves(); }
int ref_leaf(int i, int* level, double* center, int* nsrcs, int* src_idx) {
    if (i < 0 || i >= Leaf::getNumLeaves()) return 1;
    const auto& leaf = Leaf::leaves[i];
    *level = leaf->level;
    center[0] = leaf->center[0];
    center[1] = leaf->center[1];
    center[2] = leaf->center[2];
    *nsrcs = static_cast<int>(leaf->srcs.size());
    if (src_idx)
        for (size_t s = 0; s < leaf->srcs.size(); ++s) src_idx[s] = static_cast<int>(leaf->srcs[s]->getIdx());
    return 0;
}

// Radiation pattern of source s (position inside leaf i) along direction d of
// the leaf's level, two complex components (Leaf::buildRadPats, leaf.cpp:185-207).
int ref_radpat(int i, int s, int d, double* out) {
    if (i < 0 || i >= Leaf::getNumLeaves()) return 1;
    const auto& leaf = Leaf::leaves[i];
    if (d < 0 || d >= static_cast<int>(leaf->radPats.size())) return 2;
    if (s < 0 || s >= static_cast<int>(leaf->srcs.size())) return 3;
    const vec2cd& v = leaf->radPats[d][s];
    out[0] = v[0].real();
    out[1] = v[0].imag();
    out[2] = v[1].real();
    out[3] = v[1].imag();
    return 0;
}

// Far field of the given currents along unit directions khat (ndir x 3):
// the loop body of Node::printFarSols (src/fmm/node.cpp:155-164) for an
// arbitrary direction list; out is ndir x 3 complex.
int ref_farfield(const double* cur, int ndir, const double* khat, double* out) {
    if (!g.ready) return 1;
    const double k = g.einc->wavenum;
    for (int d = 0; d < ndir; ++d) {
        const vec3d kh(khat[3 * d], khat[3 * d + 1], khat[3 * d + 2]);
        const auto& krhat = kh * k;
        vec3cd dirFar = vec3cd::Zero();
        for (const auto& src : g.srcs)
            dirFar += cmplx(cur[2 * src->getIdx()], cur[2 * src->getIdx() + 1]) * src->getFarAlongDir(krhat);
        const vec3cd& far = Phys::C * k * Math::ImRR(kh) * dirFar;
        for (int c = 0; c < 3; ++c) {
            out[6 * d + 2 * c] = far[c].real();
            out[6 * d + 2 * c + 1] = far[c].imag();
        }
    }
    return 0;
}

// List sizes summed over the tree: [list2 pairs, list4 pairs, near leaf pairs,
// self entries, near entries stored, non-near entries stored].
void ref_list_stats(long long* out) {
    long long l2 = 0, l4 = 0;
    std::queue<std::shared_ptr<Node>> q;
    q.push(g.root);
    while (!q.empty()) {
        auto nd = q.front();
        q.pop();
        l2 += static_cast<long long>(nd->iList.size());
        l4 += static_cast<long long>(nd->leafIlist.size());
        for (const auto& b : nd->branches) q.push(b);
    }
    long long self = 0, nearE = 0, nonNearE = 0;
    for (const auto& leaf : Leaf::leaves) {
        self += static_cast<long long>(leaf->selfRads.size());
        for (const auto& r : leaf->nearRads) nearE += static_cast<long long>(r.size());
        for (const auto& r : leaf->nonNearRads) nonNearE += static_cast<long long>(r.size());
    }
    out[0] = l2;
    out[1] = l4;
    out[2] = static_cast<long long>(Leaf::nearPairs.size());
    out[3] = self;
    out[4] = nearE;
    out[5] = nonNearE;
}

// One entry of the impedance kernel, A_mn / (C k) (src/sources/*::getIntegratedRad).
int ref_entry(int m, int n, double* out) {
    if (!g.ready) return 1;
    const cmplx z = g.srcs[m]->getIntegratedRad(g.srcs[n]);
    out[0] = z.real();
    out[1] = z.imag();
    return 0;
}

void ref_destroy() { reset_statics(); }

}  // extern "C"
