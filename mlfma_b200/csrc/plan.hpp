// Host-side operator setup: sources, octree, interaction lists, per-level
// angular grids and tables, all in FP64 and flattened into the arrays the CUDA
// kernels consume.  This restates the reference's setup sequence
// (src/mlfma.cpp:21-64): Node::initStatic, the Stem/Leaf constructors,
// buildLists, Leaf::buildNearRads (pair enumeration only; the entries are
// assembled on the GPU), Node::buildTables and Leaf::buildRadPats (on the GPU).
#pragma once

#include <complex>
#include <string>
#include <vector>

#include "common.hpp"

namespace mlfma {

using cplx = std::complex<double>;

enum SourceKind { kDipole = 0, kRwg = 1 };

struct Config {
    // Same meaning as the reference Config fields (src/config.h:50-73).
    int quad_prec = 2;        // Precision: 0 VERYLOW(1 pt) 1 LOW(3) 2 MEDIUM(7) 3 HIGH(13)
    int digits = 3;           // excess-bandwidth digits
    int interp_order = 3;     // half-width: 2*interp_order points
    double over_interp = 2.0; // psi oversampling of the transfer function
    double root_leng = 4.0;   // root box side, centred at the origin
    int max_node_srcs = 64;   // split while a box holds more sources than this
    // Extensions.
    int max_level = 0;        // >0: never split below this level
    int ref_compat = 1;       // 1: reproduce the reference's stale-local rule
    int self_terms = 0;       // 1: unit dipole diagonal; touching RWG pairs in
                              //    mixed-potential form, 1/R extracted
    int device_tree = 0;      // 1: octree and lists built on the current CUDA
                              //    device (same nodes, order and lists)
};

struct PlaneWave {
    double amplitude = 1.0;
    double pol[3] = {1, 0, 0};
    double khat[3] = {0, 0, 1};
    double wavenum = 1.0;
};

struct Node {
    int level = 0;
    int parent = -1;
    int branch = 0;          // octant index in the parent (x + 2y + 4z bits)
    int child[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
    bool leaf = true;
    int ix = 0, iy = 0, iz = 0;  // integer coordinates at this level
    double center[3] = {0, 0, 0};
    double leng = 0;
    int src_begin = 0, src_count = 0;  // range in tree order (whole subtree)
    std::vector<int> nbors;      // equal-or-greater-size neighbours
    std::vector<int> ilist;      // list 2
    std::vector<int> leaf_ilist; // list 4
    std::vector<int> near_nbors; // list 1 (leaves only)
    int box = -1;                // index among this level's far boxes
};

// One angular level (Angles, src/fmm/angles.cpp:3-55).
struct Level {
    int level = 0, nth = 0, nph = 0, ndir = 0, L = 0, nps = 0;
    double leng = 0;
    std::vector<double> thetas, weights, phis;
    std::vector<double> khat;   // 3 per direction
    std::vector<double> thph;   // 6 per direction (row-major 2x3)
    std::vector<double> m2l_w;  // weights[ith] * 2 pi / nph per direction
    std::vector<cplx> transl;   // 316 x ndir
    std::vector<cplx> shift_up;   // 8 x ndir: e^{ik khat.(c_parent - c_child)} for a child at this level
    std::vector<cplx> shift_down; // 8 x ndir: e^{ik khat.(c_child - c_this)} on this level's grid
    std::vector<int> boxes;       // node ids of this level's non-empty boxes
    // M2L CSR over boxes: source box (this level) and offset id (0..315)
    std::vector<int> m2l_ptr, m2l_src, m2l_off;
};

// Gather-form stencil for one pass of interpolation or anterpolation:
// out[row] = sum_e coef[e] * sign(e) * in[src[e]], where a reflected entry
// also shifts phi by half a turn and flips the sign (pole crossing).
struct Stencil {
    std::vector<int> ptr, src, refl;
    std::vector<double> coef;
};

// Transition between parent level p and child level p+1.
struct Transition {
    int plevel = 0;
    Stencil up_th, up_ph;     // M2M: theta pass (child rows -> parent rows), phi pass
    Stencil dn_ph, dn_th;     // L2L: transposed phi pass, transposed theta pass
    std::vector<int> par_box;     // parent boxes (level p) that have children boxes
    std::vector<int> par_ilist;   // 1 if the parent's list 2 is non-empty
    std::vector<int> child_ptr, child_box, child_oct;
};

struct NearBlock {
    int row0, nrow, col0, ncol;  // source ranges in tree order
    long long off;               // entry offset
    int self;                    // 1: strict-lower packed self block (nrow == ncol)
};

// The near field of one leaf as a dense block row: every source of the leaf
// against the concatenated source ranges it interacts with directly (its own
// leaf, list-1 leaves, list-3/4 partners in either role).  Entries are stored
// row-major; col_off indexes the shared column list near_cols.
struct NearRow {
    int row0, nrow, ncol;
    long long off;      // entry offset
    long long col_off;  // offset into near_cols
};

// One tile of a stored near-field block for the symmetric application: the
// tile's entries are read once and give both its row sums (Z x) and its column
// sums (Z^T x).  Each sum is a partial written to its slot; a target's
// partials occupy consecutive slots (near_red_ptr), added in a second pass in a
// fixed order.  A tile holds at most kNearTileEntries entries, kNearTileRows
// rows and kNearTileCols columns, laid out in one of three ways:
//   mode 0: whole rows of a rectangular block, one contiguous span (row stride nj);
//   mode 1: whole rows of a packed self block, one contiguous span (row i0 + r
//           has i0 + r entries, i0 + r + 1 with the diagonal, from column 0);
//   mode 2: a column range of some rows (wide or large self blocks), row by row,
//           rows nj apart in the tile.
constexpr int kNearTileRows = 64;
constexpr int kNearTileCols = 64;
constexpr int kNearTileEntries = 1024;
constexpr int kNearTileRowsSplit = kNearTileEntries / kNearTileCols;  // rows of a mode-2 tile

struct NearTile {
    long long z;          // first entry (modes 0, 1) or the block's first entry (mode 2)
    int r0, c0;           // block's first row and first column source (tree order)
    int i0, ni, j0, nj;   // tile rows [i0, i0 + ni) and columns [j0, j0 + nj) within the block
    int ld;               // row stride of a rectangular block in the block storage (0 for a self block)
    int kind;             // 0 rectangular; 1 strict-lower self; 2 lower self with its diagonal
    int slot;             // near_slot offset (a multiple of 4): ni row slots, then nj column slots
    int mode;             // layout, above
};

struct FarLeaf {
    int level, box, src0, nsrc;
    long long pat_off;  // offset in units of (direction, 2 components)
};

struct Plan {
    SourceKind kind = kDipole;
    Config cfg;
    PlaneWave pw;
    int n = 0;
    // Sources in tree order; perm[t] = original index of tree slot t.
    std::vector<int> perm;
    std::vector<double> src_center;  // 3 per source (tree order)
    // Dipoles (tree order)
    std::vector<double> dip_pos, dip_phat;
    std::vector<double> dip_mom;     // original order, for the right-hand side
    // RWG (tree order) and triangles (input order)
    std::vector<RwgGeom> rwg;
    std::vector<TriGeom> tris;
    std::vector<double> tri_quad;    // nq x 3 per triangle
    std::vector<int> tri_v;          // 3 vertex indices per triangle
    std::vector<double> tri_p;       // 3 vertices x 3 coordinates per triangle
    std::vector<double> quad_w;      // nq weights (same rule for all triangles)
    int nq = 0;
    // Tree
    std::vector<Node> nodes;
    int max_level = 0;
    std::vector<int> leaves;         // DFS order (reference Leaf::leaves order)
    // Far field
    int lmin = 2;                    // coarsest level with far interactions
    std::vector<Level> levels;       // index = level (0..max_level); only >= 2 filled
    std::vector<Transition> trans;   // index = parent level
    std::vector<FarLeaf> far_leaves;
    long long pat_elems = 0;         // total (direction, 2 comp) slots
    // Near field
    std::vector<NearBlock> near_blocks;   // each interaction once (reference storage)
    long long near_entries = 0;
    std::vector<NearTile> near_tiles;     // symmetric application of near_blocks
    int near_parts = 0;                   // partial sums the tiles write
    std::vector<int> near_slot;           // per tile, padded to 4: slot of each partial
    std::vector<int> near_red_ptr;        // [n + 1]: target t's partials are slots ptr[t]..ptr[t+1]
    std::vector<NearRow> near_rows;       // both orientations, per leaf (many-rhs storage)
    std::vector<int> near_cols;
    long long near_row_entries = 0;
    // Stats
    long long n_list2 = 0, n_list4 = 0, n_near_pairs = 0;

    std::string build_dipoles(const Config& c, const PlaneWave& p, int n, const double* pos,
                              const double* mom);
    std::string build_rwg(const Config& c, const PlaneWave& p, int nv, const double* verts, int nf,
                          const int* faces, int ne, const int* rwgs);

    // b = -V in original source order (Solver ctor, src/solver.cpp:31-32).
    void rhs(cplx* b) const;
    // Same for another incident plane wave of the same wavenumber.
    void rhs_for(const PlaneWave& p, cplx* b) const;

    // RWG radiation patterns evaluated on the host exactly as the reference
    // rounds them (layout of the device pattern array).
    void rwg_patterns_host(std::vector<cplx>& pat) const;

private:
    std::string build_common(const std::vector<double>& centers);
    void build_tree(const std::vector<double>& centers);
    void build_lists();
    void build_levels();
    void build_far_plan();
    void build_near_plan();
};

// The 26 neighbour directions in the reference's order (FMM::Dir,
// src/fmm/fmm.h:13-17), 3 ints (dx, dy, dz) each.
const int* plan_directions();

// The tree and lists of P (nodes, perm, src_center, leaves, max_level, list
// counts) built on the current CUDA device from the source centres; empty on
// success.  Defined with the CUDA sources; a message beginning "host:" asks
// for the host build (a tree deeper than the device keys hold).
std::string build_tree_lists_device(Plan& P, const std::vector<double>& centers);

// Offset id of an integer M2L offset in Math::getINodeDistVecs order
// (src/math.cpp:106-122), or -1.
int offset_id(int dx, int dy, int dz);

// Closed-form RWG plane-wave integral, rounded as the reference rounds it.
void rwg_integral_exact(const RwgGeom& g, const TriGeom* tris, const double* kvec, cplx* out);

}  // namespace mlfma
