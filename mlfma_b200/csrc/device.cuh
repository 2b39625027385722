// Device-side plan: flat arrays in HBM that the kernels read, and the launch
// wrappers.  One DeviceOp per operator handle.
//
// The far field exists in one of two precisions, chosen at setup:
//   * FP64: complex double everywhere (the reference's arithmetic);
//   * mixed: outgoing/local patterns, radiation patterns, transfer functions,
//     shifts and interpolation weights in complex float, accumulated in float;
//     the near field, x, y and the combination stay complex double.  A mixed
//     operator also keeps the FP64 far field, which iterative refinement uses
//     for its FP64 residuals.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "plan.hpp"

namespace mlfma {

constexpr int kMaxLevels = 20;

enum Precision { kFp64 = 0, kMixed = 1 };

template <class R> struct Cx;
template <> struct Cx<double> { using T = double2; };
template <> struct Cx<float> { using T = float2; };

template <class R>
struct DevLevelT {
    using C = typename Cx<R>::T;
    int nth, nph, ndir, nbox;
    C* A;                        // outgoing patterns [nbox][ndir][2]
    C* B;                        // local (incoming) patterns [nbox][ndir][2]
    C* Am;                       // many right-hand sides: [nbox][ndir][2][max_rhs]
    C* Bm;
    const C* transl;             // [316][ndir]
    const R* w;                  // [ndir] quadrature weight applied after M2L
    const C* shift_up;           // [8][ndir]
    const C* shift_down;         // [8][ndir]
    const int* m2l_ptr;          // [nbox+1]
    const int* m2l_src;
    const int* m2l_off;
    const int* anti;             // [ndir]: element of the antipodal direction, for elements e < ndir
};

// Stencil rows padded to a fixed width (padding entries have coefficient 0):
// entry k of row r is at r * width + k.  The sign of a pole-reflected tap is
// folded into its coefficient.
template <class R>
struct DevStencilT {
    int width;
    const int* src;
    const int* refl;
    const R* coef;
    // the same entries tap-major: entry k of row r at k * rows + r (threads
    // on consecutive rows read consecutive words)
    int rows;
    const int* src_t;
    const R* coef_t;
};

template <class R>
struct DevTransT {
    DevStencilT<R> up_th, up_ph, dn_ph, dn_th;
    int plevel, npar;
    const int* par_box;
    const int* par_ilist;
    const int* child_ptr;
    const int* child_box;
    const int* child_oct;
    // Many right-hand sides: stencil weights with the octant shift folded in,
    //   fold_up[oct][jth][iph][k] = up_th weight (sign included) x shift_up of the
    //                                child direction that tap reads,
    //   fold_dn[oct][ith][jph][k] = dn_ph weight x shift_down of the parent
    //                                direction that tap reads.
    const typename Cx<R>::T* fold_up;
    const typename Cx<R>::T* fold_dn;
};

struct DevFarLeaf {
    int level, box, src0, nsrc;
    long long pat_off;
};

// M2L on many right-hand sides: the boxes of one level that share a parent
// (at most 8) and the union of their list-2 sources; for each candidate source
// the offset id towards every target (-1: not in that target's list 2).
constexpr int kMaxGroup = 8;
constexpr int kMaxRhs = 64;  // right-hand sides of one product

struct DevM2LGroup {
    int level, ntgt;
    int tgt[kMaxGroup];       // target boxes (this level)
    int empty_mask;           // bit t: target t has an empty list 2
    int cand0, ncand;         // candidate range
    long long t8_off;         // this group's transfer values: [ndir][ncand][kMaxGroup]
};

// A stored near-field block (the reference's storage: each interaction once)
// and one tile of it; see NearBlock and NearTile in plan.hpp.
struct DevNearBlock {
    int row0, nrow, col0, ncol;
    long long off;
    int kind, pad;  // 0 rectangular, 1 strict-lower self, 2 lower self with diagonal
};

struct DevNearTile {
    long long z;
    int r0, c0, i0, ni, j0, nj, ld, kind, slot, mode;
};

// Runs k_wait_runs_out (a bounded mbarrier wait on a barrier nothing arrives
// on) on the current device's default stream.
void launch_wait_runs_out(long long limit, int* status);

// A leaf of the block-Jacobi preconditioner: its sources [row0, row0 + nb)
// (tree order), its stored self block (entry offset, kind 1 strict lower or 2
// with the diagonal; zoff < 0: none) and its inverse's offset.
struct DevBjLeaf {
    int row0, nb, kind, pad;
    long long zoff, ioff;
};

struct DevNearRow {
    int row0, nrow, ncol, pad;
    long long off, col_off;
};

// Source geometry on the device, tree order (patterns, near field, far field).
struct DevSources {
    int kind;
    double k;
    const double* pos;      // dipole positions
    const double* phat;     // dipole unit moments
    const RwgGeom* rwg;     // RWG geometry
    const TriGeom* tris;    // triangles (input order)
    const double* tri_quad; // [tri][nq][3]
    const double* quad_w;   // [nq]
    int nq;
    int self_terms;         // see Config::self_terms
    const int* tri_v;       // [tri][3] vertex indices
    const double* tri_p;    // [tri][3][3] vertices
};

// Geometry the setup kernels need (patterns, near-field entries).
struct DevGeomLevel {
    const double* thph;  // [ndir][6]
    const double* khat;  // [ndir][3]
    int ndir;
};

struct TuneReport {
    int m2l_chunk;                 // one-vector M2L directions per block
    int m2m_rows[kMaxLevels];      // one-vector M2M parent rows per block (index: parent level)
    int multi_rows_fast;           // many-rhs M2M grid order (1 rows fastest, 0 parents fastest)
    int multi_l2l_pairs;           // many-rhs L2L column pairs per block
    float before_ms, after_ms;     // product time before and after
    int near_blocks_per_sm;        // one-vector near field: persistent blocks per SM
    int interp_path;               // tensor-core interpolation: bit 0 one vector, bit 1 many
    int schedule;                  // one-vector product: bit 0 staged M2L lists, bit 1 near field after
                                   // S2M, bit 2 two side streams for the finer levels' M2L, bit 3
                                   // chain kernels as programmatic dependent launches
    int m2m_staged, l2l_staged;    // one-vector: bit p = transition p -> p + 1 on the staged kernels
    int near_kernel;               // one-vector near field: 0 k_near_sym, 1 k_near_warp
};

// Tensor-core interpolation and anterpolation of one level transition
// (complex-float far field; kernels_tc.cuh): per pass (THETA, PHI, PHI_T,
// THETA_T) the dense weight matrix split hi + lo in the MMA's canonical layout,
// its contraction length K (reflected source rows included) and output count
// N, both padded, and for the theta passes the source row of every
// contraction index.
struct TcTrans {
    float* w[4] = {};
    int K[4] = {}, Kpad[4] = {}, N[4] = {}, Npad[4] = {};
    int* krow[4] = {};
    size_t smem[4] = {};
    int grid[4] = {};
};

struct StageTimes {
    float gather, s2m, m2m, m2l, l2l, l2t, near, finish, total;
};

// Far-field data in one precision.
template <class R>
struct FarField {
    using C = typename Cx<R>::T;
    DevLevelT<R> lv[kMaxLevels] = {};
    DevLevelT<R>* lv_dev = nullptr;
    std::vector<DevTransT<R>> trans;  // index = parent level
    C* pat = nullptr;                 // radiation patterns [pat_elems][2] (FP64; many right-hand sides)
    C* hpat = nullptr;                // complex float: directions d < ndir/2 of each source, [pat_elems / 2][2]
    C* m2l_t8 = nullptr;              // many-rhs M2L: pre-gathered weighted transfer values
};

class DeviceOp {
public:
    DeviceOp() = default;
    ~DeviceOp();
    DeviceOp(const DeviceOp&) = delete;
    DeviceOp& operator=(const DeviceOp&) = delete;

    // Uploads the plan and assembles radiation patterns and near-field blocks.
    // max_rhs > 1 also allocates the work space of products on up to max_rhs
    // right-hand sides at once.
    std::string setup(const Plan& plan, int device, int precision, int max_rhs = 1);

    // y (user order) = (accumulate ? y : 0) + A x, device pointers, on `stream`
    // (0 = the operator's own stream).  Interleaved complex FP64.
    // prec: far-field precision (-1 = the operator's own; a mixed operator
    // also carries the FP64 far field).
    // adj: y = A^H x (needs ref_compat = 0).
    std::string matvec_device(const double2* x, double2* y, bool accumulate, cudaStream_t stream, int prec = -1,
                              bool adj = false);
    // The same product on host buffers the device can address (pinned,
    // mapped; device-side addresses of them): the gather kernel reads x and
    // the finishing kernel writes y in caller order straight over the bus
    // (coalesced), no separate copies.
    std::string matvec_mapped(const double2* x, double2* y, bool accumulate, cudaStream_t stream);

    // Non-empty when a kernel of this operator gave up a bounded wait (its
    // results since then are not valid); read after the stream is synchronised.
    std::string device_error() const;

    // Operator on tree-ordered device vectors (used by the solver).
    void apply_tree(const double2* xt, double2* yt, cudaStream_t s, int prec = -1, bool adj = false);
    // Same, never capturing a graph (launches the captured one if it exists).
    void apply_tree_direct(const double2* xt, double2* yt, cudaStream_t s, int prec = -1, bool adj = false);
    // The product of what is already in the operator's input buffer (xt_buffer(),
    // tree order; for the adjoint it holds conj(x)) into yt, with plain
    // launches (for capture into a solver's step graph).
    void enqueue_apply_from_input(double2* yt, cudaStream_t s, int prec, bool adj);
    double2* input_buffer() const { return xt_; }
    // Changes whenever something a captured product depends on changes
    // (loads, launch shapes, kernel choice).
    int generation() const { return generation_; }

    // Diagonal loads z (host, caller order, n complex) added to the operator:
    // A x + z .* x (A^H x + conj(z) .* x for the adjoint).  nullptr removes them.
    std::string set_loads(const double2* z_user);
    bool ref_compat() const { return ref_compat_ != 0; }
    const DevSources& sources() const { return src_; }
    double2 ck() const { return ck_; }

    // Products on nr right-hand sides at once (1 <= nr <= max_rhs).  x and y are
    // nr vectors one after another in the caller's order ([nr][n]).
    std::string matvec_multi_device(const double2* x, double2* y, int nr, bool accumulate, cudaStream_t stream,
                                    int prec = -1);
    // Tree order, right-hand side innermost ([n][nr]), for the solver.
    void apply_tree_multi(const double2* xt, double2* yt, int nr, cudaStream_t s, int prec = -1);
    int max_rhs() const { return max_rhs_; }

    // One product on caller-order device vectors, recorded on stream s with
    // plain launches (for a capture that holds many operators' products).
    void enqueue_matvec(const double2* x, double2* y, cudaStream_t s);

    // Per-stage CUDA-event timing of one matvec on the operator's stream.
    std::string time_stages(StageTimes* out);
    // bit 0: every transition's M2M on k_m2m_sum, bit 1: L2L on k_l2l_st (where they fit)
    std::string set_staged(int mode);
    std::string set_schedule(int schedule);
    std::string set_near_kernel(int kind);  // 0 k_near_sym, 1 k_near_warp
    // per level l (index l): M2M into l, M2L at l, L2L out of l (ms; 0 where none)
    std::string time_levels(std::vector<float>& out);
    // Chooses launch shapes by timing them on this operator (see kernels.cu).
    std::string autotune(int nr, int reps, TuneReport* rep);
    // Same for a product on nr right-hand sides.
    std::string time_stages_multi(int nr, StageTimes* out);

    // Far field of currents (caller order, device) along ndir unit directions
    // (device, ndir x 3); out: ndir x 3 complex (device).
    std::string farfield(const double2* cur, int ndir, const double* khat, double2* out, cudaStream_t s);
    // y[i] = (A x)[row i] with every interaction evaluated directly (rows: tree slots).
    std::string dense_rows(const int* rows, int nrows, const double2* x, double2* y, cudaStream_t s);
    // Its adjoint: g (caller order, device, n) = M^H F for F (device, ndir x 3);
    // work: ndir x 3 complex (device).
    std::string farfield_adjoint(const double2* F, int ndir, const double* khat, double2* g, cudaStream_t s,
                                 double2* work);
    // out[i * ld + j] = A[row i][column j] (caller order), every interaction
    // evaluated directly (rows: tree slots).
    std::string dense_block(const int* rows, int nrows, double2* out, long long ld, cudaStream_t s);

    int n() const { return n_; }
    int precision() const { return precision_; }
    cudaStream_t stream() const { return stream_; }
    const int* perm() const { return perm_; }
    int device() const { return device_; }
    long long bytes_allocated() const { return bytes_; }
    int launches_per_matvec() const;

    // Interpolation and anterpolation of the complex-float far field on the
    // tensor cores (bit 0: one right-hand side, bit 1: many); false when the
    // operator has no complex-float far field or a grid is too large for them.
    bool tc_available() const { return tc_ok_; }
    // mode bit 0: one-vector M2M, bit 1: many-rhs M2M, bit 2: one-vector L2L,
    // bit 3: many-rhs L2L on the tensor cores.
    std::string set_tc(int mode);
    int tc_mode() const { return tc_mode_; }

    // Leaf block-Jacobi right preconditioner M (the diagonal blocks of A,
    // loads included): built for the current loads on first use; y = M^{-1} x
    // on tree-ordered device vectors.
    std::string bj_prepare();
    void bj_apply(const double2* x, double2* y, cudaStream_t s);

    // The level's FP64 transfer functions as built on the GPU, [316][ndir].
    std::string copy_transl(int level, double2* host);

    // Diagnostic copies of per-level patterns (level, which: 0 outgoing, 1 local),
    // widened to complex double.
    std::string copy_level(int level, int which, double2* host, long long count);

    // Algorithmic byte counts per stage for one matvec (roofline accounting).
    struct Traffic { double s2m, m2m, m2l, l2l, l2t, near, total; };
    Traffic traffic() const { return traffic_; }

private:
    template <class T> T* alloc(size_t count);
    template <class T> T* upload(const std::vector<T>& v);
    template <class R> std::string setup_far(const Plan& plan, FarField<R>& F, const double2* pat64);
    template <class R, bool TR> void run_far_t(FarField<R>& F, const double2* xt, cudaStream_t s, int stage);
    template <class R, bool TR> void run_far_overlap_t(FarField<R>& F, const double2* xt, cudaStream_t s,
                                                       cudaStream_t s2, bool near_late);
    void run_far_overlap(const double2* xt, cudaStream_t s, cudaStream_t s2, int prec, bool tr, bool late);
    // pdl: launched as a programmatic dependent launch (the predecessor on s
    // is a kernel of the chain, and the only one this launch depends on)
    template <class R, bool TR> void far_s2m(FarField<R>& F, const double2* xt, cudaStream_t s);
    template <class R, bool TR> void far_m2m(FarField<R>& F, int p, cudaStream_t s, bool pdl = false);
    template <class R, bool TR> void far_m2l(FarField<R>& F, int lo, int hi, cudaStream_t s, bool pdl = false);
    template <class R, bool TR> void far_l2l(FarField<R>& F, int p, cudaStream_t s, bool pdl = false);
    template <class R, bool TR> void far_l2t(FarField<R>& F, cudaStream_t s, bool pdl = false);
    void run_far(const double2* xt, cudaStream_t s, int stage = -1, int prec = -1, bool tr = false);
    void run_near(const double2* xt, cudaStream_t s);
    void enqueue_core(cudaStream_t s, int prec, bool tr);   // xt_ -> yfar_, ynear_
    void launch_core(cudaStream_t s, int prec, bool tr);
    template <class R> void run_far_multi_t(FarField<R>& F, int nr, cudaStream_t s, int stage);
    void run_far_multi(int nr, cudaStream_t s, int stage, int prec);
    void run_near_multi(int nr, cudaStream_t s);
    void enqueue_multi(int nr, cudaStream_t s, int prec);  // xtm_ -> yfarm_, ynearm_
    std::string setup_multi(const Plan& plan);
    std::string build_m2l_groups(const Plan& plan);
    size_t m2l_item_capacity(int min_chunk) const;
    void build_m2l_items(int max_chunk);
    std::string ensure_graph(int prec, bool tr);
    std::string setup_tc(const Plan& plan);
    std::string build_transl_device(const Level& L, double2* t);
    void far_m2m_tc(int p, int nr, cudaStream_t s);
    void far_l2l_tc(int p, int nr, cudaStream_t s);
    void drop_graphs();
    static int m2m_rows(int nth, int nph);

    int device_ = 0;
    int n_ = 0;
    int precision_ = kFp64;
    bool ready_ = false;
    cudaStream_t stream_ = nullptr, side_ = nullptr, side2_ = nullptr, side3_ = nullptr;
    cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr, ev_m2l_done_ = nullptr, ev_m2l_done2_ = nullptr;
    cudaEvent_t ev_level_[kMaxLevels] = {};  // outgoing patterns of a level final
    std::vector<void*> allocs_;
    long long bytes_ = 0;
    cudaGraph_t graph_[2][2] = {};          // per far-field precision, forward / transposed
    cudaGraphExec_t graph_exec_[2][2] = {};
    bool use_graph_ = true;

    // Shared by both precisions.
    int lmin_ = 2, lmax_ = 0, ref_compat_ = 1;
    int plan_order_ = 3;      // interp_order (2 order interpolation points)
    double wavenum_ = 0;
    int nbox_[kMaxLevels] = {}, ndir_[kMaxLevels] = {}, nth_[kMaxLevels] = {}, nph_[kMaxLevels] = {};
    int4* m2l_items_ = nullptr;          // (level, box, first direction, count)
    int n_m2l_items_ = 0;
    int m2l_first_[kMaxLevels] = {}, m2l_count_[kMaxLevels] = {};  // items of each level
    std::vector<char> m2l_has_list_[kMaxLevels];  // box has a non-empty list 2
    std::vector<int> m2l_len_[kMaxLevels];         // per level and box: list-2 length
    // Launch shapes (defaults at setup; mlfma_autotune may change them).
    int m2l_chunk_ = 128;                 // one-vector M2L directions per block
    int m2l_staged_ = 1;                  // one-vector M2L with its lists staged in shared memory
    bool near_late_ = false;              // near field after S2M (overlapping the latency-bound stages)
    int m2l_streams_ = 1;                 // side streams for the finer levels' translations
    bool chain_pdl_ = false;              // far-field chain kernels as programmatic dependent launches
    std::vector<int> m2m_rows_;           // one-vector M2M parent rows per block, per transition
    std::vector<int> m2m_pref_, l2l_pref_;  // per transition: 1 = staged kernels (k_m2m_sum, k_l2l_st) where they fit
    int dev_smem_ = 0;                    // opt-in shared memory per block
    int near_kernel_ = 0;                 // one-vector near field: 0 k_near_sym, 1 k_near_warp, 2 k_near_direct
    int near_direct_occ_ = 1;             // k_near_direct blocks per SM
    int m_m2m_rows_fast_ = -1;            // many-rhs M2M grid order (-1: precision default)
    int m_l2l_pairs_ = 0;                 // many-rhs L2L column pairs per block (0: precision default)
    std::vector<int2*> l2l_pairs_;       // per parent level: (parent, child entry)
    std::vector<int> n_l2l_pairs_, npar_, up_w_, dn_w_;
    int4* s2m_items_ = nullptr;          // (leaf, first element, element count)
    int n_s2m_items_ = 0;
    int4* s2m_items_h_ = nullptr;        // the same over the stored half (half patterns)
    int n_s2m_items_h_ = 0;
    int4* l2t_items_ = nullptr;          // (leaf, first source, source count)
    int n_l2t_items_ = 0;
    int max_src_ = 0;                    // largest far leaf
    int max_leaf_ndir_ = 0;              // most directions on a level holding far leaves
    bool far_covers_all_ = false;        // every source sits in a far leaf (L2T writes all of yfar_)
    DevFarLeaf* leaves_ = nullptr;
    int n_leaves_ = 0;
    FarField<double> f64_;
    FarField<float> f32_;

    // Near field, one vector: the stored blocks (each interaction once) applied
    // as Z and Z^T tile by tile, partial sums added per target.
    DevNearTile* near_tiles_ = nullptr;
    int n_near_tiles_ = 0;
    double2* near_bz_ = nullptr;          // block entries
    long long near_block_entries_ = 0;
    double2* near_part_ = nullptr;        // partial sums (near_parts)
    int near_grid_ = 0;                   // persistent blocks of k_near_sym
    int near_occ_ = 0;                    // its resident blocks per SM at most (occupancy)
    int near_per_sm_ = 0, sms_ = 0;       // its blocks per SM (the bound, or tuned) and the SM count
    void set_near_grid(int per_sm);
    int* err_host_ = nullptr;             // error word in mapped host memory
    int* err_dev_ = nullptr;              //   and its device address
    int* near_slot_ = nullptr;            // per tile: slots of its partials
    int* near_red_ptr_ = nullptr;         // [n + 1]: target t's slots
    // Near field, many right-hand sides: block rows (both orientations).
    DevNearRow* near_rows_ = nullptr;
    int n_near_rows_ = 0;
    int* near_cols_ = nullptr;
    double2* near_z_ = nullptr;
    long long near_entries_ = 0;

    int* perm_ = nullptr;
    int* tpos_ = nullptr;  // inverse of perm_: caller index -> tree position
    DevSources src_{};         // source geometry (setup kernels, far field)
    double2* xt_ = nullptr;    // tree-ordered input
    double2* yfar_ = nullptr;  // tree-ordered far result (before C k)
    double2* ynear_ = nullptr; // tree-ordered near result (before C k)
    double2* yt_ = nullptr;    // tree-ordered total (stage timing)
    // Many right-hand sides ([n][max_rhs], tree order) and their work items.
    int max_rhs_ = 1;
    double2* xtm_ = nullptr;
    double2* yfarm_ = nullptr;
    double2* ynearm_ = nullptr;
    double2* ytm_ = nullptr;
    int2* s2m_items_m_ = nullptr;
    int n_s2m_items_m_ = 0;
    int2* l2t_items_m_ = nullptr;
    int n_l2t_items_m_ = 0;
    int2* near_items_m_ = nullptr;
    int n_near_items_m_ = 0;
    DevM2LGroup* m2l_groups_ = nullptr;   // M2L sibling groups (many-rhs path)
    std::vector<DevM2LGroup> h_groups_;
    std::vector<short> h_cand_off_;        // [candidate][kMaxGroup] offset ids (-1: none)
    int* m2l_cand_src_ = nullptr;
    int2* m2l_items_m_ = nullptr;
    int n_m2l_items_m_ = 0;
    // Tensor-core interpolation (complex-float far field), per transition.
    std::vector<TcTrans> tc_;
    float* tc_scratch_ = nullptr;       // intermediate of the two passes of a stage
    size_t tc_scratch_floats_ = 0;
    bool tc_ok_ = false;
    int tc_mode_ = 0;  // see set_tc
    int generation_ = 0;
    // Leaf block-Jacobi preconditioner
    std::vector<DevBjLeaf> h_bj_;
    DevBjLeaf* bj_leaves_ = nullptr;
    int* bj_ok_ = nullptr;
    double2* bj_inv_ = nullptr;
    int bj_gen_ = -1;
    double2 ck_{};             // Phys::C * k
    double2* loads_ = nullptr; // diagonal loads, tree order
    bool has_loads_ = false;
    Traffic traffic_{};
};

}  // namespace mlfma
