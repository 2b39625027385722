// Device-side plan: flat arrays in HBM that the kernels read, and the launch
// wrappers.  One DeviceOp per operator handle.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "plan.hpp"

namespace mlfma {

constexpr int kMaxLevels = 20;
constexpr int kM2MThreads = 256;  // threads per M2M block
constexpr int kM2MOut = 8;        // parent outputs per thread (registers)

struct DevLevel {
    int nth, nph, ndir, nbox;
    double2* A;                  // outgoing patterns [nbox][ndir][2]
    double2* B;                  // local (incoming) patterns [nbox][ndir][2]
    const double2* transl;       // [316][ndir]
    const double* w;             // [ndir] quadrature weight applied after M2L
    const double2* shift_up;     // [8][ndir]
    const double2* shift_down;   // [8][ndir]
    const double* thph;          // [ndir][6]
    const double* khat;          // [ndir][3]
    const int* m2l_ptr;          // [nbox+1]
    const int* m2l_src;
    const int* m2l_off;
};

struct DevLevels {
    DevLevel lv[kMaxLevels];
    int lmin, lmax;
    double k;
    int ref_compat;
};

// Stencil rows padded to a fixed width (padding entries have coefficient 0):
// entry k of row r is at r * width + k.  The sign of a pole-reflected tap is
// folded into its coefficient.
struct DevStencil {
    int width;
    const int* src;
    const int* refl;
    const double* coef;
};

struct DevTrans {
    DevStencil up_th, up_ph, dn_ph, dn_th;
    int plevel, npar;
    const int* par_box;
    const int* par_ilist;
    const int* child_ptr;
    const int* child_box;
    const int* child_oct;
};

struct DevFarLeaf {
    int level, box, src0, nsrc;
    long long pat_off;
};

struct DevNearBlock {
    int row0, nrow, col0, ncol;
    long long off;
    int self, pad;
};

struct DevNearRow {
    int row0, nrow, ncol, pad;
    long long off, col_off;
};

struct StageTimes {
    float gather, s2m, m2m, m2l, l2l, l2t, near, finish, total;
};

class DeviceOp {
public:
    DeviceOp() = default;
    ~DeviceOp();
    DeviceOp(const DeviceOp&) = delete;
    DeviceOp& operator=(const DeviceOp&) = delete;

    // Uploads the plan and assembles radiation patterns and near-field blocks.
    std::string setup(const Plan& plan, int device);

    // y (user order) = (accumulate ? y : 0) + A x, device pointers, on `stream`
    // (0 = the operator's own stream).  Interleaved complex FP64.
    std::string matvec_device(const double2* x, double2* y, bool accumulate, cudaStream_t stream);

    // Operator on tree-ordered device vectors (used by the solver).
    void apply_tree(const double2* xt, double2* yt, cudaStream_t s);
    // Same, never capturing a graph (launches the captured one if it exists).
    void apply_tree_direct(const double2* xt, double2* yt, cudaStream_t s);

    // Per-stage CUDA-event timing of one matvec on the operator's stream.
    std::string time_stages(StageTimes* out);

    int n() const { return n_; }
    cudaStream_t stream() const { return stream_; }
    double2* scratch_x() { return xt_; }
    double2* scratch_y() { return yfar_; }
    const int* perm() const { return perm_; }
    int device() const { return device_; }
    long long bytes_allocated() const { return bytes_; }
    int launches_per_matvec() const;
    const std::vector<DevFarLeaf>& far_leaves_host() const { return h_leaves_; }

    // Diagnostic copies of per-level patterns (level, which: 0 outgoing, 1 local).
    std::string copy_level(int level, int which, double2* host, long long count);

    // Algorithmic byte counts per stage for one matvec (roofline accounting).
    struct Traffic { double s2m, m2m, m2l, l2l, l2t, near, total; };
    Traffic traffic() const { return traffic_; }

private:
    template <class T> T* alloc(size_t count);
    template <class T> T* upload(const std::vector<T>& v);
    void run_far(const double2* xt, cudaStream_t s);
    void run_near(const double2* xt, cudaStream_t s);

    int device_ = 0;
    int n_ = 0;
    bool ready_ = false;
    cudaStream_t stream_ = nullptr, side_ = nullptr;
    cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;
    std::vector<void*> allocs_;
    long long bytes_ = 0;

    static int m2m_rows(int nth, int nph);
    void stage_s2m(const double2* xt, cudaStream_t s);
    void stage_m2m(cudaStream_t s);
    void stage_m2l(cudaStream_t s);
    void stage_l2l(cudaStream_t s);
    void stage_l2t(cudaStream_t s);
    void enqueue_core(cudaStream_t s);   // xt_ -> yfar_, ynear_
    std::string ensure_graph();

    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
    bool use_graph_ = true;

    DevLevels lv_{};
    DevLevel* lv_dev_ = nullptr;        // device copy of lv_.lv
    std::vector<DevTrans> trans_;       // index = parent level
    int4* m2l_items_ = nullptr;         // (level, box, first direction, count)
    int n_m2l_items_ = 0;
    std::vector<int2*> l2l_pairs_;      // per parent level: (parent, child entry)
    std::vector<int> n_l2l_pairs_;
    int4* s2m_items_ = nullptr;          // (leaf, first element, element count)
    int n_s2m_items_ = 0;
    int4* l2t_items_ = nullptr;          // (leaf, first source, source count)
    int n_l2t_items_ = 0;
    int max_src_ = 0;                    // largest far leaf
    DevFarLeaf* leaves_ = nullptr;
    std::vector<DevFarLeaf> h_leaves_;
    int n_leaves_ = 0;
    double2* pat_ = nullptr;            // [pat_elems][2]
    DevNearBlock* near_blocks_ = nullptr;
    int n_near_blocks_ = 0;
    double2* near_z_ = nullptr;
    long long near_entries_ = 0;
    DevNearRow* near_rows_ = nullptr;   // block rows (device storage of the near field)
    int n_near_rows_ = 0;
    int* near_cols_ = nullptr;
    int4* near_items_ = nullptr;        // (row block, first row, row count)
    int n_near_items_ = 0;
    int* perm_ = nullptr;
    double2* xt_ = nullptr;    // tree-ordered input
    double2* yfar_ = nullptr;  // tree-ordered far result (before C k)
    double2* ynear_ = nullptr; // tree-ordered near result (before C k)
    double2* yt_ = nullptr;    // tree-ordered total (solver use)
    double2 ck_{};             // Phys::C * k
    int max_ndir_ = 0;
    Traffic traffic_{};
};

}  // namespace mlfma
