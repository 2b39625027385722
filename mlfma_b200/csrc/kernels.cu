// The device operator: uploads the host plan, assembles the radiation
// patterns and near-field blocks, and launches the MLFMA matvec
// (kernels in kernels_far.cuh and kernels_near.cuh).
//
// Data layout in HBM (all complex values interleaved re/im, double2):
//   * sources are permuted into tree order so every octree box owns a
//     contiguous range; x and y are gathered/scattered at the boundary;
//   * per level l: outgoing patterns A_l and local patterns B_l as
//     [box][direction][2 polarisation components];
//   * radiation patterns as [source][direction of its leaf level][2];
//   * transfer functions as [316 offsets][direction] per level;
//   * near-field blocks dense row-major (list 1 and list 3/4 pairs) or
//     strict-lower packed (self blocks), each applied as Z and Z^T.
//
// One matvec: the near field runs on a side stream while the far-field chain
// S2M -> M2M (fine to coarse) -> M2L (all levels) -> L2L (coarse to fine) ->
// L2T runs on the caller's stream; a final kernel combines both.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

#include "device.cuh"
#include "kernels_far.cuh"
#include "kernels_near.cuh"
#include "zmath.cuh"

namespace mlfma {

#define MLFMA_CK(call)                                                                  \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return std::string(#call) + ": " + cudaGetErrorString(e_);                  \
    } while (0)

namespace {

__global__ void k_gather(const double2* __restrict__ x, const int* __restrict__ perm,
                         double2* __restrict__ xt, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) xt[t] = x[perm[t]];
}

// y[perm[t]] (+)= ck * (yfar[t] + ynear[t]); perm == nullptr keeps tree order.
__global__ void k_finish(const double2* __restrict__ yfar, const double2* __restrict__ ynear,
                         const int* __restrict__ perm, double2* __restrict__ y, int n, double2 ck,
                         int accumulate) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double2 v = cmul(ck, cadd(yfar[t], ynear[t]));
    const int o = perm ? perm[t] : t;
    y[o] = accumulate ? cadd(y[o], v) : v;
}

inline int blocks_for(long long n, int bs) { return static_cast<int>((n + bs - 1) / bs); }

}  // namespace

// ================================================================= DeviceOp

DeviceOp::~DeviceOp() {
    if (device_ >= 0) cudaSetDevice(device_);
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (graph_) cudaGraphDestroy(graph_);
    for (void* p : allocs_) cudaFree(p);
    if (ev_fork_) cudaEventDestroy(ev_fork_);
    if (ev_join_) cudaEventDestroy(ev_join_);
    if (stream_) cudaStreamDestroy(stream_);
    if (side_) cudaStreamDestroy(side_);
}

template <class T>
T* DeviceOp::alloc(size_t count) {
    void* p = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    if (cudaMalloc(&p, bytes) != cudaSuccess) throw std::runtime_error("cudaMalloc failed");
    allocs_.push_back(p);
    bytes_ += static_cast<long long>(bytes);
    return static_cast<T*>(p);
}

template <class T>
T* DeviceOp::upload(const std::vector<T>& v) {
    T* p = alloc<T>(v.size());
    if (!v.empty() && cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("cudaMemcpy failed");
    return p;
}

static std::vector<double2> to_d2(const std::vector<cplx>& v) {
    std::vector<double2> o(v.size());
    for (size_t i = 0; i < v.size(); ++i) o[i] = make_double2(v[i].real(), v[i].imag());
    return o;
}

int DeviceOp::m2m_rows(int nth, int nph) {
    // about one parent output per thread of a 128-thread block
    return std::max(1, std::min(nth, 128 / std::max(nph, 1)));
}

std::string DeviceOp::setup(const Plan& plan, int device) {
    try {
        device_ = device;
        MLFMA_CK(cudaSetDevice(device));
        MLFMA_CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        MLFMA_CK(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
        MLFMA_CK(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
        MLFMA_CK(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming));
        n_ = plan.n;
        if (plan.max_level >= kMaxLevels) return "tree deeper than supported";
        const cplx ck = cplx(0, -kC0 * kMu0 / (4.0 * kPi)) * plan.pw.wavenum;
        ck_ = make_double2(ck.real(), ck.imag());
        perm_ = upload(plan.perm);
        xt_ = alloc<double2>(n_);
        yfar_ = alloc<double2>(n_);
        ynear_ = alloc<double2>(n_);
        yt_ = alloc<double2>(n_);

        // ---- levels
        std::memset(&lv_, 0, sizeof(lv_));
        lv_.lmin = plan.lmin;
        lv_.lmax = plan.max_level;
        lv_.k = plan.pw.wavenum;
        lv_.ref_compat = plan.cfg.ref_compat;
        traffic_ = Traffic{};
        std::vector<int4> items;
        for (int l = plan.lmin; l <= plan.max_level; ++l) {
            const Level& L = plan.levels[l];
            DevLevel& d = lv_.lv[l];
            d.nth = L.nth;
            d.nph = L.nph;
            d.ndir = L.ndir;
            d.nbox = static_cast<int>(L.boxes.size());
            const size_t cnt = static_cast<size_t>(d.nbox) * L.ndir * 2;
            d.A = alloc<double2>(cnt);
            d.B = alloc<double2>(cnt);
            MLFMA_CK(cudaMemset(d.A, 0, cnt * sizeof(double2)));
            MLFMA_CK(cudaMemset(d.B, 0, cnt * sizeof(double2)));
            d.transl = upload(to_d2(L.transl));
            d.w = upload(L.m2l_w);
            d.shift_up = upload(to_d2(L.shift_up));
            d.shift_down = upload(to_d2(L.shift_down));
            d.thph = upload(L.thph);
            d.khat = upload(L.khat);
            d.m2l_ptr = upload(L.m2l_ptr);
            d.m2l_src = upload(L.m2l_src);
            d.m2l_off = upload(L.m2l_off);
            max_ndir_ = std::max(max_ndir_, L.ndir);
            // M2L reads every source box's pattern and the transfer table once
            // (repeats hit L2) and writes every local pattern once.
            traffic_.m2l += static_cast<double>(cnt) * 16.0 * 2.0 + 316.0 * L.ndir * 16.0;
            // M2L work items: direction chunks of at most 128 of equal size.
            const int nchunk = (L.ndir + 127) / 128;
            const int chunk = (L.ndir + nchunk - 1) / nchunk;
            for (int b = 0; b < d.nbox; ++b) {
                if (plan.cfg.ref_compat && L.m2l_ptr[b + 1] == L.m2l_ptr[b]) continue;
                for (int d0 = 0; d0 < L.ndir; d0 += chunk) items.push_back(make_int4(l, b, d0, std::min(chunk, L.ndir - d0)));
            }
        }
        lv_dev_ = upload(std::vector<DevLevel>(lv_.lv, lv_.lv + kMaxLevels));
        n_m2l_items_ = static_cast<int>(items.size());
        m2l_items_ = upload(items);

        // ---- transitions
        trans_.assign(std::max(plan.max_level, 0) + 1, DevTrans{});
        l2l_pairs_.assign(std::max(plan.max_level, 0) + 1, nullptr);
        n_l2l_pairs_.assign(std::max(plan.max_level, 0) + 1, 0);
        size_t m2m_smem = 0, l2l_smem = 0;
        for (int p = plan.lmin; p < plan.max_level; ++p) {
            const Transition& T = plan.trans[p];
            DevTrans& d = trans_[p];
            auto width_of = [](const Stencil& s) {
                int w = 1;
                for (size_t r = 0; r + 1 < s.ptr.size(); ++r) w = std::max(w, s.ptr[r + 1] - s.ptr[r]);
                return w;
            };
            // The kernels are instantiated for fixed tap counts (fully unrolled).
            const int w_up = width_of(T.up_th);
            if (w_up != width_of(T.up_ph) || w_up % 2 || w_up < 2 || w_up > 10)
                return "interp_order must be 1..5";
            const int w_dn_need = std::max(width_of(T.dn_ph), width_of(T.dn_th));
            int w_dn = 0;
            for (int c : {8, 12, 16, 24, 32})
                if (!w_dn && w_dn_need <= c) w_dn = c;
            if (!w_dn) return "anterpolation stencil wider than 32 taps";
            auto st = [&](const Stencil& s, int wpad) {
                // pad rows to a fixed width; fold the reflection sign into the coefficient
                const int rows = static_cast<int>(s.ptr.size()) - 1;
                const int w = wpad;
                std::vector<int> src(static_cast<size_t>(rows) * w, 0), refl(static_cast<size_t>(rows) * w, 0);
                std::vector<double> coef(static_cast<size_t>(rows) * w, 0.0);
                for (int r = 0; r < rows; ++r)
                    for (int q = s.ptr[r]; q < s.ptr[r + 1]; ++q) {
                        const size_t at = static_cast<size_t>(r) * w + (q - s.ptr[r]);
                        src[at] = s.src[q];
                        refl[at] = s.refl[q];
                        coef[at] = s.refl[q] ? -s.coef[q] : s.coef[q];
                    }
                return DevStencil{w, upload(src), upload(refl), upload(coef)};
            };
            d.up_th = st(T.up_th, w_up);
            d.up_ph = st(T.up_ph, w_up);
            d.dn_ph = st(T.dn_ph, w_dn);
            d.dn_th = st(T.dn_th, w_dn);
            d.plevel = p;
            d.npar = static_cast<int>(T.par_box.size());
            d.par_box = upload(T.par_box);
            d.par_ilist = upload(T.par_ilist);
            d.child_ptr = upload(T.child_ptr);
            d.child_box = upload(T.child_box);
            d.child_oct = upload(T.child_oct);
            std::vector<int2> pairs;
            for (int q = 0; q < d.npar; ++q) {
                if (plan.cfg.ref_compat && !T.par_ilist[q]) continue;  // stem.cpp:115
                for (int c = T.child_ptr[q]; c < T.child_ptr[q + 1]; ++c) pairs.push_back(make_int2(q, c));
            }
            n_l2l_pairs_[p] = static_cast<int>(pairs.size());
            l2l_pairs_[p] = upload(pairs);
            const Level& Lp = plan.levels[p];
            const Level& Lc = plan.levels[p + 1];
            const double nch = static_cast<double>(T.child_box.size());
            traffic_.m2m += nch * Lc.ndir * 32.0 + d.npar * Lp.ndir * 32.0;
            traffic_.l2l += d.npar * Lp.ndir * 32.0 + nch * Lc.ndir * 32.0 * 2.0;
            m2m_smem = std::max(m2m_smem, static_cast<size_t>(8) * m2m_rows(Lp.nth, Lp.nph) * Lc.nph * 2 * sizeof(double2));
            l2l_smem = std::max(l2l_smem, static_cast<size_t>(Lp.nth) * Lc.nph * 2 * sizeof(double2));
        }

        // ---- far leaves (grouped by level for S2M/L2T) and radiation patterns
        h_leaves_.clear();
        std::vector<DevFarLeafGeom> geo;
        std::vector<int4> s2m_items, l2t_items;
        max_src_ = 0;
        for (const FarLeaf& f : plan.far_leaves) {
            const DevFarLeaf dl{f.level, f.box, f.src0, f.nsrc, f.pat_off};
            h_leaves_.push_back(dl);
            const int li = static_cast<int>(h_leaves_.size()) - 1;
            const int ne = 2 * plan.levels[f.level].ndir;
            const int nchunk = (ne + kS2MThreads - 1) / kS2MThreads;
            const int chunk = (ne + nchunk - 1) / nchunk;
            for (int e0 = 0; e0 < ne; e0 += chunk) s2m_items.push_back(make_int4(li, e0, std::min(chunk, ne - e0), 0));
            for (int s0 = 0; s0 < f.nsrc; s0 += kL2TSrcPerBlock)
                l2t_items.push_back(make_int4(li, s0, std::min(kL2TSrcPerBlock, f.nsrc - s0), 0));
            max_src_ = std::max(max_src_, f.nsrc);
            const Node& nd = plan.nodes[plan.levels[f.level].boxes[f.box]];
            geo.push_back(DevFarLeafGeom{{nd.center[0], nd.center[1], nd.center[2]}});
        }
        n_s2m_items_ = static_cast<int>(s2m_items.size());
        s2m_items_ = upload(s2m_items);
        n_l2t_items_ = static_cast<int>(l2t_items.size());
        l2t_items_ = upload(l2t_items);
        n_leaves_ = static_cast<int>(h_leaves_.size());
        leaves_ = upload(h_leaves_);
        DevFarLeafGeom* d_geo = upload(geo);
        pat_ = alloc<double2>(static_cast<size_t>(plan.pat_elems) * 2);
        traffic_.s2m = plan.pat_elems * 32.0 + n_ * 16.0;
        traffic_.l2t = plan.pat_elems * 32.0 + n_ * 16.0;

        DevSources S{};
        S.kind = plan.kind;
        S.k = plan.pw.wavenum;
        if (plan.kind == kDipole) {
            S.pos = upload(plan.dip_pos);
            S.phat = upload(plan.dip_phat);
        } else {
            S.rwg = upload(plan.rwg);
            S.tris = upload(plan.tris);
            S.tri_quad = upload(plan.tri_quad);
            S.quad_w = upload(plan.quad_w);
            S.nq = plan.nq;
        }
        if (n_leaves_ > 0 && plan.kind == kRwg && plan.cfg.ref_compat) {
            // Reference-compatible RWG patterns: the closed-form integral is
            // ill-conditioned near alpha, beta, gamma = 0, so it is evaluated on
            // the host with the reference's exact rounding and uploaded.
            std::vector<cplx> hp;
            plan.rwg_patterns_host(hp);
            MLFMA_CK(cudaMemcpy(pat_, hp.data(), hp.size() * sizeof(cplx), cudaMemcpyHostToDevice));
        } else if (n_leaves_ > 0) {
            k_patterns<<<n_leaves_, 256, 0, stream_>>>(lv_dev_, leaves_, d_geo, S, pat_);
            MLFMA_CK(cudaGetLastError());
        }

        // ---- near field
        // Stored as block rows (both orientations): gather-only application.
        std::vector<DevNearRow> nr;
        std::vector<int4> nitems;
        for (const NearRow& r : plan.near_rows) {
            nr.push_back(DevNearRow{r.row0, r.nrow, r.ncol, 0, r.off, r.col_off});
            for (int i0 = 0; i0 < r.nrow; i0 += kNearRowsPerBlock)
                nitems.push_back(make_int4(static_cast<int>(nr.size()) - 1, i0, std::min(kNearRowsPerBlock, r.nrow - i0), 0));
        }
        n_near_rows_ = static_cast<int>(nr.size());
        near_rows_ = upload(nr);
        near_cols_ = upload(plan.near_cols);
        n_near_items_ = static_cast<int>(nitems.size());
        near_items_ = upload(nitems);
        near_entries_ = plan.near_row_entries;
        near_z_ = alloc<double2>(static_cast<size_t>(near_entries_));
        if (near_entries_ > 0) {
            k_near_rows_assemble<<<blocks_for(near_entries_, 128), 128, 0, stream_>>>(
                near_rows_, n_near_rows_, near_entries_, near_cols_, S, near_z_);
            MLFMA_CK(cudaGetLastError());
        }
        traffic_.near = near_entries_ * 16.0 + n_ * 16.0 * 2.0;
        traffic_.total = traffic_.s2m + traffic_.m2m + traffic_.m2l + traffic_.l2l + traffic_.l2t + traffic_.near;

        // Shared-memory limits.
        int dev_smem = 0;
        MLFMA_CK(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
        const size_t s2m_smem = static_cast<size_t>(std::max(1, max_src_)) * sizeof(double2);
        if (m2m_smem > static_cast<size_t>(dev_smem) || l2l_smem > static_cast<size_t>(dev_smem) ||
            s2m_smem > static_cast<size_t>(dev_smem))
            return "angular grid or leaf too large for the kernels' shared memory";
        {
            const int a = static_cast<int>(std::max<size_t>(m2m_smem, 1));
            const int b = static_cast<int>(std::max<size_t>(l2l_smem, 1));
            const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
            MLFMA_CK(cudaFuncSetAttribute(k_m2m<2>, attr, a));
            MLFMA_CK(cudaFuncSetAttribute(k_m2m<4>, attr, a));
            MLFMA_CK(cudaFuncSetAttribute(k_m2m<6>, attr, a));
            MLFMA_CK(cudaFuncSetAttribute(k_m2m<8>, attr, a));
            MLFMA_CK(cudaFuncSetAttribute(k_m2m<10>, attr, a));
            MLFMA_CK(cudaFuncSetAttribute(k_l2l<8>, attr, b));
            MLFMA_CK(cudaFuncSetAttribute(k_l2l<12>, attr, b));
            MLFMA_CK(cudaFuncSetAttribute(k_l2l<16>, attr, b));
            MLFMA_CK(cudaFuncSetAttribute(k_l2l<24>, attr, b));
            MLFMA_CK(cudaFuncSetAttribute(k_l2l<32>, attr, b));
        }
        MLFMA_CK(cudaFuncSetAttribute(k_s2m, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(std::max<size_t>(s2m_smem, 1))));
        MLFMA_CK(cudaStreamSynchronize(stream_));
        MLFMA_CK(cudaGetLastError());
        ready_ = true;
        return {};
    } catch (const std::exception& e) {
        return e.what();
    }
}

int DeviceOp::launches_per_matvec() const {
    int n = 2;  // gather + finish
    if (n_leaves_) {
        n += 2;  // S2M + L2T
        for (int p = lv_.lmin; p < lv_.lmax; ++p) {
            if (trans_[p].npar) n += 1;    // M2M
            if (n_l2l_pairs_[p]) n += 1;   // L2L
        }
        if (n_m2l_items_) n += 1;
    }
    if (n_near_items_) n += 1;
    return n;
}

void DeviceOp::stage_s2m(const double2* xt, cudaStream_t s) {
    if (n_s2m_items_)
        k_s2m<<<n_s2m_items_, kS2MThreads, sizeof(double2) * std::max(1, max_src_), s>>>(lv_dev_, s2m_items_, leaves_,
                                                                                         pat_, xt);
}

void DeviceOp::stage_m2m(cudaStream_t s) {
    for (int p = lv_.lmax - 1; p >= lv_.lmin; --p) {
        const DevTrans& T = trans_[p];
        if (T.npar == 0) continue;
        const DevLevel& P = lv_.lv[p];
        const DevLevel& C = lv_.lv[p + 1];
        const int rows = m2m_rows(P.nth, P.nph);
        const dim3 grid(T.npar, (P.nth + rows - 1) / rows);
        const size_t smem = static_cast<size_t>(8) * rows * C.nph * 2 * sizeof(double2);
        switch (T.up_th.width) {
            case 2: k_m2m<2><<<grid, 128, smem, s>>>(lv_dev_, T, rows); break;
            case 4: k_m2m<4><<<grid, 128, smem, s>>>(lv_dev_, T, rows); break;
            case 6: k_m2m<6><<<grid, 128, smem, s>>>(lv_dev_, T, rows); break;
            case 8: k_m2m<8><<<grid, 128, smem, s>>>(lv_dev_, T, rows); break;
            default: k_m2m<10><<<grid, 128, smem, s>>>(lv_dev_, T, rows); break;
        }
    }
}

void DeviceOp::stage_m2l(cudaStream_t s) {
    if (n_m2l_items_) k_m2l<<<n_m2l_items_, 128, 0, s>>>(lv_dev_, m2l_items_, lv_.ref_compat ? 0 : 1);
}

void DeviceOp::stage_l2l(cudaStream_t s) {
    for (int p = lv_.lmin; p < lv_.lmax; ++p) {
        if (!n_l2l_pairs_[p]) continue;
        const size_t smem = static_cast<size_t>(lv_.lv[p].nth) * lv_.lv[p + 1].nph * 2 * sizeof(double2);
        const int g = n_l2l_pairs_[p];
        switch (trans_[p].dn_ph.width) {
            case 8: k_l2l<8><<<g, 256, smem, s>>>(lv_dev_, trans_[p], l2l_pairs_[p]); break;
            case 12: k_l2l<12><<<g, 256, smem, s>>>(lv_dev_, trans_[p], l2l_pairs_[p]); break;
            case 16: k_l2l<16><<<g, 256, smem, s>>>(lv_dev_, trans_[p], l2l_pairs_[p]); break;
            case 24: k_l2l<24><<<g, 256, smem, s>>>(lv_dev_, trans_[p], l2l_pairs_[p]); break;
            default: k_l2l<32><<<g, 256, smem, s>>>(lv_dev_, trans_[p], l2l_pairs_[p]); break;
        }
    }
}

void DeviceOp::stage_l2t(cudaStream_t s) {
    if (n_l2t_items_) k_l2t<<<n_l2t_items_, kL2TThreads, 0, s>>>(lv_dev_, l2t_items_, leaves_, pat_, yfar_);
}

void DeviceOp::run_far(const double2* xt, cudaStream_t s) {
    if (n_leaves_ == 0) return;
    stage_s2m(xt, s);
    stage_m2m(s);
    stage_m2l(s);
    stage_l2l(s);
    stage_l2t(s);
}

void DeviceOp::run_near(const double2* xt, cudaStream_t s) {
    if (n_near_items_ == 0) return;
    k_near_rows<<<n_near_items_, kNearRowThreads, 0, s>>>(near_rows_, near_items_, near_z_, near_cols_, xt, ynear_);
}

// The tree-ordered product xt_ -> (yfar_, ynear_): near field on the side
// stream, far-field chain on s.  Captured once into a CUDA graph.
void DeviceOp::enqueue_core(cudaStream_t s) {
    cudaMemsetAsync(yfar_, 0, sizeof(double2) * n_, s);
    cudaMemsetAsync(ynear_, 0, sizeof(double2) * n_, s);
    cudaEventRecord(ev_fork_, s);
    cudaStreamWaitEvent(side_, ev_fork_, 0);
    run_near(xt_, side_);
    cudaEventRecord(ev_join_, side_);
    run_far(xt_, s);
    cudaStreamWaitEvent(s, ev_join_, 0);
}

std::string DeviceOp::ensure_graph() {
    if (graph_exec_ || !use_graph_) return {};
    MLFMA_CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    enqueue_core(stream_);
    MLFMA_CK(cudaStreamEndCapture(stream_, &graph_));
    MLFMA_CK(cudaGraphInstantiate(&graph_exec_, graph_, 0));
    return {};
}

void DeviceOp::apply_tree(const double2* xt, double2* yt, cudaStream_t s) {
    if (!ensure_graph().empty()) use_graph_ = false;
    if (xt != xt_) cudaMemcpyAsync(xt_, xt, sizeof(double2) * n_, cudaMemcpyDeviceToDevice, s);
    if (graph_exec_) cudaGraphLaunch(graph_exec_, s); else enqueue_core(s);
    k_finish<<<blocks_for(n_, 256), 256, 0, s>>>(yfar_, ynear_, nullptr, yt, n_, ck_, 0);
}

void DeviceOp::apply_tree_direct(const double2* xt, double2* yt, cudaStream_t s) {
    if (xt != xt_) cudaMemcpyAsync(xt_, xt, sizeof(double2) * n_, cudaMemcpyDeviceToDevice, s);
    if (graph_exec_) cudaGraphLaunch(graph_exec_, s); else enqueue_core(s);
    k_finish<<<blocks_for(n_, 256), 256, 0, s>>>(yfar_, ynear_, nullptr, yt, n_, ck_, 0);
}

std::string DeviceOp::matvec_device(const double2* x, double2* y, bool accumulate, cudaStream_t stream) {
    if (!ready_) return "operator not set up";
    cudaStream_t s = stream ? stream : stream_;
    MLFMA_CK(cudaSetDevice(device_));
    std::string e = ensure_graph();
    if (!e.empty()) return e;
    k_gather<<<blocks_for(n_, 256), 256, 0, s>>>(x, perm_, xt_, n_);
    if (graph_exec_) cudaGraphLaunch(graph_exec_, s); else enqueue_core(s);
    k_finish<<<blocks_for(n_, 256), 256, 0, s>>>(yfar_, ynear_, perm_, y, n_, ck_, accumulate ? 1 : 0);
    MLFMA_CK(cudaGetLastError());
    return {};
}

std::string DeviceOp::time_stages(StageTimes* out) {
    if (!ready_) return "operator not set up";
    MLFMA_CK(cudaSetDevice(device_));
    cudaEvent_t ev[9];
    for (auto& e : ev) MLFMA_CK(cudaEventCreate(&e));
    cudaStream_t s = stream_;
    cudaEventRecord(ev[0], s);
    cudaMemsetAsync(yfar_, 0, sizeof(double2) * n_, s);
    cudaMemsetAsync(ynear_, 0, sizeof(double2) * n_, s);
    cudaEventRecord(ev[1], s);
    if (n_leaves_) stage_s2m(xt_, s);
    cudaEventRecord(ev[2], s);
    if (n_leaves_) stage_m2m(s);
    cudaEventRecord(ev[3], s);
    if (n_leaves_) stage_m2l(s);
    cudaEventRecord(ev[4], s);
    if (n_leaves_) stage_l2l(s);
    cudaEventRecord(ev[5], s);
    if (n_leaves_) stage_l2t(s);
    cudaEventRecord(ev[6], s);
    run_near(xt_, s);
    cudaEventRecord(ev[7], s);
    k_finish<<<blocks_for(n_, 256), 256, 0, s>>>(yfar_, ynear_, nullptr, yt_, n_, ck_, 0);
    cudaEventRecord(ev[8], s);
    MLFMA_CK(cudaEventSynchronize(ev[8]));
    float t[8];
    for (int i = 0; i < 8; ++i) cudaEventElapsedTime(&t[i], ev[i], ev[i + 1]);
    out->gather = t[0];
    out->s2m = t[1];
    out->m2m = t[2];
    out->m2l = t[3];
    out->l2l = t[4];
    out->l2t = t[5];
    out->near = t[6];
    out->finish = t[7];
    cudaEventElapsedTime(&out->total, ev[0], ev[8]);
    for (auto& e : ev) cudaEventDestroy(e);
    MLFMA_CK(cudaGetLastError());
    return {};
}

std::string DeviceOp::copy_level(int level, int which, double2* host, long long count) {
    if (level < lv_.lmin || level > lv_.lmax) return "level out of range";
    const DevLevel& d = lv_.lv[level];
    const long long cnt = static_cast<long long>(d.nbox) * d.ndir * 2;
    if (count < cnt) return "buffer too small";
    MLFMA_CK(cudaSetDevice(device_));
    MLFMA_CK(cudaStreamSynchronize(stream_));
    MLFMA_CK(cudaMemcpy(host, which ? d.B : d.A, cnt * sizeof(double2), cudaMemcpyDeviceToHost));
    return {};
}

}  // namespace mlfma
