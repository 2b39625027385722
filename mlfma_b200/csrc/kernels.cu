// The device operator: uploads the host plan, assembles the radiation
// patterns and near-field blocks, and launches the MLFMA matvec
// (kernels in kernels_far.cuh and kernels_near.cuh).
//
// Data layout in HBM (complex values interleaved re/im):
//   * sources are permuted into tree order so every octree box owns a
//     contiguous range; x and y are gathered/scattered at the boundary;
//   * per level l: outgoing patterns A_l and local patterns B_l as
//     [box][direction][2 polarisation components];
//   * radiation patterns as [source][direction of its leaf level][2];
//   * transfer functions as [316 offsets][direction] per level;
//   * the near field as the reference stores it, each interaction once
//     (rectangular blocks row-major, self blocks packed lower-triangular),
//     applied as Z and Z^T; with many right-hand sides also as block rows
//     (both orientations) with a shared column list per leaf.
// The far-field arrays are complex double (FP64 path) or complex float (mixed
// path); x, y and the near field are complex double in both.
//
// One matvec: the near field runs on a side stream while the far-field chain
// S2M -> M2M (fine to coarse) -> M2L (all levels) -> L2L (coarse to fine) ->
// L2T runs on the caller's stream; a final kernel combines both.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>

#include "device.cuh"
#include "kernels_far.cuh"
#include "kernels_multi.cuh"
#include "kernels_near.cuh"
#include "kernels_tables.cuh"
#include "kernels_tc.cuh"
#include "zmath.cuh"

namespace mlfma {

#define MLFMA_CK(call)                                                                  \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return std::string(#call) + ": " + cudaGetErrorString(e_);                  \
    } while (0)

namespace {

// Launch kernel k on s; with pdl as a programmatic dependent launch (its blocks
// may be scheduled while the predecessor on s drains; the far-field kernels
// wait for it in chain_wait before touching its data).
template <typename... P, typename... A>
void launch_k(bool pdl, void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A... args) {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, k, static_cast<P>(args)...);
}

// xt[t] = x[perm[t]] (conjugated when cj)
__global__ void k_gather(const double2* __restrict__ x, const int* __restrict__ perm,
                         double2* __restrict__ xt, int n, int cj) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double2 v = x[perm[t]];
    if (cj) v.y = -v.y;
    xt[t] = v;
}

__global__ void k_conj_copy(const double2* __restrict__ x, double2* __restrict__ out, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = make_double2(x[t].x, -x[t].y);
}

// v = ck (yfar[t] + ynear[t]) + loads[t] xt[t] (loads: a diagonal added to the
// operator, may be null), conjugated when cj (the adjoint, xt then holding
// conj(x)); y[perm[t]] (+)= v, perm == nullptr keeps tree order.
__global__ void k_finish(const double2* __restrict__ yfar, const double2* __restrict__ ynear,
                         const int* __restrict__ perm, double2* __restrict__ y, int n, double2 ck,
                         int accumulate, const double2* __restrict__ xt, const double2* __restrict__ loads, int cj) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double2 v = cmul(ck, cadd(yfar[t], ynear[t]));
    if (loads) v = cfma(loads[t], xt[t], v);
    if (cj) v.y = -v.y;
    const int o = perm ? perm[t] : t;
    y[o] = accumulate ? cadd(y[o], v) : v;
}

// The boundary kernels of a product on mapped host buffers, indexed by the
// caller's order so that every warp reads x and writes y in one contiguous
// run across the bus: xt[tpos[c]] = x[c]; y[c] (+)= ck (yfar + ynear)[tpos[c]]
// + loads xt (the same value k_finish forms).
__global__ void k_gather_caller(const double2* __restrict__ x, const int* __restrict__ tpos,
                                double2* __restrict__ xt, int n) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n) xt[tpos[c]] = x[c];
}
__global__ void k_finish_caller(const double2* __restrict__ yfar, const double2* __restrict__ ynear,
                                const int* __restrict__ tpos, double2* __restrict__ y, int n, double2 ck,
                                int accumulate, const double2* __restrict__ xt, const double2* __restrict__ loads) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int t = tpos[c];
    double2 v = cmul(ck, cadd(yfar[t], ynear[t]));
    if (loads) v = cfma(loads[t], xt[t], v);
    y[c] = accumulate ? cadd(y[c], v) : v;
}

inline int blocks_for(long long n, int bs) { return static_cast<int>((n + bs - 1) / bs); }

template <class C> C host_c(const cplx& v);
template <> double2 host_c<double2>(const cplx& v) { return make_double2(v.real(), v.imag()); }
template <> float2 host_c<float2>(const cplx& v) {
    return make_float2(static_cast<float>(v.real()), static_cast<float>(v.imag()));
}
template <class C> std::vector<C> conv_c(const std::vector<cplx>& v) {
    std::vector<C> o(v.size());
    for (size_t i = 0; i < v.size(); ++i) o[i] = host_c<C>(v[i]);
    return o;
}
template <class R> std::vector<R> conv_r(const std::vector<double>& v) {
    return std::vector<R>(v.begin(), v.end());
}

// Tap counts for which the interpolation kernels are instantiated.
constexpr int kUpWidths[] = {2, 4, 6, 8, 10};
constexpr int kDnWidths[] = {8, 12, 16, 24, 32};

}  // namespace

// ================================================================= DeviceOp

DeviceOp::~DeviceOp() {
    if (device_ >= 0) cudaSetDevice(device_);
    for (int p = 0; p < 2; ++p)
        for (int t = 0; t < 2; ++t) {
            if (graph_exec_[p][t]) cudaGraphExecDestroy(graph_exec_[p][t]);
            if (graph_[p][t]) cudaGraphDestroy(graph_[p][t]);
        }
    for (void* p : allocs_) cudaFree(p);
    if (ev_fork_) cudaEventDestroy(ev_fork_);
    if (ev_join_) cudaEventDestroy(ev_join_);
    if (ev_m2l_done_) cudaEventDestroy(ev_m2l_done_);
    if (ev_m2l_done2_) cudaEventDestroy(ev_m2l_done2_);
    if (side3_) cudaStreamDestroy(side3_);
    for (auto& e : ev_level_)
        if (e) cudaEventDestroy(e);
    if (side2_) cudaStreamDestroy(side2_);
    if (stream_) cudaStreamDestroy(stream_);
    if (side_) cudaStreamDestroy(side_);
    if (err_host_) cudaFreeHost(err_host_);
}

// Persistent blocks of k_near_sym: per_sm per SM, but at least four tiles per
// block, so that a small operator leaves room for the kernels of others
// running beside it.
void DeviceOp::set_near_grid(int per_sm) {
    if (near_kernel_ == 1) per_sm = 1;  // k_near_warp: one block per SM (its ring fills the shared memory)
    if (near_kernel_ == 2) {            // k_near_direct: every resident warp of the grid takes tiles
        near_grid_ = std::max(1, std::min((n_near_tiles_ + kNdThreads / 32 - 1) / (kNdThreads / 32),
                                          std::max(1, per_sm) * sms_));
        return;
    }
    near_grid_ = std::max(1, std::min(n_near_tiles_ / 4, std::max(1, per_sm) * sms_));
}

void launch_wait_runs_out(long long limit, int* status) { k_wait_runs_out<<<1, 32>>>(limit, status); }

std::string DeviceOp::device_error() const {
    const int e = err_host_ ? *static_cast<volatile int*>(err_host_) : 0;
    if (e == 1) return "near-field kernel: a bulk copy did not complete within its bounded wait";
    if (e == 2) return "tensor-core interpolation kernel: a copy or an MMA did not complete within its bounded wait";
    return {};
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

// Host-to-device copy that has landed when it returns.  cudaMemcpy from
// pageable memory may return once the data is staged, before the DMA (on the
// legacy default stream) reaches device memory, and kernels on this operator's
// non-blocking streams are not ordered after it.
static cudaError_t h2d_landed(void* dst, const void* src, size_t bytes) {
    cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
    return e;
}

template <class T>
T* DeviceOp::upload(const std::vector<T>& v) {
    T* p = alloc<T>(v.size());
    if (!v.empty() && h2d_landed(p, v.data(), v.size() * sizeof(T)) != cudaSuccess)
        throw std::runtime_error("cudaMemcpy failed");
    return p;
}

int DeviceOp::m2m_rows(int nth, int nph) {
    // about one parent output per thread of a 128-thread block
    return std::max(1, std::min(nth, 128 / std::max(nph, 1)));
}

// One-vector M2L work items (level, box, first direction, count) for a
// direction chunk of at most max_chunk, written to the device array; items of
// each level are contiguous (m2l_first_, m2l_count_).
size_t DeviceOp::m2l_item_capacity(int min_chunk) const {
    size_t n = 1;
    for (int l = lmin_; l <= lmax_; ++l) n += static_cast<size_t>(nbox_[l]) * ((ndir_[l] + min_chunk - 1) / min_chunk + 1);
    return n;
}

void DeviceOp::build_m2l_items(int max_chunk) {
    std::vector<int4> items;
    for (int l = lmin_; l <= lmax_; ++l) {
        const int nchunk = (ndir_[l] + max_chunk - 1) / max_chunk;
        const int chunk = (ndir_[l] + nchunk - 1) / nchunk;
        m2l_first_[l] = static_cast<int>(items.size());
        // boxes with the longest lists first (the last wave short); each box's
        // direction chunks write their own outputs, so the order changes no result
        std::vector<int> order(nbox_[l]);
        for (int b = 0; b < nbox_[l]; ++b) order[b] = b;
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return m2l_len_[l][a] > m2l_len_[l][b]; });
        for (int b : order) {
            if (ref_compat_ && !m2l_has_list_[l][b]) continue;
            for (int d0 = 0; d0 < ndir_[l]; d0 += chunk) items.push_back(make_int4(l, b, d0, std::min(chunk, ndir_[l] - d0)));
        }
        m2l_count_[l] = static_cast<int>(items.size()) - m2l_first_[l];
    }
    n_m2l_items_ = static_cast<int>(items.size());
    m2l_chunk_ = max_chunk;
    if (!items.empty()) h2d_landed(m2l_items_, items.data(), sizeof(int4) * items.size());
}

// The 316 x ndir transfer functions of level L on the GPU (k_tables_alpha,
// k_tables_transl), complex double, into t.
std::string DeviceOp::build_transl_device(const Level& L, double2* t) {
    // offsets in the order of Math::getINodeDistVecs (src/math.cpp:106-122);
    // the distinct squared lengths index the alpha rows
    std::vector<int> r2list, rix;
    std::vector<double> uhat;
    for (int dz = -3; dz <= 3; ++dz)
        for (int dy = -3; dy <= 3; ++dy)
            for (int dx = -3; dx <= 3; ++dx) {
                if (std::max({std::abs(dx), std::abs(dy), std::abs(dz)}) <= 1) continue;
                const int r2 = dx * dx + dy * dy + dz * dz;
                auto it = std::find(r2list.begin(), r2list.end(), r2);
                if (it == r2list.end()) {
                    r2list.push_back(r2);
                    it = r2list.end() - 1;
                }
                rix.push_back(static_cast<int>(it - r2list.begin()));
                const double r = std::sqrt(static_cast<double>(r2));
                uhat.push_back(dx / r);
                uhat.push_back(dy / r);
                uhat.push_back(dz / r);
            }
    const int order = plan_order_;
    if (2 * order > 2 * kTabMaxOrder || L.nps < 2 * order || L.nps < 2) return "interp_order out of range for the tables";
    const int nr = static_cast<int>(r2list.size());
    int* d_r2 = upload(r2list);
    int* d_rix = upload(rix);
    double* d_u = upload(uhat);
    double* d_kh = upload(L.khat);
    double2* d_alpha = alloc<double2>(static_cast<size_t>(nr) * L.nps);
    k_tables_alpha<<<blocks_for(static_cast<long long>(nr) * L.nps, kTabThreads), kTabThreads, 0, stream_>>>(
        d_r2, nr, L.nps, L.L, wavenum_, L.leng, d_alpha);
    k_tables_transl<<<blocks_for(316ll * L.ndir, kTabThreads), kTabThreads, 0, stream_>>>(d_u, d_rix, d_alpha, L.nps,
                                                                                         order, d_kh, L.ndir, t);
    MLFMA_CK(cudaGetLastError());
    return {};
}

// Far-field arrays in precision R (levels, transitions, patterns).
template <class R>
std::string DeviceOp::setup_far(const Plan& plan, FarField<R>& F, const double2* pat64) {
    using C = typename Cx<R>::T;
    for (int l = lmin_; l <= lmax_; ++l) {
        const Level& L = plan.levels[l];
        DevLevelT<R>& d = F.lv[l];
        d.nth = L.nth;
        d.nph = L.nph;
        d.ndir = L.ndir;
        d.nbox = static_cast<int>(L.boxes.size());
        const size_t cnt = static_cast<size_t>(d.nbox) * L.ndir * 2;
        d.A = alloc<C>(cnt);
        d.B = alloc<C>(cnt);
        MLFMA_CK(cudaMemset(d.A, 0, cnt * sizeof(C)));
        MLFMA_CK(cudaMemset(d.B, 0, cnt * sizeof(C)));
        d.Am = d.Bm = nullptr;
        if (max_rhs_ > 1) {
            d.Am = alloc<C>(cnt * max_rhs_);
            d.Bm = alloc<C>(cnt * max_rhs_);
            MLFMA_CK(cudaMemset(d.Am, 0, cnt * max_rhs_ * sizeof(C)));
            MLFMA_CK(cudaMemset(d.Bm, 0, cnt * max_rhs_ * sizeof(C)));
        }
        if constexpr (std::is_same<R, double>::value) {
            // transfer functions built on the GPU (kernels_tables.cuh)
            double2* t = alloc<double2>(static_cast<size_t>(316) * L.ndir);
            std::string e = build_transl_device(L, t);
            if (!e.empty()) return e;
            d.transl = t;
        } else {
            // the complex-float far field narrows the FP64 table
            C* t = alloc<C>(static_cast<size_t>(316) * L.ndir);
            const long long cnt = 316ll * L.ndir;
            k_narrow<C><<<blocks_for(cnt, 256), 256, 0, stream_>>>(f64_.lv[l].transl, t, cnt);
            MLFMA_CK(cudaGetLastError());
            d.transl = t;
        }
        d.w = upload(conv_r<R>(L.m2l_w));
        d.shift_up = upload(conv_c<C>(L.shift_up));
        d.shift_down = upload(conv_c<C>(L.shift_down));
        d.m2l_ptr = upload(L.m2l_ptr);
        d.m2l_src = upload(L.m2l_src);
        d.m2l_off = upload(L.m2l_off);
        // antipode of direction (ith, iph): (nth - 1 - ith, iph + nph / 2); the
        // first half of the directions (d < ndir / 2) meets every pair once
        std::vector<int> anti(L.ndir);
        for (int e = 0; e < L.ndir; ++e) {
            const int dd = e >> 1, ith = dd / L.nph, iph = dd % L.nph;
            anti[e] = (((L.nth - 1 - ith) * L.nph + (iph + L.nph / 2) % L.nph) << 1) | (e & 1);
        }
        d.anti = upload(anti);
    }
    F.lv_dev = upload(std::vector<DevLevelT<R>>(F.lv, F.lv + kMaxLevels));
    F.trans.assign(std::max(lmax_, 0) + 1, DevTransT<R>{});
    for (int p = lmin_; p < lmax_; ++p) {
        const Transition& T = plan.trans[p];
        DevTransT<R>& d = F.trans[p];
        auto st = [&](const Stencil& s, int w) {
            // pad rows to a fixed width; fold the reflection sign into the coefficient
            const int rows = static_cast<int>(s.ptr.size()) - 1;
            std::vector<int> src(static_cast<size_t>(rows) * w, 0), refl(static_cast<size_t>(rows) * w, 0);
            std::vector<R> coef(static_cast<size_t>(rows) * w, R(0));
            for (int r = 0; r < rows; ++r)
                for (int q = s.ptr[r]; q < s.ptr[r + 1]; ++q) {
                    const size_t at = static_cast<size_t>(r) * w + (q - s.ptr[r]);
                    src[at] = s.src[q];
                    refl[at] = s.refl[q];
                    coef[at] = static_cast<R>(s.refl[q] ? -s.coef[q] : s.coef[q]);
                }
            std::vector<int> src_t(src.size());
            std::vector<R> coef_t(coef.size());
            for (int r = 0; r < rows; ++r)
                for (int k = 0; k < w; ++k) {
                    src_t[static_cast<size_t>(k) * rows + r] = src[static_cast<size_t>(r) * w + k];
                    coef_t[static_cast<size_t>(k) * rows + r] = coef[static_cast<size_t>(r) * w + k];
                }
            return DevStencilT<R>{w, upload(src), upload(refl), upload(coef), rows, upload(src_t), upload(coef_t)};
        };
        d.up_th = st(T.up_th, up_w_[p]);
        d.up_ph = st(T.up_ph, up_w_[p]);
        d.dn_ph = st(T.dn_ph, dn_w_[p]);
        d.dn_th = st(T.dn_th, dn_w_[p]);
        d.plevel = p;
        d.npar = static_cast<int>(T.par_box.size());
        d.fold_up = d.fold_dn = nullptr;
        if (max_rhs_ > 1) {
            const Level& PL = plan.levels[p];
            const Level& CL = plan.levels[p + 1];
            const int wu = up_w_[p], wd = dn_w_[p];
            const int mph = CL.nph, halfm = CL.nph / 2;
            std::vector<cplx> fu(static_cast<size_t>(8) * PL.nth * mph * wu, cplx(0));
            for (int oct = 0; oct < 8; ++oct)
                for (int jth = 0; jth < PL.nth; ++jth)
                    for (int q = T.up_th.ptr[jth]; q < T.up_th.ptr[jth + 1]; ++q) {
                        const int k = q - T.up_th.ptr[jth];
                        const double cf = T.up_th.refl[q] ? -T.up_th.coef[q] : T.up_th.coef[q];
                        for (int iph = 0; iph < mph; ++iph) {
                            const int sp = T.up_th.refl[q] ? (iph < halfm ? iph + halfm : iph - halfm) : iph;
                            const int dd = T.up_th.src[q] * mph + sp;
                            fu[((static_cast<size_t>(oct) * PL.nth + jth) * mph + iph) * wu + k] =
                                cf * CL.shift_up[static_cast<size_t>(oct) * CL.ndir + dd];
                        }
                    }
            std::vector<cplx> fd(static_cast<size_t>(8) * PL.nth * CL.nph * wd, cplx(0));
            for (int oct = 0; oct < 8; ++oct)
                for (int ith = 0; ith < PL.nth; ++ith)
                    for (int jph = 0; jph < CL.nph; ++jph)
                        for (int q = T.dn_ph.ptr[jph]; q < T.dn_ph.ptr[jph + 1]; ++q) {
                            const int k = q - T.dn_ph.ptr[jph];
                            const double cf = T.dn_ph.refl[q] ? -T.dn_ph.coef[q] : T.dn_ph.coef[q];
                            const int dd = ith * PL.nph + T.dn_ph.src[q];
                            fd[((static_cast<size_t>(oct) * PL.nth + ith) * CL.nph + jph) * wd + k] =
                                cf * PL.shift_down[static_cast<size_t>(oct) * PL.ndir + dd];
                        }
            d.fold_up = upload(conv_c<C>(fu));
            d.fold_dn = upload(conv_c<C>(fd));
        }
        d.par_box = upload(T.par_box);
        d.par_ilist = upload(T.par_ilist);
        d.child_ptr = upload(T.child_ptr);
        d.child_box = upload(T.child_box);
        d.child_oct = upload(T.child_oct);
    }
    if (std::is_same<R, double>::value) {
        F.pat = reinterpret_cast<C*>(const_cast<double2*>(pat64));
    } else if (max_rhs_ > 1) {
        const long long cnt = plan.pat_elems * 2;
        F.pat = alloc<C>(static_cast<size_t>(cnt));
        if (cnt) k_narrow<C><<<blocks_for(cnt, 256), 256, 0, stream_>>>(pat64, F.pat, cnt);
        MLFMA_CK(cudaGetLastError());
    }
    if constexpr (!std::is_same<R, double>::value) {  // half patterns for the complex-float far field
        F.hpat = alloc<C>(static_cast<size_t>(plan.pat_elems));
        if (n_leaves_) k_half_patterns<R><<<n_leaves_, 256, 0, stream_>>>(F.lv_dev, leaves_, pat64, F.hpat);
        MLFMA_CK(cudaGetLastError());
    }
    // Shared-memory limits.
    size_t m2m_smem = 1, l2l_smem = 1;
    for (int p = lmin_; p < lmax_; ++p) {
        m2m_smem = std::max(m2m_smem, static_cast<size_t>(8) * m2m_rows(nth_[p], nph_[p]) * nph_[p + 1] * 2 * sizeof(C));
        l2l_smem = std::max(l2l_smem, static_cast<size_t>(nth_[p]) * nph_[p + 1] * 2 * sizeof(C));
    }
    int dev_smem = 0;
    MLFMA_CK(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device_));
    const size_t s2m_smem = static_cast<size_t>(std::max(1, max_src_)) * sizeof(C);
    // k_l2t_half (complex-float far field) stages a leaf's local pattern twice
    const size_t l2t_smem = 2 * sizeof(C) * static_cast<size_t>(max_leaf_ndir_);
    if (m2m_smem > static_cast<size_t>(dev_smem) || l2l_smem > static_cast<size_t>(dev_smem) ||
        s2m_smem > static_cast<size_t>(dev_smem) ||
        (!std::is_same<R, double>::value && l2t_smem > static_cast<size_t>(dev_smem)))
        return "angular grid or leaf too large for the kernels' shared memory";
    // The limit is a property of the kernel, shared by every operator in the
    // process: set it to the device's opt-in maximum (this operator's needs
    // were checked above), never to this operator's own size, or an operator
    // set up later with smaller leaves or grids would make an earlier one's
    // launches fail.
    const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
    for (int tr = 0; tr < 2; ++tr) {  // forward and transposed variants
        const bool t = tr != 0;
        MLFMA_CK(cudaFuncSetAttribute(t ? k_m2m<R, 2, true> : k_m2m<R, 2, false>, attr, dev_smem));
        MLFMA_CK(cudaFuncSetAttribute(t ? k_m2m<R, 4, true> : k_m2m<R, 4, false>, attr, dev_smem));
        MLFMA_CK(cudaFuncSetAttribute(t ? k_m2m<R, 6, true> : k_m2m<R, 6, false>, attr, dev_smem));
        MLFMA_CK(cudaFuncSetAttribute(t ? k_m2m<R, 8, true> : k_m2m<R, 8, false>, attr, dev_smem));
        MLFMA_CK(cudaFuncSetAttribute(t ? k_m2m<R, 10, true> : k_m2m<R, 10, false>, attr, dev_smem));
        MLFMA_CK(cudaFuncSetAttribute(t ? k_l2l<R, 8, true> : k_l2l<R, 8, false>, attr, dev_smem));
        MLFMA_CK(cudaFuncSetAttribute(t ? k_l2l<R, 12, true> : k_l2l<R, 12, false>, attr, dev_smem));
        MLFMA_CK(cudaFuncSetAttribute(t ? k_l2l<R, 16, true> : k_l2l<R, 16, false>, attr, dev_smem));
        MLFMA_CK(cudaFuncSetAttribute(t ? k_l2l<R, 24, true> : k_l2l<R, 24, false>, attr, dev_smem));
        MLFMA_CK(cudaFuncSetAttribute(t ? k_l2l<R, 32, true> : k_l2l<R, 32, false>, attr, dev_smem));
        MLFMA_CK(cudaFuncSetAttribute(t ? k_s2m<R, true> : k_s2m<R, false>, attr, dev_smem));
        if constexpr (!std::is_same<R, double>::value) {
            MLFMA_CK(cudaFuncSetAttribute(t ? k_s2m_half<R, true> : k_s2m_half<R, false>, attr, dev_smem));
            MLFMA_CK(cudaFuncSetAttribute(t ? k_l2t_half<R, true> : k_l2t_half<R, false>, attr, dev_smem));
        }
    }
    {  // staged interpolation: dynamic shared memory up to the limit less the static part
        auto dyn = [&](const void* fn) -> cudaError_t {
            cudaFuncAttributes fa{};
            cudaError_t e = cudaFuncGetAttributes(&fa, fn);
            if (e != cudaSuccess) return e;
            return cudaFuncSetAttribute(fn, attr, dev_smem - static_cast<int>(fa.sharedSizeBytes));
        };
        for (int cs = 0; cs < 2; ++cs) {
            const bool c = cs != 0;
            MLFMA_CK(dyn(reinterpret_cast<const void*>(c ? k_m2m_sum<R, 2, true> : k_m2m_sum<R, 2, false>)));
            MLFMA_CK(dyn(reinterpret_cast<const void*>(c ? k_m2m_sum<R, 4, true> : k_m2m_sum<R, 4, false>)));
            MLFMA_CK(dyn(reinterpret_cast<const void*>(c ? k_m2m_sum<R, 6, true> : k_m2m_sum<R, 6, false>)));
            MLFMA_CK(dyn(reinterpret_cast<const void*>(c ? k_m2m_sum<R, 8, true> : k_m2m_sum<R, 8, false>)));
            MLFMA_CK(dyn(reinterpret_cast<const void*>(c ? k_m2m_sum<R, 10, true> : k_m2m_sum<R, 10, false>)));
        }
        for (int v = 0; v < 4; ++v) {  // (transposed, column-stationary)
            const void* fns[] = {
#define MLFMA_L2L_ST_FN(WW)                                                                                  \
    (v == 0 ? reinterpret_cast<const void*>(k_l2l_st<R, WW, false, false>)                                 \
     : v == 1 ? reinterpret_cast<const void*>(k_l2l_st<R, WW, true, false>)                                \
     : v == 2 ? reinterpret_cast<const void*>(k_l2l_st<R, WW, false, true>)                                \
              : reinterpret_cast<const void*>(k_l2l_st<R, WW, true, true>))
                MLFMA_L2L_ST_FN(8), MLFMA_L2L_ST_FN(12), MLFMA_L2L_ST_FN(16), MLFMA_L2L_ST_FN(24),
                MLFMA_L2L_ST_FN(32)};
#undef MLFMA_L2L_ST_FN
            for (const void* fn : fns) MLFMA_CK(dyn(fn));
        }
        for (int tr = 0; tr < 2; ++tr) {
            const bool t = tr != 0;
            MLFMA_CK(dyn(reinterpret_cast<const void*>(t ? k_l2l_pipe<R, 8, true> : k_l2l_pipe<R, 8, false>)));
            MLFMA_CK(dyn(reinterpret_cast<const void*>(t ? k_l2l_pipe<R, 12, true> : k_l2l_pipe<R, 12, false>)));
            MLFMA_CK(dyn(reinterpret_cast<const void*>(t ? k_l2l_pipe<R, 16, true> : k_l2l_pipe<R, 16, false>)));
            MLFMA_CK(dyn(reinterpret_cast<const void*>(t ? k_l2l_pipe<R, 24, true> : k_l2l_pipe<R, 24, false>)));
            MLFMA_CK(dyn(reinterpret_cast<const void*>(t ? k_l2l_pipe<R, 32, true> : k_l2l_pipe<R, 32, false>)));
        }
    }
    if (max_rhs_ > 1) {
        // dynamic shared memory up to the opt-in limit less the kernel's static part
        auto dyn = [&](const void* fn) -> cudaError_t {
            cudaFuncAttributes fa{};
            cudaError_t e = cudaFuncGetAttributes(&fa, fn);
            if (e != cudaSuccess) return e;
            return cudaFuncSetAttribute(fn, attr, dev_smem - static_cast<int>(fa.sharedSizeBytes));
        };
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_m2m_m<R, 2, 8>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_m2m_m<R, 4, 8>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_m2m_m<R, 6, 8>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_m2m_m<R, 8, 8>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_m2m_m<R, 10, 8>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_m2m_m<R, 2, kM2MOut>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_m2m_m<R, 4, kM2MOut>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_m2m_m<R, 6, kM2MOut>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_m2m_m<R, 8, kM2MOut>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_m2m_m<R, 10, kM2MOut>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_l2l_m<R, 8, 1>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_l2l_m<R, 12, 1>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_l2l_m<R, 16, 1>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_l2l_m<R, 24, 1>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_l2l_m<R, 32, 1>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_l2l_m<R, 8, 2>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_l2l_m<R, 12, 2>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_l2l_m<R, 16, 2>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_l2l_m<R, 24, 2>)));
        MLFMA_CK(dyn(reinterpret_cast<const void*>(k_l2l_m<R, 32, 2>)));
        for (int p = lmin_; p < lmax_; ++p) {
            const size_t m2m1 = static_cast<size_t>(nph_[p + 1]) * 32 * m2m_rpl<R>() * sizeof(C);
            const size_t l2l1 = static_cast<size_t>(nth_[p]) * 2 * 1 * 64 * sizeof(C) +
                                static_cast<size_t>(nth_[p + 1]) * dn_w_[p] * (sizeof(R) + 2 * sizeof(int));
            // (the static stencil staging takes at most 11 KB)
            if (m2m1 + 11264 > static_cast<size_t>(dev_smem) || l2l1 + 1024 > static_cast<size_t>(dev_smem) ||
                nph_[p] > kM2MOut * kInterpWarps)
                return "angular grid too large for the many-right-hand-side interpolation kernels";
        }
    }
    return {};
}



std::string DeviceOp::setup(const Plan& plan, int device, int precision, int max_rhs) {
    try {
        device_ = device;
        precision_ = precision;
        if (precision != kFp64 && precision != kMixed) return "precision must be 0 (FP64) or 1 (mixed)";
        if (max_rhs < 1 || max_rhs > kMaxRhs) return "max_rhs must be 1..64";
        max_rhs_ = max_rhs;
        MLFMA_CK(cudaSetDevice(device));
        // The far-field chain (the product's critical path) gets the highest
        // priority; the near field and the finer levels' translations, which
        // run beside it, the lowest: pending chain blocks are scheduled first.
        int prio_low = 0, prio_high = 0;
        MLFMA_CK(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
        MLFMA_CK(cudaStreamCreateWithPriority(&stream_, cudaStreamNonBlocking, prio_high));
        MLFMA_CK(cudaStreamCreateWithPriority(&side_, cudaStreamNonBlocking, prio_low));
        MLFMA_CK(cudaStreamCreateWithPriority(&side2_, cudaStreamNonBlocking, prio_low));
        MLFMA_CK(cudaStreamCreateWithPriority(&side3_, cudaStreamNonBlocking, prio_low));
        // error word of the kernels with bounded waits, read by the host after a sync
        MLFMA_CK(cudaHostAlloc(reinterpret_cast<void**>(&err_host_), sizeof(int), cudaHostAllocMapped));
        *err_host_ = 0;
        MLFMA_CK(cudaHostGetDevicePointer(reinterpret_cast<void**>(&err_dev_), err_host_, 0));
        MLFMA_CK(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
        MLFMA_CK(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming));
        MLFMA_CK(cudaEventCreateWithFlags(&ev_m2l_done_, cudaEventDisableTiming));
        MLFMA_CK(cudaEventCreateWithFlags(&ev_m2l_done2_, cudaEventDisableTiming));
        for (auto& e : ev_level_) MLFMA_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        n_ = plan.n;
        if (plan.max_level >= kMaxLevels) return "tree deeper than supported";
        const cplx ck = cplx(0, -kC0 * kMu0 / (4.0 * kPi)) * plan.pw.wavenum;
        ck_ = make_double2(ck.real(), ck.imag());
        perm_ = upload(plan.perm);
        {
            std::vector<int> tpos(plan.perm.size());
            for (size_t t = 0; t < plan.perm.size(); ++t) tpos[plan.perm[t]] = static_cast<int>(t);
            tpos_ = upload(tpos);
        }
        xt_ = alloc<double2>(n_);
        yfar_ = alloc<double2>(n_);
        ynear_ = alloc<double2>(n_);
        yt_ = alloc<double2>(n_);
        lmin_ = plan.lmin;
        lmax_ = plan.max_level;
        plan_order_ = plan.cfg.interp_order;
        wavenum_ = plan.pw.wavenum;
        ref_compat_ = plan.cfg.ref_compat;
        traffic_ = Traffic{};
        const double cbytes = precision == kFp64 ? 16.0 : 8.0;  // one far-field complex value

        // ---- level sizes and M2L work items: direction chunks of at most 128
        for (int l = lmin_; l <= lmax_; ++l) {
            const Level& L = plan.levels[l];
            nbox_[l] = static_cast<int>(L.boxes.size());
            ndir_[l] = L.ndir;
            nth_[l] = L.nth;
            nph_[l] = L.nph;
            const double cnt = static_cast<double>(nbox_[l]) * L.ndir * 2;
            // M2L reads every source box's pattern and the transfer table once
            // (repeats hit L2) and writes every local pattern once.
            traffic_.m2l += cnt * cbytes * 2.0 + 316.0 * L.ndir * cbytes;
            m2l_has_list_[l].resize(nbox_[l]);
            m2l_len_[l].resize(nbox_[l]);
            for (int b = 0; b < nbox_[l]; ++b) {
                m2l_has_list_[l][b] = L.m2l_ptr[b + 1] > L.m2l_ptr[b];
                m2l_len_[l][b] = L.m2l_ptr[b + 1] - L.m2l_ptr[b];
            }
        }
        m2l_items_ = alloc<int4>(m2l_item_capacity(8));
        build_m2l_items(128);

        // ---- transitions: L2L pairs and stencil widths
        l2l_pairs_.assign(std::max(lmax_, 0) + 1, nullptr);
        m2m_rows_.assign(std::max(lmax_, 0) + 1, 1);
        m2m_pref_.assign(std::max(lmax_, 0) + 1, 0);
        l2l_pref_.assign(std::max(lmax_, 0) + 1, 0);
        MLFMA_CK(cudaDeviceGetAttribute(&dev_smem_, cudaDevAttrMaxSharedMemoryPerBlockOptin, device_));
        n_l2l_pairs_.assign(std::max(lmax_, 0) + 1, 0);
        npar_.assign(std::max(lmax_, 0) + 1, 0);
        up_w_.assign(std::max(lmax_, 0) + 1, 0);
        dn_w_.assign(std::max(lmax_, 0) + 1, 0);
        for (int p = lmin_; p < lmax_; ++p) {
            const Transition& T = plan.trans[p];
            auto width_of = [](const Stencil& s) {
                int w = 1;
                for (size_t r = 0; r + 1 < s.ptr.size(); ++r) w = std::max(w, s.ptr[r + 1] - s.ptr[r]);
                return w;
            };
            const int w_up = width_of(T.up_th);
            if (w_up != width_of(T.up_ph) || std::find(std::begin(kUpWidths), std::end(kUpWidths), w_up) ==
                                                 std::end(kUpWidths))
                return "interp_order must be 1..5";
            const int need = std::max(width_of(T.dn_ph), width_of(T.dn_th));
            int w_dn = 0;
            for (int c : kDnWidths)
                if (!w_dn && need <= c) w_dn = c;
            if (!w_dn) return "anterpolation stencil wider than 32 taps";
            up_w_[p] = w_up;
            dn_w_[p] = w_dn;
            m2m_rows_[p] = m2m_rows(nth_[p], nph_[p]);
            m2m_pref_[p] = 1;
            l2l_pref_[p] = 1;
            npar_[p] = static_cast<int>(T.par_box.size());
            std::vector<int2> pairs;
            for (int q = 0; q < npar_[p]; ++q) {
                if (ref_compat_ && !T.par_ilist[q]) continue;  // stem.cpp:115
                for (int c = T.child_ptr[q]; c < T.child_ptr[q + 1]; ++c) pairs.push_back(make_int2(q, c));
            }
            n_l2l_pairs_[p] = static_cast<int>(pairs.size());
            l2l_pairs_[p] = upload(pairs);
            const double nch = static_cast<double>(T.child_box.size());
            traffic_.m2m += (nch * ndir_[p + 1] + npar_[p] * ndir_[p]) * 2.0 * cbytes;
            traffic_.l2l += (npar_[p] * ndir_[p] + nch * ndir_[p + 1] * 2.0) * 2.0 * cbytes;
        }

        // ---- far leaves and work items
        std::vector<DevFarLeaf> h_leaves;
        std::vector<DevFarLeafGeom> geo;
        std::vector<int4> s2m_items, s2m_items_h, l2t_items;
        max_src_ = 0;
        for (const FarLeaf& f : plan.far_leaves) {
            h_leaves.push_back(DevFarLeaf{f.level, f.box, f.src0, f.nsrc, f.pat_off});
            const int li = static_cast<int>(h_leaves.size()) - 1;
            const int ne = 2 * plan.levels[f.level].ndir;
            const int nchunk = (ne + kS2MThreads - 1) / kS2MThreads;
            const int chunk = (ne + nchunk - 1) / nchunk;
            for (int e0 = 0; e0 < ne; e0 += chunk) s2m_items.push_back(make_int4(li, e0, std::min(chunk, ne - e0), 0));
            // half patterns (complex-float far field): elements of the first half of the directions
            const int nh = ne / 2;
            const int nchunk_h = (nh + kS2MThreads - 1) / kS2MThreads;
            const int chunk_h = (nh + nchunk_h - 1) / nchunk_h;
            for (int e0 = 0; e0 < nh; e0 += chunk_h)
                s2m_items_h.push_back(make_int4(li, e0, std::min(chunk_h, nh - e0), 0));
            for (int s0 = 0; s0 < f.nsrc; s0 += kL2TSrcPerBlock)
                l2t_items.push_back(make_int4(li, s0, std::min(kL2TSrcPerBlock, f.nsrc - s0), 0));
            max_src_ = std::max(max_src_, f.nsrc);
            max_leaf_ndir_ = std::max(max_leaf_ndir_, plan.levels[f.level].ndir);
            const Node& nd = plan.nodes[plan.levels[f.level].boxes[f.box]];
            geo.push_back(DevFarLeafGeom{{nd.center[0], nd.center[1], nd.center[2]}});
        }
        n_leaves_ = static_cast<int>(h_leaves.size());
        leaves_ = upload(h_leaves);
        // Largest work items first: a leaf's S2M block streams all its sources'
        // patterns (1 to max_node_srcs of them), so launching the long blocks
        // first keeps the last wave short.  Items write disjoint outputs; the
        // order changes no result.
        auto by_work = [&](std::vector<int4>& items, bool per_source) {
            auto work = [&](const int4& it) {
                const DevFarLeaf& f = h_leaves[it.x];
                const long long nd = plan.levels[f.level].ndir;
                return per_source ? static_cast<long long>(it.z) * nd : static_cast<long long>(f.nsrc) * it.z;
            };
            std::stable_sort(items.begin(), items.end(),
                             [&](const int4& a, const int4& b) { return work(a) > work(b); });
        };
        by_work(s2m_items, false);
        by_work(s2m_items_h, false);
        by_work(l2t_items, true);

        n_s2m_items_ = static_cast<int>(s2m_items.size());
        s2m_items_ = upload(s2m_items);
        n_s2m_items_h_ = static_cast<int>(s2m_items_h.size());
        if (precision != kFp64) s2m_items_h_ = upload(s2m_items_h);
        n_l2t_items_ = static_cast<int>(l2t_items.size());
        l2t_items_ = upload(l2t_items);
        long long far_srcs = 0;
        for (const FarLeaf& f : plan.far_leaves) far_srcs += f.nsrc;
        far_covers_all_ = n_leaves_ > 0 && far_srcs == n_;
        // the complex-float far field keeps half the patterns (antipodes by symmetry)
        const double pat_copies = precision == kFp64 ? 2.0 : 1.0;
        traffic_.s2m = plan.pat_elems * pat_copies * cbytes + n_ * 16.0;
        traffic_.l2t = plan.pat_elems * pat_copies * cbytes + n_ * 16.0;

        // ---- radiation patterns (complex double first)
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
            S.tri_v = upload(plan.tri_v);
            S.tri_p = upload(plan.tri_p);
        }
        S.self_terms = plan.cfg.self_terms;
        src_ = S;
        // Complex double patterns: the FP64 far field reads them; the mixed far
        // field reads a complex float copy.  A mixed operator keeps the FP64
        // far field too, for the FP64 residual of iterative refinement.
        double2* pat64 = alloc<double2>(static_cast<size_t>(plan.pat_elems) * 2);
        if (n_leaves_ > 0 && plan.kind == kRwg && plan.cfg.ref_compat) {
            // Reference-compatible RWG patterns: the closed-form integral is
            // ill-conditioned near alpha, beta, gamma = 0, so it is evaluated on
            // the host with the reference's exact rounding and uploaded.
            std::vector<cplx> hp;
            plan.rwg_patterns_host(hp);
            MLFMA_CK(h2d_landed(pat64, hp.data(), hp.size() * sizeof(cplx)));
        } else if (n_leaves_ > 0) {
            std::vector<DevGeomLevel> gl(kMaxLevels, DevGeomLevel{nullptr, nullptr, 0});
            for (int l = lmin_; l <= lmax_; ++l)
                gl[l] = DevGeomLevel{upload(plan.levels[l].thph), upload(plan.levels[l].khat), plan.levels[l].ndir};
            DevGeomLevel* d_gl = upload(gl);
            DevFarLeafGeom* d_geo = upload(geo);
            k_patterns<<<n_leaves_, 256, 0, stream_>>>(d_gl, leaves_, d_geo, S, pat64);
            MLFMA_CK(cudaGetLastError());
        }

        // ---- far field in the chosen precision
        std::string err = setup_far<double>(plan, f64_, pat64);
        if (!err.empty()) return err;
        if (precision != kFp64) {
            err = setup_far<float>(plan, f32_, pat64);
            if (!err.empty()) return err;
            err = setup_tc(plan);
            if (!err.empty()) return err;
        }

        // ---- near field: the stored blocks (each interaction once), applied
        // as Z and Z^T tile by tile (one right-hand side)
        {
            std::vector<DevNearBlock> nb;
            for (const NearBlock& b : plan.near_blocks)
                nb.push_back(DevNearBlock{b.row0, b.nrow, b.col0, b.ncol, b.off,
                                          b.self ? (plan.cfg.self_terms ? 2 : 1) : 0, 0});
            std::vector<DevNearTile> nt;
            for (const NearTile& t : plan.near_tiles)
                nt.push_back(DevNearTile{t.z, t.r0, t.c0, t.i0, t.ni, t.j0, t.nj, t.ld, t.kind, t.slot, t.mode});
            near_block_entries_ = plan.near_entries;
            n_near_tiles_ = static_cast<int>(nt.size());
            if (n_near_tiles_ > 0) {
                near_tiles_ = upload(nt);
                near_bz_ = alloc<double2>(static_cast<size_t>(near_block_entries_));
                near_part_ = alloc<double2>(static_cast<size_t>(plan.near_parts));
                near_red_ptr_ = upload(plan.near_red_ptr);
                near_slot_ = upload(plan.near_slot);
                MLFMA_CK(cudaFuncSetAttribute(k_near_sym, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              static_cast<int>(kSymSmemBytes)));
                MLFMA_CK(cudaFuncSetAttribute(k_near_warp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              static_cast<int>(kNwSmemBytes)));
                MLFMA_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&near_occ_, k_near_sym, kSymThreads,
                                                                       kSymSmemBytes));
                near_occ_ = std::max(1, near_occ_);
                MLFMA_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&near_direct_occ_, k_near_direct, kNdThreads, 0));
                near_direct_occ_ = std::max(1, near_direct_occ_);
                near_per_sm_ = near_occ_;
                MLFMA_CK(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_));
                set_near_grid(near_per_sm_);
                DevNearBlock* d_nb = upload(nb);
                k_near_blocks_assemble<<<blocks_for(near_block_entries_, 128), 128, 0, stream_>>>(
                    d_nb, static_cast<int>(nb.size()), near_block_entries_, S, near_bz_);
                MLFMA_CK(cudaGetLastError());
            }
        }
        // leaves of the block-Jacobi preconditioner (built on first use)
        {
            std::vector<long long> self_off(n_ + 1, -1);
            std::vector<int> self_kind(n_ + 1, 0);
            for (const NearBlock& b : plan.near_blocks)
                if (b.self) {
                    self_off[b.row0] = b.off;
                    self_kind[b.row0] = plan.cfg.self_terms ? 2 : 1;
                }
            h_bj_.clear();
            long long ioff = 0;
            for (int id : plan.leaves) {
                const Node& nd = plan.nodes[id];
                if (nd.src_count <= 0) continue;
                DevBjLeaf L{nd.src_begin, nd.src_count, self_kind[nd.src_begin], 0, self_off[nd.src_begin], ioff};
                if (L.nb <= kBjMax) ioff += static_cast<long long>(L.nb) * L.nb;
                h_bj_.push_back(L);
            }
        }
        // many right-hand sides: block rows (both orientations), gather-only GEMM tiles
        if (max_rhs > 1) {
            std::vector<DevNearRow> nr;
            for (const NearRow& r : plan.near_rows) nr.push_back(DevNearRow{r.row0, r.nrow, r.ncol, 0, r.off, r.col_off});
            n_near_rows_ = static_cast<int>(nr.size());
            near_rows_ = upload(nr);
            near_cols_ = upload(plan.near_cols);
            near_entries_ = plan.near_row_entries;
            near_z_ = alloc<double2>(static_cast<size_t>(near_entries_));
            if (near_entries_ > 0) {
                k_near_rows_assemble<<<blocks_for(near_entries_, 128), 128, 0, stream_>>>(
                    near_rows_, n_near_rows_, near_entries_, near_cols_, S, near_z_);
                MLFMA_CK(cudaGetLastError());
            }
        }
        traffic_.near = near_block_entries_ * 16.0 + n_ * 16.0 * 2.0;
        traffic_.total = traffic_.s2m + traffic_.m2m + traffic_.m2l + traffic_.l2l + traffic_.l2t + traffic_.near;
        if (max_rhs_ > 1) {
            err = build_m2l_groups(plan);
            if (!err.empty()) return err;
            err = setup_multi(plan);
            if (!err.empty()) return err;
        }
        MLFMA_CK(cudaStreamSynchronize(stream_));
        MLFMA_CK(cudaStreamSynchronize(cudaStreamLegacy));  // the memsets above run there
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
        for (int p = lmin_; p < lmax_; ++p) {
            if (npar_[p]) n += 1;           // M2M
            if (n_l2l_pairs_[p]) n += 1;    // L2L
        }
        for (int l = lmin_; l <= lmax_; ++l)
            if (m2l_count_[l]) n += 1;  // one M2L launch per level
    }
    if (n_near_tiles_) n += 2;  // tiles + per-target sums
    return n;
}

// stage: -1 all, 0 S2M, 1 M2M, 2 M2L, 3 L2L, 4 L2T.
// TR: the transposed far field, Far^T = S2M^T L2L^T M2L^T M2M^T L2T^T, run in
// the same order with the mirrored kernels: conjugated patterns going up,
// interpolation with the shift after it (L2L^T), negated translation offsets,
// anterpolation with the shift after it (M2M^T), plain patterns coming down.
template <class R, bool TR>
void DeviceOp::far_s2m(FarField<R>& F, const double2* xt, cudaStream_t s) {
    using C = typename Cx<R>::T;
    if constexpr (std::is_same<R, double>::value) {
        if (n_s2m_items_)
            k_s2m<R, TR><<<n_s2m_items_, kS2MThreads, sizeof(C) * std::max(1, max_src_), s>>>(F.lv_dev, s2m_items_,
                                                                                                leaves_, F.pat, xt);
    } else if (n_s2m_items_h_) {
        k_s2m_half<R, TR><<<n_s2m_items_h_, kS2MThreads, sizeof(C) * std::max(1, max_src_), s>>>(
            F.lv_dev, s2m_items_h_, leaves_, F.hpat, xt);
    }
}

template <class R, bool TR>
void DeviceOp::far_m2m(FarField<R>& F, int p, cudaStream_t s, bool pdl) {
    using C = typename Cx<R>::T;
    if (npar_[p] == 0) return;
    const int rows = m2m_rows_[p];
    const dim3 grid(npar_[p], (nth_[p] + rows - 1) / rows);
    const DevTransT<R>& T = F.trans[p];
    const size_t ssum = m2m_sum_smem(nth_[p + 1], nph_[p + 1], rows, sizeof(C));
    if (!TR && m2m_pref_[p] && ssum + 1024 <= static_cast<size_t>(dev_smem_)) {
        const bool cs = m2m_pref_[p] == 2;
#define MLFMA_M2M_SUM(WW) \
    launch_k(pdl, cs ? k_m2m_sum<R, WW, true> : k_m2m_sum<R, WW, false>, grid, 256, ssum, s, F.lv_dev, T, rows)
        switch (up_w_[p]) {
            case 2: MLFMA_M2M_SUM(2); break;
            case 4: MLFMA_M2M_SUM(4); break;
            case 6: MLFMA_M2M_SUM(6); break;
            case 8: MLFMA_M2M_SUM(8); break;
            default: MLFMA_M2M_SUM(10); break;
        }
#undef MLFMA_M2M_SUM
        return;
    }
    const size_t smem = static_cast<size_t>(8) * rows * nph_[p + 1] * 2 * sizeof(C);
    switch (up_w_[p]) {
        case 2: launch_k(pdl, k_m2m<R, 2, TR>, grid, 128, smem, s, F.lv_dev, T, rows); break;
        case 4: launch_k(pdl, k_m2m<R, 4, TR>, grid, 128, smem, s, F.lv_dev, T, rows); break;
        case 6: launch_k(pdl, k_m2m<R, 6, TR>, grid, 128, smem, s, F.lv_dev, T, rows); break;
        case 8: launch_k(pdl, k_m2m<R, 8, TR>, grid, 128, smem, s, F.lv_dev, T, rows); break;
        default: launch_k(pdl, k_m2m<R, 10, TR>, grid, 128, smem, s, F.lv_dev, T, rows); break;
    }
}

// M2L of levels lo..hi (their items are contiguous, level by level).
template <class R, bool TR>
void DeviceOp::far_m2l(FarField<R>& F, int lo, int hi, cudaStream_t s, bool pdl) {
    if (lo > hi) return;
    const int first = m2l_first_[lo];
    const int count = m2l_first_[hi] + m2l_count_[hi] - first;
    if (count <= 0) return;
    launch_k(pdl, m2l_staged_ ? k_m2l_staged<R, TR> : k_m2l<R, TR>, count, 128, 0, s, F.lv_dev, m2l_items_ + first,
             ref_compat_ ? 0 : 1);
}

template <class R, bool TR>
void DeviceOp::far_l2l(FarField<R>& F, int p, cudaStream_t s, bool pdl) {
    using C = typename Cx<R>::T;
    const int g = n_l2l_pairs_[p];
    if (!g) return;
    const DevTransT<R>& T = F.trans[p];
    const size_t sst = l2l_st_smem(nth_[p], nph_[p], nph_[p + 1], sizeof(C));
    const size_t spipe = l2l_pipe_smem(nth_[p], nph_[p], nth_[p + 1], nph_[p + 1], sizeof(C));
    if (l2l_pref_[p] == 3 && spipe + 1024 <= static_cast<size_t>(dev_smem_)) {
        // persistent: as many blocks as fit on the SMs at once
#define MLFMA_L2L_PIPE(WW)                                                                                 \
    do {                                                                                                   \
        const void* fn = reinterpret_cast<const void*>(k_l2l_pipe<R, WW, TR>);                             \
        int occ = 0;                                                                                       \
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 256, spipe) != cudaSuccess || occ < 1) \
            occ = 1;                                                                                       \
        const int grid = std::max(1, std::min(g, occ * sms_));                                             \
        launch_k(pdl, k_l2l_pipe<R, WW, TR>, grid, 256, spipe, s, F.lv_dev, T, l2l_pairs_[p], g);          \
    } while (0)
        switch (dn_w_[p]) {
            case 8: MLFMA_L2L_PIPE(8); break;
            case 12: MLFMA_L2L_PIPE(12); break;
            case 16: MLFMA_L2L_PIPE(16); break;
            case 24: MLFMA_L2L_PIPE(24); break;
            default: MLFMA_L2L_PIPE(32); break;
        }
#undef MLFMA_L2L_PIPE
        return;
    }
    if (l2l_pref_[p] && l2l_pref_[p] != 3 && sst + 1024 <= static_cast<size_t>(dev_smem_)) {
        const bool cs = l2l_pref_[p] == 2;
#define MLFMA_L2L_ST(WW)                                                                             \
    launch_k(pdl, cs ? k_l2l_st<R, WW, TR, true> : k_l2l_st<R, WW, TR, false>, g, 256, sst, s, F.lv_dev, T, \
             l2l_pairs_[p])
        switch (dn_w_[p]) {
            case 8: MLFMA_L2L_ST(8); break;
            case 12: MLFMA_L2L_ST(12); break;
            case 16: MLFMA_L2L_ST(16); break;
            case 24: MLFMA_L2L_ST(24); break;
            default: MLFMA_L2L_ST(32); break;
        }
#undef MLFMA_L2L_ST
        return;
    }
    const size_t smem = static_cast<size_t>(nth_[p]) * nph_[p + 1] * 2 * sizeof(C);
    switch (dn_w_[p]) {
        case 8: launch_k(pdl, k_l2l<R, 8, TR>, g, 256, smem, s, F.lv_dev, T, l2l_pairs_[p]); break;
        case 12: launch_k(pdl, k_l2l<R, 12, TR>, g, 256, smem, s, F.lv_dev, T, l2l_pairs_[p]); break;
        case 16: launch_k(pdl, k_l2l<R, 16, TR>, g, 256, smem, s, F.lv_dev, T, l2l_pairs_[p]); break;
        case 24: launch_k(pdl, k_l2l<R, 24, TR>, g, 256, smem, s, F.lv_dev, T, l2l_pairs_[p]); break;
        default: launch_k(pdl, k_l2l<R, 32, TR>, g, 256, smem, s, F.lv_dev, T, l2l_pairs_[p]); break;
    }
}

template <class R, bool TR>
void DeviceOp::far_l2t(FarField<R>& F, cudaStream_t s, bool pdl) {
    if (!n_l2t_items_) return;
    if constexpr (std::is_same<R, double>::value)
        launch_k(pdl, k_l2t<R, !TR>, n_l2t_items_, kL2TThreads, 0, s, F.lv_dev, l2t_items_, leaves_, F.pat, yfar_);
    else
        launch_k(pdl, k_l2t_half<R, !TR>, n_l2t_items_, kL2TThreads, 2 * sizeof(typename Cx<R>::T) * max_leaf_ndir_, s,
                 F.lv_dev, l2t_items_, leaves_, F.hpat, yfar_);
}

// stage: -1 all, 0 S2M, 1 M2M, 2 M2L, 3 L2L, 4 L2T, in sequence on s.
// TR: the transposed far field, Far^T = S2M^T L2L^T M2L^T M2M^T L2T^T, run in
// the same order with the mirrored kernels: conjugated patterns going up,
// interpolation with the shift after it (L2L^T), negated translation offsets,
// anterpolation with the shift after it (M2M^T), plain patterns coming down.
template <class R, bool TR>
void DeviceOp::run_far_t(FarField<R>& F, const double2* xt, cudaStream_t s, int stage) {
    if (n_leaves_ == 0) return;
    const bool tcf = std::is_same<R, float>::value && !TR;
    const bool tc_up = tcf && (tc_mode_ & 1), tc_dn = tcf && (tc_mode_ & 4);
    if (stage < 0 || stage == 0) far_s2m<R, TR>(F, xt, s);
    if (stage < 0 || stage == 1)
        for (int p = lmax_ - 1; p >= lmin_; --p) {
            if (tc_up) far_m2m_tc(p, 1, s); else far_m2m<R, TR>(F, p, s);
        }
    if (stage < 0 || stage == 2) far_m2l<R, TR>(F, lmin_, lmax_, s);
    if (stage < 0 || stage == 3)
        for (int p = lmin_; p < lmax_; ++p) {
            if (tc_dn) far_l2l_tc(p, 1, s); else far_l2l<R, TR>(F, p, s);
        }
    if (stage < 0 || stage == 4) far_l2t<R, TR>(F, s);
}

// The same chain with the translations of the finer levels taken off the
// critical path: M2L at level l needs only the outgoing patterns of level l,
// final once S2M (l = max level) or M2M(l+1 -> l) has run, so levels
// lmax..lmin+1 translate on s2 while the interpolations climb to the coarsest
// level on s; the anterpolations wait for both.
// near_late: the near field (on side_) starts once S2M has run, so that it
// overlaps the latency-bound stages instead of competing with S2M for
// bandwidth.  The finer levels' translations alternate between m2l_streams_
// side streams (s2, side3_).
template <class R, bool TR>
void DeviceOp::run_far_overlap_t(FarField<R>& F, const double2* xt, cudaStream_t s, cudaStream_t s2,
                                 bool near_late) {
    if (n_leaves_ == 0) return;
    if (lmax_ <= lmin_) {  // one far level: nothing to overlap
        run_far_t<R, TR>(F, xt, s, -1);
        return;
    }
    const bool tcf = std::is_same<R, float>::value && !TR;
    const bool tc_up = tcf && (tc_mode_ & 1), tc_dn = tcf && (tc_mode_ & 4);
    far_s2m<R, TR>(F, xt, s);
    // chain: the last operation on s is a kernel of the chain (a programmatic
    // dependent launch may follow it), not a memset or a join of side streams
    bool chain = (std::is_same<R, double>::value ? n_s2m_items_ : n_s2m_items_h_) > 0;
    cudaEventRecord(ev_level_[lmax_], s);
    if (near_late) {
        cudaStreamWaitEvent(side_, ev_level_[lmax_], 0);
        run_near(xt_, side_);
        cudaEventRecord(ev_join_, side_);
    }
    for (int p = lmax_ - 1; p >= lmin_; --p) {
        if (tc_up) far_m2m_tc(p, 1, s); else far_m2m<R, TR>(F, p, s, chain_pdl_ && chain);
        chain = chain || npar_[p] > 0;
        cudaEventRecord(ev_level_[p], s);
    }
    cudaStream_t ms[2] = {s2, side3_};
    // the second stream only when it gets a level (an event recorded on a
    // stream outside a capture cannot be waited on inside it)
    const int nms = m2l_streams_ > 1 && lmax_ - lmin_ >= 2 ? 2 : 1;
    for (int l = lmax_, i = 0; l > lmin_; --l, ++i) {
        cudaStream_t q = ms[i % nms];
        cudaStreamWaitEvent(q, ev_level_[l], 0);
        far_m2l<R, TR>(F, l, l, q);
    }
    cudaEventRecord(ev_m2l_done_, s2);
    if (nms > 1) cudaEventRecord(ev_m2l_done2_, side3_);
    far_m2l<R, TR>(F, lmin_, lmin_, s, chain_pdl_ && chain);
    cudaStreamWaitEvent(s, ev_m2l_done_, 0);
    if (nms > 1) cudaStreamWaitEvent(s, ev_m2l_done2_, 0);
    chain = false;  // the join: the next launch depends on more than one kernel
    for (int p = lmin_; p < lmax_; ++p) {
        if (tc_dn) far_l2l_tc(p, 1, s); else far_l2l<R, TR>(F, p, s, chain_pdl_ && chain);
        chain = chain || n_l2l_pairs_[p] > 0;
    }
    far_l2t<R, TR>(F, s, chain_pdl_ && chain);
}

void DeviceOp::run_far(const double2* xt, cudaStream_t s, int stage, int prec, bool tr) {
    if (prec < 0) prec = precision_;
    if (prec == kFp64) {
        if (tr) run_far_t<double, true>(f64_, xt, s, stage); else run_far_t<double, false>(f64_, xt, s, stage);
    } else {
        if (tr) run_far_t<float, true>(f32_, xt, s, stage); else run_far_t<float, false>(f32_, xt, s, stage);
    }
}

void DeviceOp::run_far_overlap(const double2* xt, cudaStream_t s, cudaStream_t s2, int prec, bool tr, bool late) {
    if (prec < 0) prec = precision_;
    if (prec == kFp64) {
        if (tr) run_far_overlap_t<double, true>(f64_, xt, s, s2, late);
        else run_far_overlap_t<double, false>(f64_, xt, s, s2, late);
    } else {
        if (tr) run_far_overlap_t<float, true>(f32_, xt, s, s2, late);
        else run_far_overlap_t<float, false>(f32_, xt, s, s2, late);
    }
}

void DeviceOp::run_near(const double2* xt, cudaStream_t s) {
    if (n_near_tiles_ == 0) {
        cudaMemsetAsync(ynear_, 0, sizeof(double2) * n_, s);
        return;
    }
    if (near_kernel_ == 2)
        k_near_direct<<<near_grid_, kNdThreads, 0, s>>>(near_tiles_, n_near_tiles_, near_bz_, xt, near_slot_,
                                                         near_part_);
    else if (near_kernel_ == 1)
        k_near_warp<<<near_grid_, kNwThreads, kNwSmemBytes, s>>>(near_tiles_, n_near_tiles_, near_bz_, xt, near_slot_,
                                                                 near_part_, err_dev_);
    else
        k_near_sym<<<near_grid_, kSymThreads, kSymSmemBytes, s>>>(near_tiles_, n_near_tiles_, near_bz_, xt, near_slot_,
                                                                 near_part_, err_dev_);
    k_near_reduce<<<blocks_for(static_cast<long long>(n_) * kReduceLanes, 256), 256, 0, s>>>(near_red_ptr_, near_part_,
                                                                                           n_, ynear_);
}

// The tree-ordered product xt_ -> (yfar_, ynear_): near field on the side
// stream, far-field chain on s in precision prec (transposed when tr).
// Captured once per (precision, direction) into a CUDA graph.  The near field
// is symmetric (each stored block is applied as Z and Z^T), so the transposed
// product reuses it; run_near writes every entry of ynear_.
void DeviceOp::enqueue_core(cudaStream_t s, int prec, bool tr) {
    // L2T writes (not adds) every far-leaf source's entry: zero yfar_ only
    // when some source sits in a leaf without far interactions
    if (!far_covers_all_) cudaMemsetAsync(yfar_, 0, sizeof(double2) * n_, s);
    cudaEventRecord(ev_fork_, s);
    const bool late = near_late_ && n_leaves_ > 0 && lmax_ > lmin_;
    if (!late) {
        cudaStreamWaitEvent(side_, ev_fork_, 0);
        run_near(xt_, side_);
        cudaEventRecord(ev_join_, side_);
    }
    run_far_overlap(xt_, s, side2_, prec, tr, late);
    cudaStreamWaitEvent(s, ev_join_, 0);
}

std::string DeviceOp::ensure_graph(int prec, bool tr) {
    const int t = tr ? 1 : 0;
    if (graph_exec_[prec][t] || !use_graph_) return {};
    MLFMA_CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    enqueue_core(stream_, prec, tr);
    MLFMA_CK(cudaStreamEndCapture(stream_, &graph_[prec][t]));
    MLFMA_CK(cudaGraphInstantiate(&graph_exec_[prec][t], graph_[prec][t], cudaGraphInstantiateFlagUseNodePriority));
    return {};
}

void DeviceOp::launch_core(cudaStream_t s, int prec, bool tr) {
    const int t = tr ? 1 : 0;
    if (graph_exec_[prec][t]) cudaGraphLaunch(graph_exec_[prec][t], s); else enqueue_core(s, prec, tr);
}

std::string DeviceOp::set_loads(const double2* z_user) {
    if (!ready_) return "operator not set up";
    MLFMA_CK(cudaSetDevice(device_));
    if (!z_user) {
        if (has_loads_) ++generation_;
        has_loads_ = false;
        return {};
    }
    ++generation_;
    if (!loads_) loads_ = alloc<double2>(n_);
    MLFMA_CK(cudaMemcpyAsync(yt_, z_user, sizeof(double2) * n_, cudaMemcpyHostToDevice, stream_));
    k_gather<<<blocks_for(n_, 256), 256, 0, stream_>>>(yt_, perm_, loads_, n_, 0);
    MLFMA_CK(cudaStreamSynchronize(stream_));
    has_loads_ = true;
    return {};
}

// Tree-ordered y = A x (adj: y = A^H x = conj(A^T conj(x))), loads included.
void DeviceOp::apply_tree(const double2* xt, double2* yt, cudaStream_t s, int prec, bool adj) {
    if (prec < 0) prec = precision_;
    if (!ensure_graph(prec, adj).empty()) use_graph_ = false;
    if (adj) k_conj_copy<<<blocks_for(n_, 256), 256, 0, s>>>(xt, xt_, n_);
    else if (xt != xt_) cudaMemcpyAsync(xt_, xt, sizeof(double2) * n_, cudaMemcpyDeviceToDevice, s);
    launch_core(s, prec, adj);
    k_finish<<<blocks_for(n_, 256), 256, 0, s>>>(yfar_, ynear_, nullptr, yt, n_, ck_, 0, xt_,
                                                 has_loads_ ? loads_ : nullptr, adj ? 1 : 0);
}

void DeviceOp::enqueue_apply_from_input(double2* yt, cudaStream_t s, int prec, bool adj) {
    if (prec < 0) prec = precision_;
    enqueue_core(s, prec, adj);
    k_finish<<<blocks_for(n_, 256), 256, 0, s>>>(yfar_, ynear_, nullptr, yt, n_, ck_, 0, xt_,
                                                 has_loads_ ? loads_ : nullptr, adj ? 1 : 0);
}

void DeviceOp::apply_tree_direct(const double2* xt, double2* yt, cudaStream_t s, int prec, bool adj) {
    if (prec < 0) prec = precision_;
    if (adj) k_conj_copy<<<blocks_for(n_, 256), 256, 0, s>>>(xt, xt_, n_);
    else if (xt != xt_) cudaMemcpyAsync(xt_, xt, sizeof(double2) * n_, cudaMemcpyDeviceToDevice, s);
    launch_core(s, prec, adj);
    k_finish<<<blocks_for(n_, 256), 256, 0, s>>>(yfar_, ynear_, nullptr, yt, n_, ck_, 0, xt_,
                                                 has_loads_ ? loads_ : nullptr, adj ? 1 : 0);
}

std::string DeviceOp::matvec_device(const double2* x, double2* y, bool accumulate, cudaStream_t stream, int prec,
                                    bool adj) {
    if (!ready_) return "operator not set up";
    if (prec < 0) prec = precision_;
    if (prec != kFp64 && precision_ == kFp64) return "the FP64 operator has no mixed far field";
    if (adj && ref_compat_) return "arg:the adjoint needs ref_compat = 0 (the reference's rule keeps state between products)";
    cudaStream_t s = stream ? stream : stream_;
    MLFMA_CK(cudaSetDevice(device_));
    std::string e = ensure_graph(prec, adj);
    if (!e.empty()) return e;
    k_gather<<<blocks_for(n_, 256), 256, 0, s>>>(x, perm_, xt_, n_, adj ? 1 : 0);
    launch_core(s, prec, adj);
    k_finish<<<blocks_for(n_, 256), 256, 0, s>>>(yfar_, ynear_, perm_, y, n_, ck_, accumulate ? 1 : 0, xt_,
                                                 has_loads_ ? loads_ : nullptr, adj ? 1 : 0);
    MLFMA_CK(cudaGetLastError());
    return {};
}

std::string DeviceOp::matvec_mapped(const double2* x, double2* y, bool accumulate, cudaStream_t stream) {
    if (!ready_) return "operator not set up";
    cudaStream_t s = stream ? stream : stream_;
    MLFMA_CK(cudaSetDevice(device_));
    std::string e = ensure_graph(precision_, false);
    if (!e.empty()) return e;
    k_gather_caller<<<blocks_for(n_, 256), 256, 0, s>>>(x, tpos_, xt_, n_);
    launch_core(s, precision_, false);
    k_finish_caller<<<blocks_for(n_, 256), 256, 0, s>>>(yfar_, ynear_, tpos_, y, n_, ck_, accumulate ? 1 : 0, xt_,
                                                        has_loads_ ? loads_ : nullptr);
    MLFMA_CK(cudaGetLastError());
    return {};
}

// One product y = A x (caller order, device) on stream s, without graph
// launches: for recording into a larger capture (many operators in one graph).
void DeviceOp::enqueue_matvec(const double2* x, double2* y, cudaStream_t s) {
    k_gather<<<blocks_for(n_, 256), 256, 0, s>>>(x, perm_, xt_, n_, 0);
    enqueue_core(s, precision_, false);
    k_finish<<<blocks_for(n_, 256), 256, 0, s>>>(yfar_, ynear_, perm_, y, n_, ck_, 0, xt_,
                                                 has_loads_ ? loads_ : nullptr, 0);
}

std::string DeviceOp::time_stages(StageTimes* out) {
    if (!ready_) return "operator not set up";
    MLFMA_CK(cudaSetDevice(device_));
    cudaEvent_t ev[9];
    for (auto& e : ev) MLFMA_CK(cudaEventCreate(&e));
    cudaStream_t s = stream_;
    cudaEventRecord(ev[0], s);
    cudaMemsetAsync(yfar_, 0, sizeof(double2) * n_, s);
    cudaEventRecord(ev[1], s);
    for (int st = 0; st < 5; ++st) {
        run_far(xt_, s, st);
        cudaEventRecord(ev[2 + st], s);
    }
    run_near(xt_, s);
    cudaEventRecord(ev[7], s);
    k_finish<<<blocks_for(n_, 256), 256, 0, s>>>(yfar_, ynear_, nullptr, yt_, n_, ck_, 0, xt_, nullptr, 0);
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

std::string DeviceOp::time_levels(std::vector<float>& out) {
    if (!ready_) return "operator not set up";
    MLFMA_CK(cudaSetDevice(device_));
    out.assign(3 * static_cast<size_t>(lmax_ + 1), 0.0f);
    if (n_leaves_ == 0) return {};
    const bool tcf = precision_ != kFp64;
    const bool tc_up = tcf && (tc_mode_ & 1), tc_dn = tcf && (tc_mode_ & 4);
    cudaStream_t s = stream_;
    cudaEvent_t a, b;
    MLFMA_CK(cudaEventCreate(&a));
    MLFMA_CK(cudaEventCreate(&b));
    auto timed = [&](auto&& fn) {
        cudaEventRecord(a, s);
        fn();
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        return ms;
    };
    if (precision_ == kFp64) far_s2m<double, false>(f64_, xt_, s); else far_s2m<float, false>(f32_, xt_, s);
    for (int p = lmax_ - 1; p >= lmin_; --p)
        out[3 * p] = timed([&] {
            if (tc_up) far_m2m_tc(p, 1, s);
            else if (precision_ == kFp64) far_m2m<double, false>(f64_, p, s);
            else far_m2m<float, false>(f32_, p, s);
        });
    for (int l = lmax_; l >= lmin_; --l)
        out[3 * l + 1] = timed([&] {
            if (precision_ == kFp64) far_m2l<double, false>(f64_, l, l, s); else far_m2l<float, false>(f32_, l, l, s);
        });
    for (int p = lmin_; p < lmax_; ++p)
        out[3 * p + 2] = timed([&] {
            if (tc_dn) far_l2l_tc(p, 1, s);
            else if (precision_ == kFp64) far_l2l<double, false>(f64_, p, s);
            else far_l2l<float, false>(f32_, p, s);
        });
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    MLFMA_CK(cudaGetLastError());
    return {};
}

std::string DeviceOp::farfield(const double2* cur, int ndir, const double* khat, double2* out, cudaStream_t s) {
    if (!ready_) return "operator not set up";
    if (ndir <= 0) return {};
    MLFMA_CK(cudaSetDevice(device_));
    k_farfield<<<ndir, kFarThreads, 0, s>>>(src_, perm_, cur, n_, khat, ck_, out);
    MLFMA_CK(cudaGetLastError());
    return {};
}

std::string DeviceOp::dense_rows(const int* rows, int nrows, const double2* x, double2* y, cudaStream_t s) {
    if (!ready_) return "operator not set up";
    if (nrows <= 0) return {};
    MLFMA_CK(cudaSetDevice(device_));
    k_dense_rows<<<nrows, kDenseThreads, 0, s>>>(src_, rows, perm_, x, n_, ck_, y);
    MLFMA_CK(cudaGetLastError());
    return {};
}

std::string DeviceOp::farfield_adjoint(const double2* F, int ndir, const double* khat, double2* g, cudaStream_t s,
                                       double2* PF) {
    if (!ready_) return "operator not set up";
    MLFMA_CK(cudaSetDevice(device_));
    if (ndir <= 0) {
        MLFMA_CK(cudaMemsetAsync(g, 0, sizeof(double2) * n_, s));
        return {};
    }
    k_project<<<blocks_for(ndir, 128), 128, 0, s>>>(khat, F, ndir, PF);
    k_farfield_adj<<<blocks_for(n_, 128), 128, 0, s>>>(src_, perm_, n_, khat, PF, ndir, ck_, g);
    MLFMA_CK(cudaGetLastError());
    return {};
}

std::string DeviceOp::dense_block(const int* rows, int nrows, double2* out, long long ld, cudaStream_t s) {
    if (!ready_) return "operator not set up";
    if (nrows <= 0) return {};
    MLFMA_CK(cudaSetDevice(device_));
    const dim3 grid(blocks_for(n_, kDenseThreads), nrows);
    k_dense_block<<<grid, kDenseThreads, 0, s>>>(src_, rows, perm_, n_, ck_, out, ld);
    MLFMA_CK(cudaGetLastError());
    return {};
}

namespace {
template <class C>
__global__ void k_widen(const C* __restrict__ src, double2* __restrict__ dst, long long n) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = to_d2(src[i]);
}
}  // namespace

std::string DeviceOp::bj_prepare() {
    if (!ready_) return "operator not set up";
    if (bj_gen_ == generation_ && bj_leaves_) return {};
    MLFMA_CK(cudaSetDevice(device_));
    if (h_bj_.empty()) return "arg:no leaves to precondition";
    if (!bj_leaves_) {
        long long entries = 0;
        for (const DevBjLeaf& L : h_bj_)
            if (L.nb <= kBjMax) entries += static_cast<long long>(L.nb) * L.nb;
        bj_leaves_ = upload(h_bj_);
        bj_ok_ = alloc<int>(h_bj_.size());
        bj_inv_ = alloc<double2>(static_cast<size_t>(std::max(1ll, entries)));
        int dev_smem = 0;
        MLFMA_CK(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device_));
        cudaFuncAttributes fa{};
        MLFMA_CK(cudaFuncGetAttributes(&fa, k_bj_build));
        MLFMA_CK(cudaFuncSetAttribute(k_bj_build, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      dev_smem - static_cast<int>(fa.sharedSizeBytes)));
    }
    const size_t smem = sizeof(double2) * 2 * kBjMax * kBjMax;
    k_bj_build<<<static_cast<int>(h_bj_.size()), kBjThreads, smem, stream_>>>(bj_leaves_, near_bz_, ck_,
                                                                             has_loads_ ? loads_ : nullptr, bj_inv_,
                                                                             bj_ok_);
    MLFMA_CK(cudaGetLastError());
    MLFMA_CK(cudaStreamSynchronize(stream_));
    bj_gen_ = generation_;
    return {};
}

void DeviceOp::bj_apply(const double2* x, double2* y, cudaStream_t s) {
    k_bj_apply<<<static_cast<int>(h_bj_.size()), kBjThreads, 0, s>>>(bj_leaves_, bj_ok_, bj_inv_, x, y);
}

std::string DeviceOp::copy_transl(int level, double2* host) {
    if (level < lmin_ || level > lmax_) return "level out of range";
    MLFMA_CK(cudaSetDevice(device_));
    MLFMA_CK(cudaStreamSynchronize(stream_));
    MLFMA_CK(cudaMemcpy(host, f64_.lv[level].transl, sizeof(double2) * 316 * ndir_[level], cudaMemcpyDeviceToHost));
    return {};
}

std::string DeviceOp::copy_level(int level, int which, double2* host, long long count) {
    if (level < lmin_ || level > lmax_) return "level out of range";
    const long long cnt = static_cast<long long>(nbox_[level]) * ndir_[level] * 2;
    if (count < cnt) return "buffer too small";
    MLFMA_CK(cudaSetDevice(device_));
    MLFMA_CK(cudaStreamSynchronize(stream_));
    if (precision_ == kFp64) {
        const DevLevelT<double>& d = f64_.lv[level];
        MLFMA_CK(cudaMemcpy(host, which ? d.B : d.A, cnt * sizeof(double2), cudaMemcpyDeviceToHost));
        return {};
    }
    const DevLevelT<float>& d = f32_.lv[level];
    double2* tmp = yt_;  // reuse work space in chunks of n
    for (long long o = 0; o < cnt; o += n_) {
        const long long m = std::min<long long>(n_, cnt - o);
        k_widen<float2><<<blocks_for(m, 256), 256, 0, stream_>>>((which ? d.B : d.A) + o, tmp, m);
        MLFMA_CK(cudaMemcpyAsync(host + o, tmp, m * sizeof(double2), cudaMemcpyDeviceToHost, stream_));
        MLFMA_CK(cudaStreamSynchronize(stream_));
    }
    return {};
}

// ================================================================= many right-hand sides

// Work items of the many-rhs kernels and the M2L sibling groups.
std::string DeviceOp::setup_multi(const Plan& plan) {
    const size_t nm = static_cast<size_t>(n_) * max_rhs_;
    xtm_ = alloc<double2>(nm);
    yfarm_ = alloc<double2>(nm);
    ynearm_ = alloc<double2>(nm);
    ytm_ = alloc<double2>(nm);
    MLFMA_CK(cudaMemset(xtm_, 0, nm * sizeof(double2)));
    MLFMA_CK(cudaMemset(yfarm_, 0, nm * sizeof(double2)));
    MLFMA_CK(cudaMemset(ynearm_, 0, nm * sizeof(double2)));
    // S2M and L2T: tiles of kBM pattern rows / sources per leaf.
    std::vector<int2> s2m, l2t;
    for (size_t i = 0; i < plan.far_leaves.size(); ++i) {
        const FarLeaf& f = plan.far_leaves[i];
        const int ne = 2 * plan.levels[f.level].ndir;
        for (int e0 = 0; e0 < ne; e0 += kBM) s2m.push_back(make_int2(static_cast<int>(i), e0));
        for (int s0 = 0; s0 < f.nsrc; s0 += kBM) l2t.push_back(make_int2(static_cast<int>(i), s0));
    }
    n_s2m_items_m_ = static_cast<int>(s2m.size());
    s2m_items_m_ = upload(s2m);
    n_l2t_items_m_ = static_cast<int>(l2t.size());
    l2t_items_m_ = upload(l2t);
    // Near field: tiles of kBM rows per block row.
    std::vector<int2> nit;
    for (size_t i = 0; i < plan.near_rows.size(); ++i)
        for (int r0 = 0; r0 < plan.near_rows[i].nrow; r0 += kBM) nit.push_back(make_int2(static_cast<int>(i), r0));
    n_near_items_m_ = static_cast<int>(nit.size());
    near_items_m_ = upload(nit);
    // Many-rhs M2L: weighted transfer values per (group, direction, candidate,
    // target), and direction-major items (the blocks in flight together all
    // read the patterns of one direction, 2 KB per box at 64 rhs, which stay
    // in L2 for every group that needs them).
    std::vector<cplx> t8;
    std::vector<int2> items;
    for (int l = lmin_; l <= lmax_; ++l) {
        const Level& L = plan.levels[l];
        std::vector<int> gl;
        for (size_t gi = 0; gi < h_groups_.size(); ++gi)
            if (h_groups_[gi].level == l) gl.push_back(static_cast<int>(gi));
        for (int gi : gl) {
            DevM2LGroup& g = h_groups_[gi];
            g.t8_off = static_cast<long long>(t8.size());
            t8.resize(t8.size() + static_cast<size_t>(L.ndir) * g.ncand * kMaxGroup, cplx(0));
            for (int d = 0; d < L.ndir; ++d)
                for (int c = 0; c < g.ncand; ++c)
                    for (int t = 0; t < kMaxGroup; ++t) {
                        const int o = h_cand_off_[(static_cast<size_t>(g.cand0) + c) * kMaxGroup + t];
                        if (o >= 0)
                            t8[g.t8_off + (static_cast<size_t>(d) * g.ncand + c) * kMaxGroup + t] =
                                L.transl[static_cast<size_t>(o) * L.ndir + d] * L.m2l_w[d];
                    }
        }
        for (int d = 0; d < L.ndir; ++d)
            for (int gi : gl) items.push_back(make_int2(gi, d));
    }
    MLFMA_CK(h2d_landed(m2l_groups_, h_groups_.data(), sizeof(DevM2LGroup) * h_groups_.size()));
    f64_.m2l_t8 = upload(conv_c<double2>(t8));
    if (precision_ != kFp64) f32_.m2l_t8 = upload(conv_c<float2>(t8));
    n_m2l_items_m_ = static_cast<int>(items.size());
    m2l_items_m_ = upload(items);
    return {};
}

// M2L sibling groups of the many-rhs path: the boxes of a level that share a
// parent node (at most 8) and the union of their list-2 sources, with each
// candidate's offset id towards every target (-1: not in that target's list 2).
// (A one-vector M2L over the same groups measured slower than the per-box
// kernel k_m2l: 59 against 58 us in FP64, 55 against 37 us mixed, on the
// r = 2 lambda sphere; its few, register-heavy blocks do not hide latency.)
std::string DeviceOp::build_m2l_groups(const Plan& plan) {
    h_groups_.clear();
    h_cand_off_.clear();
    std::vector<int> cand_src;
    for (int l = lmin_; l <= lmax_; ++l) {
        const Level& L = plan.levels[l];
        std::vector<int> order(L.boxes.size());
        for (size_t b = 0; b < order.size(); ++b) order[b] = static_cast<int>(b);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            return plan.nodes[L.boxes[a]].parent < plan.nodes[L.boxes[b]].parent;
        });
        for (size_t i = 0; i < order.size();) {
            const int par = plan.nodes[L.boxes[order[i]]].parent;
            size_t j = i;
            while (j < order.size() && plan.nodes[L.boxes[order[j]]].parent == par) ++j;
            if (j - i > static_cast<size_t>(kMaxGroup)) return "internal: sibling group larger than 8";
            DevM2LGroup g{};
            g.level = l;
            g.ntgt = static_cast<int>(j - i);
            g.cand0 = static_cast<int>(cand_src.size());
            std::vector<int> cands;
            std::vector<std::array<short, kMaxGroup>> offs;
            for (int t = 0; t < g.ntgt; ++t) {
                const int b = order[i + t];
                g.tgt[t] = b;
                if (L.m2l_ptr[b + 1] == L.m2l_ptr[b]) g.empty_mask |= 1 << t;
                for (int q = L.m2l_ptr[b]; q < L.m2l_ptr[b + 1]; ++q) {
                    const int src = L.m2l_src[q];
                    size_t c = 0;
                    while (c < cands.size() && cands[c] != src) ++c;
                    if (c == cands.size()) {
                        cands.push_back(src);
                        std::array<short, kMaxGroup> o;
                        o.fill(-1);
                        offs.push_back(o);
                    }
                    offs[c][t] = static_cast<short>(L.m2l_off[q]);
                }
            }
            i = j;
            const bool all_empty = g.empty_mask == (1 << g.ntgt) - 1;
            if (all_empty && ref_compat_) continue;  // nothing written (node.cpp:106-108)
            g.ncand = static_cast<int>(cands.size());
            for (size_t c = 0; c < cands.size(); ++c) {
                cand_src.push_back(cands[c]);
                h_cand_off_.insert(h_cand_off_.end(), offs[c].begin(), offs[c].end());
            }
            h_groups_.push_back(g);
        }
    }
    m2l_groups_ = upload(h_groups_);
    m2l_cand_src_ = upload(cand_src);
    return {};
}

// stage: -1 all, 0 S2M, 1 M2M, 2 M2L, 3 L2L, 4 L2T.
template <class R>
void DeviceOp::run_far_multi_t(FarField<R>& F, int nr, cudaStream_t s, int stage) {
    using C = typename Cx<R>::T;
    if (n_leaves_ == 0) return;
    if ((stage < 0 || stage == 0) && n_s2m_items_m_)
        k_s2m_m<R><<<n_s2m_items_m_, kGemmThreads, 0, s>>>(F.lv_dev, s2m_items_m_, leaves_, F.pat, xtm_, nr);
    const bool tc_up = std::is_same<R, float>::value && (tc_mode_ & 2);
    const bool tc_dn = std::is_same<R, float>::value && (tc_mode_ & 8);
    if ((stage < 0 || stage == 1) && tc_up)
        for (int p = lmax_ - 1; p >= lmin_; --p) far_m2m_tc(p, nr, s);
    if ((stage < 0 || stage == 1) && !tc_up)
        for (int p = lmax_ - 1; p >= lmin_; --p) {
            if (npar_[p] == 0) continue;
            constexpr int rc = 16 * m2m_rpl<R>();
            const int rows_fast = m_m2m_rows_fast_ < 0 ? (m2m_rows_fast<R>() ? 1 : 0) : m_m2m_rows_fast_;
            const dim3 grid = rows_fast ? dim3(nth_[p], (nr + rc - 1) / rc, npar_[p])
                                        : dim3(npar_[p], nth_[p], (nr + rc - 1) / rc);
            const size_t smem = static_cast<size_t>(nph_[p + 1]) * 32 * m2m_rpl<R>() * sizeof(C);
            const DevTransT<R>& T = F.trans[p];
            const bool small = nph_[p] <= 8 * kInterpWarps;
#define MLFMA_M2M_M(WW)                                                                        \
    (small ? k_m2m_m<R, WW, 8><<<grid, kInterpThreads, smem, s>>>(F.lv_dev, T, nr, rows_fast)            \
           : k_m2m_m<R, WW, kM2MOut><<<grid, kInterpThreads, smem, s>>>(F.lv_dev, T, nr, rows_fast))
            switch (up_w_[p]) {
                case 2: MLFMA_M2M_M(2); break;
                case 4: MLFMA_M2M_M(4); break;
                case 6: MLFMA_M2M_M(6); break;
                case 8: MLFMA_M2M_M(8); break;
                default: MLFMA_M2M_M(10); break;
            }
#undef MLFMA_M2M_M
        }
    if ((stage < 0 || stage == 2) && n_m2l_items_m_) {
        const int threads = std::min(kM2LmThreads, ((2 * nr + 31) / 32) * 32);
        k_m2l_m<R><<<n_m2l_items_m_, threads, 0, s>>>(F.lv_dev, m2l_items_m_, m2l_groups_, m2l_cand_src_,
                                                      F.m2l_t8, nr, ref_compat_ ? 0 : 1);
    }
    if ((stage < 0 || stage == 3) && tc_dn)
        for (int p = lmin_; p < lmax_; ++p) far_l2l_tc(p, nr, s);
    if ((stage < 0 || stage == 3) && !tc_dn)
        for (int p = lmin_; p < lmax_; ++p) {
            const int g = n_l2l_pairs_[p];
            if (!g) continue;
            const int pairs = m_l2l_pairs_ > 0 ? m_l2l_pairs_ : l2l_pairs<R>();
            const dim3 grid(g, (nph_[p + 1] / 2 + pairs - 1) / pairs, (nr + kRc - 1) / kRc);
            const size_t smem = static_cast<size_t>(nth_[p]) * 2 * pairs * 64 * sizeof(C) +
                                static_cast<size_t>(nth_[p + 1]) * dn_w_[p] * (sizeof(R) + 2 * sizeof(int));
            const DevTransT<R>& T = F.trans[p];
#define MLFMA_L2L_M(WW)                                                                                    \
    (pairs == 1 ? k_l2l_m<R, WW, 1><<<grid, kInterpThreads, smem, s>>>(F.lv_dev, T, l2l_pairs_[p], nr)     \
                : k_l2l_m<R, WW, 2><<<grid, kInterpThreads, smem, s>>>(F.lv_dev, T, l2l_pairs_[p], nr))
            switch (dn_w_[p]) {
                case 8: MLFMA_L2L_M(8); break;
                case 12: MLFMA_L2L_M(12); break;
                case 16: MLFMA_L2L_M(16); break;
                case 24: MLFMA_L2L_M(24); break;
                default: MLFMA_L2L_M(32); break;
            }
#undef MLFMA_L2L_M
        }
    if ((stage < 0 || stage == 4) && n_l2t_items_m_)
        k_l2t_m<R><<<n_l2t_items_m_, kGemmThreads, 0, s>>>(F.lv_dev, l2t_items_m_, leaves_, F.pat, yfarm_, nr);
}

void DeviceOp::run_far_multi(int nr, cudaStream_t s, int stage, int prec) {
    if (prec < 0) prec = precision_;
    if (prec == kFp64) run_far_multi_t(f64_, nr, s, stage); else run_far_multi_t(f32_, nr, s, stage);
}

void DeviceOp::run_near_multi(int nr, cudaStream_t s) {
    if (n_near_items_m_ == 0) return;
    k_near_m<<<n_near_items_m_, kGemmThreads, 0, s>>>(near_rows_, near_items_m_, near_z_, near_cols_, xtm_, ynearm_,
                                                       nr);
}

// xtm_ -> (yfarm_, ynearm_): near field on the side stream, far field on s.
void DeviceOp::enqueue_multi(int nr, cudaStream_t s, int prec) {
    const size_t bytes = sizeof(double2) * static_cast<size_t>(n_) * nr;
    cudaMemsetAsync(yfarm_, 0, bytes, s);
    cudaMemsetAsync(ynearm_, 0, bytes, s);
    cudaEventRecord(ev_fork_, s);
    cudaStreamWaitEvent(side_, ev_fork_, 0);
    run_near_multi(nr, side_);
    cudaEventRecord(ev_join_, side_);
    run_far_multi(nr, s, -1, prec);
    cudaStreamWaitEvent(s, ev_join_, 0);
}

std::string DeviceOp::matvec_multi_device(const double2* x, double2* y, int nr, bool accumulate, cudaStream_t stream,
                                          int prec) {
    if (!ready_) return "operator not set up";
    if (nr < 1 || nr > max_rhs_) return "arg:nrhs must be between 1 and the operator's max_rhs";
    if (prec < 0) prec = precision_;
    if (prec != kFp64 && precision_ == kFp64) return "the FP64 operator has no mixed far field";
    cudaStream_t s = stream ? stream : stream_;
    MLFMA_CK(cudaSetDevice(device_));
    const long long tot = static_cast<long long>(n_) * nr;
    k_gather_m<<<blocks_for(tot, 256), 256, 0, s>>>(x, perm_, xtm_, n_, nr);
    enqueue_multi(nr, s, prec);
    k_finish_m<<<blocks_for(tot, 256), 256, 0, s>>>(yfarm_, ynearm_, perm_, y, n_, nr, ck_, accumulate ? 1 : 0, xtm_,
                                                     has_loads_ ? loads_ : nullptr);
    MLFMA_CK(cudaGetLastError());
    return {};
}

void DeviceOp::apply_tree_multi(const double2* xt, double2* yt, int nr, cudaStream_t s, int prec) {
    if (prec < 0) prec = precision_;
    const long long tot = static_cast<long long>(n_) * nr;
    if (xt != xtm_) cudaMemcpyAsync(xtm_, xt, sizeof(double2) * tot, cudaMemcpyDeviceToDevice, s);
    enqueue_multi(nr, s, prec);
    k_finish_m<<<blocks_for(tot, 256), 256, 0, s>>>(yfarm_, ynearm_, nullptr, yt, n_, nr, ck_, 0, xtm_,
                                                     has_loads_ ? loads_ : nullptr);
}

std::string DeviceOp::time_stages_multi(int nr, StageTimes* out) {
    if (!ready_) return "operator not set up";
    if (nr < 1 || nr > max_rhs_) return "arg:nrhs must be between 1 and the operator's max_rhs";
    MLFMA_CK(cudaSetDevice(device_));
    cudaEvent_t ev[9];
    for (auto& e : ev) MLFMA_CK(cudaEventCreate(&e));
    cudaStream_t s = stream_;
    const size_t bytes = sizeof(double2) * static_cast<size_t>(n_) * nr;
    cudaEventRecord(ev[0], s);
    cudaMemsetAsync(yfarm_, 0, bytes, s);
    cudaMemsetAsync(ynearm_, 0, bytes, s);
    cudaEventRecord(ev[1], s);
    for (int st = 0; st < 5; ++st) {
        run_far_multi(nr, s, st, precision_);
        cudaEventRecord(ev[2 + st], s);
    }
    run_near_multi(nr, s);
    cudaEventRecord(ev[7], s);
    const long long tot = static_cast<long long>(n_) * nr;
    k_finish_m<<<blocks_for(tot, 256), 256, 0, s>>>(yfarm_, ynearm_, nullptr, ytm_, n_, nr, ck_, 0, xtm_, nullptr);
    cudaEventRecord(ev[8], s);
    MLFMA_CK(cudaEventSynchronize(ev[8]));
    float t[8];
    for (int i = 0; i < 8; ++i) cudaEventElapsedTime(&t[i], ev[i], ev[i + 1]);
    *out = StageTimes{t[0], t[1], t[2], t[3], t[4], t[5], t[6], t[7], 0.f};
    cudaEventElapsedTime(&out->total, ev[0], ev[8]);
    for (auto& e : ev) cudaEventDestroy(e);
    MLFMA_CK(cudaGetLastError());
    return {};
}

// ================================================================= tensor-core interpolation

namespace {

// The shared-memory limit is a property of the kernel, shared by every
// operator: set it to the device's opt-in maximum less the kernel's static
// shared memory; *dyn_max receives that limit.
template <int KIND>
cudaError_t tc_prepare(int smem, int* dyn_max) {
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, k_tc_pass<KIND>);
    if (e != cudaSuccess) return e;
    *dyn_max = smem - static_cast<int>(fa.sharedSizeBytes);
    return cudaFuncSetAttribute(k_tc_pass<KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, *dyn_max);
}

}  // namespace

// Weights, contraction tables and the intermediate buffer of the tensor-core
// passes of every transition; tc_ok_ stays false (the CUDA-core kernels run)
// when a grid needs more shared memory than a CTA has.
std::string DeviceOp::setup_tc(const Plan& plan) {
    tc_ok_ = false;
    tc_.assign(std::max(lmax_, 0) + 1, TcTrans{});
    int dev_smem = 0;
    MLFMA_CK(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device_));
    if (!sms_) MLFMA_CK(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_));
    size_t scr_one = 1, scr_many = 1;
    for (int p = lmin_; p < lmax_; ++p) {
        const Transition& T = plan.trans[p];
        TcTrans& t = tc_[p];
        TcDense d[4];
        std::string e;
        if ((e = tc_dense_weights(T.up_th, nth_[p + 1], true, d[kTcTheta])).size() ||
            (e = tc_dense_weights(T.up_ph, nph_[p + 1], false, d[kTcPhi])).size() ||
            (e = tc_dense_weights(T.dn_ph, nph_[p], false, d[kTcPhiT])).size() ||
            (e = tc_dense_weights(T.dn_th, nth_[p], true, d[kTcThetaT])).size())
            return {};  // not expressible: keep the CUDA-core kernels
        for (int k = 0; k < 4; ++k) {
            t.K[k] = d[k].K;
            t.Kpad[k] = (d[k].K + 7) / 8 * 8;
            t.N[k] = d[k].N;
            t.Npad[k] = (d[k].N + 15) / 16 * 16;
            if (t.Npad[k] > 256) return {};
            t.smem[k] = tc_smem_bytes(t.Npad[k], t.Kpad[k], t.K[k]);
            if (t.smem[k] > static_cast<size_t>(dev_smem)) return {};
        }
        for (int k = 0; k < 4; ++k) {
            t.w[k] = upload(tc_pack_weights(d[k], t.Npad[k], t.Kpad[k]));
            if (k == kTcTheta || k == kTcThetaT) t.krow[k] = upload(d[k].krow);
        }
        const size_t per_item = static_cast<size_t>(nth_[p]) * nph_[p + 1] * 4;  // one vector: [nth_p][mph][4]
        const size_t items = static_cast<size_t>(std::max(npar_[p], n_l2l_pairs_[p]));
        scr_one = std::max(scr_one, per_item * items);
        scr_many = std::max(scr_many, per_item * items * max_rhs_);
    }
    // many right-hand sides: items in chunks whose intermediate fits the buffer
    // (at most 64 MB beyond what one vector needs)
    tc_scratch_floats_ = std::max(scr_one, std::min(scr_many, static_cast<size_t>(16) << 20));
    for (int p = lmin_; p < lmax_; ++p)  // one item's intermediate must fit (chunks of at least one item)
        if (static_cast<size_t>(nth_[p]) * nph_[p + 1] * 4 * max_rhs_ > tc_scratch_floats_) return {};
    tc_scratch_ = alloc<float>(tc_scratch_floats_);
    int dyn[4] = {};
    MLFMA_CK(tc_prepare<kTcTheta>(dev_smem, &dyn[kTcTheta]));
    MLFMA_CK(tc_prepare<kTcPhi>(dev_smem, &dyn[kTcPhi]));
    MLFMA_CK(tc_prepare<kTcPhiT>(dev_smem, &dyn[kTcPhiT]));
    MLFMA_CK(tc_prepare<kTcThetaT>(dev_smem, &dyn[kTcThetaT]));
    for (int p = lmin_; p < lmax_; ++p)
        for (int k = 0; k < 4; ++k)
            if (tc_[p].smem[k] > static_cast<size_t>(dyn[k])) return {};  // keep the CUDA-core kernels
    const auto ncols_of = [](int npad) { int c = 32; while (c < npad) c <<= 1; return c; };
    const void* fns[4] = {reinterpret_cast<const void*>(k_tc_pass<kTcTheta>),
                          reinterpret_cast<const void*>(k_tc_pass<kTcPhi>),
                          reinterpret_cast<const void*>(k_tc_pass<kTcPhiT>),
                          reinterpret_cast<const void*>(k_tc_pass<kTcThetaT>)};
    int sm_bytes = 0, sm_regs = 0;
    MLFMA_CK(cudaDeviceGetAttribute(&sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device_));
    MLFMA_CK(cudaDeviceGetAttribute(&sm_regs, cudaDevAttrMaxRegistersPerMultiprocessor, device_));
    for (int p = lmin_; p < lmax_; ++p)
        for (int k = 0; k < 4; ++k) {
            // persistent CTAs: as many per SM as shared memory (with the 1 KB
            // each block reserves), registers, warps and the 512 tensor-memory
            // columns of an SM allow
            TcTrans& t = tc_[p];
            cudaFuncAttributes fa{};
            MLFMA_CK(cudaFuncGetAttributes(&fa, fns[k]));
            MLFMA_CK(cudaFuncSetAttribute(fns[k], cudaFuncAttributePreferredSharedMemoryCarveout, 100));
            const int by_smem = sm_bytes / static_cast<int>(t.smem[k] + fa.sharedSizeBytes + 1024);
            const int by_regs = sm_regs / std::max(1, fa.numRegs * kTcThreads);
            const int occ = std::max(1, std::min({by_smem, by_regs, 64 / (kTcThreads / 32), 512 / ncols_of(t.Npad[k])}));
            t.grid[k] = occ * sms_;
        }
    tc_ok_ = true;
    return {};
}

namespace {
TcArgs tc_args_common(int nr, const DevTransT<float>& T, const TcTrans& t, int kind, int mth, int mph, int nth,
                      int nph) {
    TcArgs a{};
    a.K = t.K[kind];
    a.Kpad = t.Kpad[kind];
    a.N = t.N[kind];
    a.Npad = t.Npad[kind];
    a.w = t.w[kind];
    a.krow = t.krow[kind];
    a.nr = nr;
    a.Q = 4 * nr;
    a.mth = mth;
    a.mph = mph;
    a.nth = nth;
    a.nph = nph;
    a.child_ptr = T.child_ptr;
    a.child_box = T.child_box;
    a.child_oct = T.child_oct;
    a.par_box = T.par_box;
    return a;
}

template <int KIND>
void tc_launch(const TcArgs& a, const TcTrans& t, int* err, cudaStream_t s) {
    const long long rows = static_cast<long long>(a.J) * a.Q * a.nitems;
    const long long tiles = (rows + kTcRows - 1) / kTcRows;
    if (tiles <= 0) return;
    const int grid = static_cast<int>(std::min<long long>(tiles, t.grid[KIND]));
    k_tc_pass<KIND><<<grid, kTcThreads, t.smem[KIND], s>>>(a, err);
}
}  // namespace

// M2M of transition p on nr right-hand sides (nr = 1: the one-vector
// patterns A; nr > 1: the many-rhs patterns Am), parents in chunks whose
// intermediate fits the buffer.
void DeviceOp::far_m2m_tc(int p, int nr, cudaStream_t s) {
    if (npar_[p] == 0) return;
    const TcTrans& t = tc_[p];
    const DevTransT<float>& T = f32_.trans[p];
    const DevLevelT<float>& P = f32_.lv[p];
    const DevLevelT<float>& C = f32_.lv[p + 1];
    const size_t per_item = static_cast<size_t>(nth_[p]) * nph_[p + 1] * 4 * nr;
    const int chunk = static_cast<int>(std::max<size_t>(1, std::min<size_t>(npar_[p], tc_scratch_floats_ / per_item)));
    for (int i0 = 0; i0 < npar_[p]; i0 += chunk) {
        const int ni = std::min(chunk, npar_[p] - i0);
        TcArgs a = tc_args_common(nr, T, t, kTcTheta, nth_[p + 1], nph_[p + 1], nth_[p], nph_[p]);
        a.item0 = i0;
        a.nitems = ni;
        a.J = nph_[p + 1];
        a.pat_in = nr == 1 ? C.A : C.Am;
        a.shift = C.shift_up;
        a.scr_out = tc_scratch_;
        tc_launch<kTcTheta>(a, t, err_dev_, s);
        TcArgs b = tc_args_common(nr, T, t, kTcPhi, nth_[p + 1], nph_[p + 1], nth_[p], nph_[p]);
        b.item0 = i0;
        b.nitems = ni;
        b.J = nth_[p];
        b.scr_in = tc_scratch_;
        b.pat_out = nr == 1 ? P.A : P.Am;
        tc_launch<kTcPhi>(b, t, err_dev_, s);
    }
}

// L2L of transition p on nr right-hand sides, (parent, child) pairs in chunks.
void DeviceOp::far_l2l_tc(int p, int nr, cudaStream_t s) {
    const int npairs = n_l2l_pairs_[p];
    if (npairs == 0) return;
    const TcTrans& t = tc_[p];
    const DevTransT<float>& T = f32_.trans[p];
    const DevLevelT<float>& P = f32_.lv[p];
    const DevLevelT<float>& C = f32_.lv[p + 1];
    const size_t per_item = static_cast<size_t>(nth_[p]) * nph_[p + 1] * 4 * nr;
    const int chunk = static_cast<int>(std::max<size_t>(1, std::min<size_t>(npairs, tc_scratch_floats_ / per_item)));
    for (int i0 = 0; i0 < npairs; i0 += chunk) {
        const int ni = std::min(chunk, npairs - i0);
        TcArgs a = tc_args_common(nr, T, t, kTcPhiT, nth_[p + 1], nph_[p + 1], nth_[p], nph_[p]);
        a.item0 = i0;
        a.nitems = ni;
        a.J = nth_[p];
        a.pat_in = nr == 1 ? P.B : P.Bm;
        a.shift = P.shift_down;
        a.pairs = l2l_pairs_[p];
        a.scr_out = tc_scratch_;
        tc_launch<kTcPhiT>(a, t, err_dev_, s);
        TcArgs b = tc_args_common(nr, T, t, kTcThetaT, nth_[p + 1], nph_[p + 1], nth_[p], nph_[p]);
        b.item0 = i0;
        b.nitems = ni;
        b.J = nph_[p + 1];
        b.pairs = l2l_pairs_[p];
        b.scr_in = tc_scratch_;
        b.pat_out = nr == 1 ? C.B : C.Bm;
        tc_launch<kTcThetaT>(b, t, err_dev_, s);
    }
}

void DeviceOp::drop_graphs() {
    for (int p = 0; p < 2; ++p)
        for (int t = 0; t < 2; ++t) {
            if (graph_exec_[p][t]) cudaGraphExecDestroy(graph_exec_[p][t]);
            if (graph_[p][t]) cudaGraphDestroy(graph_[p][t]);
            graph_exec_[p][t] = nullptr;
            graph_[p][t] = nullptr;
        }
}

std::string DeviceOp::set_tc(int mode) {
    if (!ready_) return "operator not set up";
    if (mode < 0 || mode > 15) return "arg:mode must be 0..15";
    if (mode && !tc_ok_)
        return "arg:no tensor-core interpolation on this operator (FP64 far field only, or a grid too large)";
    if ((mode & 10) && max_rhs_ < 2) return "arg:the many-right-hand-side modes need max_rhs > 1";
    MLFMA_CK(cudaSetDevice(device_));
    MLFMA_CK(cudaStreamSynchronize(stream_));
    tc_mode_ = mode;
    drop_graphs();  // recaptured with the chosen kernels on the next product
    ++generation_;
    return {};
}

std::string DeviceOp::set_near_kernel(int kind) {
    if (!ready_) return "operator not set up";
    if (kind < 0 || kind > 2) return "arg:kind must be 0, 1 or 2";
    MLFMA_CK(cudaSetDevice(device_));
    MLFMA_CK(cudaStreamSynchronize(stream_));
    near_kernel_ = kind;
    near_per_sm_ = kind == 2 ? near_direct_occ_ : kind == 1 ? 1 : near_occ_;
    set_near_grid(near_per_sm_);
    drop_graphs();
    ++generation_;
    return {};
}

std::string DeviceOp::set_schedule(int schedule) {
    if (!ready_) return "operator not set up";
    if (schedule < 0 || schedule > 15) return "arg:schedule must be 0..15";
    MLFMA_CK(cudaSetDevice(device_));
    MLFMA_CK(cudaStreamSynchronize(stream_));
    m2l_staged_ = schedule & 1;
    near_late_ = (schedule & 2) != 0;
    m2l_streams_ = (schedule & 4) ? 2 : 1;
    chain_pdl_ = (schedule & 8) != 0;
    drop_graphs();
    ++generation_;
    return {};
}

std::string DeviceOp::set_staged(int mode) {
    if (!ready_) return "operator not set up";
    if (mode < 0 || mode > 15) return "arg:mode must be 0..15";
    MLFMA_CK(cudaSetDevice(device_));
    MLFMA_CK(cudaStreamSynchronize(stream_));
    const int kind = (mode & 4) ? 2 : 1;
    for (int p = lmin_; p < lmax_; ++p) {
        m2m_pref_[p] = (mode & 1) ? kind : 0;
        l2l_pref_[p] = (mode & 8) ? 3 : (mode & 2) ? kind : 0;
    }
    drop_graphs();
    ++generation_;
    return {};
}

// ================================================================= autotuner

// Times the candidate launch shapes of the stages on this operator (CUDA
// events on the operator's stream, after one untimed launch each) and keeps
// the fastest: nr = 1 tunes the one-vector path (M2L directions per block,
// M2M parent rows per block per level transition), nr > 1 the many-rhs path at
// that width (interpolation grid order, anterpolation column pairs).  The
// local patterns are saved and restored around the trial launches, so the
// reference's stale-local rule sees no change; captured graphs are dropped
// and recaptured with the new shapes on the next product.
std::string DeviceOp::autotune(int nr, int reps, TuneReport* rep) {
    if (!ready_) return "operator not set up";
    if (nr < 1 || (nr > 1 && nr > max_rhs_)) return "arg:nrhs must be 1 or between 2 and the operator's max_rhs";
    if (reps < 1) reps = 5;
    MLFMA_CK(cudaSetDevice(device_));
    cudaStream_t s = stream_;
    int dev_smem = 0;
    MLFMA_CK(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device_));
    const size_t csize = precision_ == kFp64 ? sizeof(double2) : sizeof(float2);
    // save the local patterns of the tuned precision
    std::vector<std::pair<void*, size_t>> saved;
    std::vector<void*> tmp;
    auto save = [&](void* p, size_t bytes) -> std::string {
        void* t = nullptr;
        MLFMA_CK(cudaMalloc(&t, bytes));
        MLFMA_CK(cudaMemcpyAsync(t, p, bytes, cudaMemcpyDeviceToDevice, s));
        saved.emplace_back(p, bytes);
        tmp.push_back(t);
        return {};
    };
    for (int l = lmin_; l <= lmax_; ++l) {
        const size_t cnt = static_cast<size_t>(nbox_[l]) * ndir_[l] * 2;
        void* B = precision_ == kFp64 ? static_cast<void*>(f64_.lv[l].B) : static_cast<void*>(f32_.lv[l].B);
        void* Bm = precision_ == kFp64 ? static_cast<void*>(f64_.lv[l].Bm) : static_cast<void*>(f32_.lv[l].Bm);
        std::string e = save(B, cnt * csize);
        if (!e.empty()) return e;
        if (nr > 1 && Bm) {
            e = save(Bm, cnt * max_rhs_ * csize);
            if (!e.empty()) return e;
        }
    }
    cudaEvent_t e0, e1;
    MLFMA_CK(cudaEventCreate(&e0));
    MLFMA_CK(cudaEventCreate(&e1));
    auto timed = [&](const auto& launch) -> float {
        launch();
        cudaEventRecord(e0, s);
        for (int i = 0; i < reps; ++i) launch();
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms / reps;
    };
    TuneReport r{};
    r.near_blocks_per_sm = near_per_sm_;
    if (nr == 1) {
        auto product = [&] { enqueue_core(s, precision_, false); };
        r.before_ms = timed(product);
        // M2L: directions per block
        float best = 1e30f;
        int best_chunk = m2l_chunk_;
        for (int chunk : {32, 64, 96, 128}) {  // k_m2l runs 128 threads: one direction each
            build_m2l_items(chunk);
            const float t = timed([&] { run_far(xt_, s, 2, precision_, false); });
            if (t < best) { best = t; best_chunk = chunk; }
        }
        build_m2l_items(best_chunk);
        r.m2l_chunk = best_chunk;
        // M2M: kernel (per child or children summed first, staged) and parent
        // rows per block, per transition; L2L: kernel (staged or not)
        for (int p = lmin_; p < lmax_; ++p) {
            if (!npar_[p]) continue;
            float bt = 1e30f;
            int brows = m2m_rows_[p], bkind = m2m_pref_[p];
            for (int kind : {0, 1, 2})
                for (int rows : {1, 2, 4, 8, 16, 32, 64}) {
                    if (rows > nth_[p] && rows != 1) continue;
                    const size_t need = kind ? m2m_sum_smem(nth_[p + 1], nph_[p + 1], rows, csize) + 1024
                                             : static_cast<size_t>(8) * rows * nph_[p + 1] * 2 * csize;
                    if (need > static_cast<size_t>(dev_smem) || (!kind && rows > 16)) continue;
                    m2m_rows_[p] = rows;
                    m2m_pref_[p] = kind;
                    const float t = timed([&] {
                        if (precision_ == kFp64) far_m2m<double, false>(f64_, p, s); else far_m2m<float, false>(f32_, p, s);
                    });
                    if (t < bt) { bt = t; brows = rows; bkind = kind; }
                }
            m2m_rows_[p] = brows;
            m2m_pref_[p] = bkind;
            r.m2m_rows[p] = brows;
            if (n_l2l_pairs_[p]) {
                float lt = 1e30f;
                int lkind = l2l_pref_[p];
                for (int kind : {0, 1, 2, 3}) {
                    l2l_pref_[p] = kind;
                    const float t = timed([&] {
                        if (precision_ == kFp64) far_l2l<double, false>(f64_, p, s); else far_l2l<float, false>(f32_, p, s);
                    });
                    if (t < lt) { lt = t; lkind = kind; }
                }
                l2l_pref_[p] = lkind;
            }
        }
        // near field: persistent blocks per SM, timed on the whole product (it
        // runs beside the far-field chain and competes with it for the SMs)
        if (n_near_tiles_) {
            float bt = 1e30f;
            int bk = near_per_sm_, bkind = near_kernel_;
            for (int kind : {0, 1, 2})
                for (int k : kind == 2 ? std::vector<int>{near_direct_occ_ / 2, near_direct_occ_}
                                       : kind == 1 ? std::vector<int>{1} : [&] {
                                             std::vector<int> v;
                                             for (int q = 1; q <= near_occ_; ++q) v.push_back(q);
                                             return v;
                                         }()) {
                    if (k < 1) continue;
                    near_kernel_ = kind;
                    set_near_grid(k);
                    const float t = timed(product);
                    if (t < bt) { bt = t; bk = k; bkind = kind; }
                }
            near_kernel_ = bkind;
            near_per_sm_ = bk;
            set_near_grid(bk);
        }
        r.near_blocks_per_sm = near_per_sm_;
        // product schedule: translation kernel (list staged or not), near field
        // early or after S2M, one or two side streams for the finer translations
        {
            float bt = 1e30f;
            int bst = m2l_staged_, bnl = near_late_ ? 1 : 0, bms = m2l_streams_, bpdl = chain_pdl_ ? 1 : 0;
            for (int st : {0, 1})
                for (int nl : {0, 1})
                    for (int ms : {1, 2})
                        for (int pd : {0, 1}) {
                            m2l_staged_ = st;
                            near_late_ = nl != 0;
                            m2l_streams_ = ms;
                            chain_pdl_ = pd != 0;
                            const float t = timed(product);
                            if (t < bt) { bt = t; bst = st; bnl = nl; bms = ms; bpdl = pd; }
                        }
            m2l_staged_ = bst;
            near_late_ = bnl != 0;
            m2l_streams_ = bms;
            chain_pdl_ = bpdl != 0;
            r.schedule = bst | (bnl << 1) | ((bms - 1) << 2) | (bpdl << 3);
        }
        // interpolation and anterpolation: tensor cores or CUDA cores (the
        // complex-float far field), timed on the whole product
        if (tc_ok_ && precision_ != kFp64)
            for (int bit : {1, 4}) {  // M2M, then L2L: each stage on the faster kernels
                const int st = bit == 1 ? 1 : 3;
                tc_mode_ &= ~bit;
                const float t_cc = timed([&] { run_far(xt_, s, st, precision_, false); });
                tc_mode_ |= bit;
                const float t_tc = timed([&] { run_far(xt_, s, st, precision_, false); });
                if (!(t_tc < t_cc)) tc_mode_ &= ~bit;
            }
        r.after_ms = timed(product);
    } else {
        auto product = [&] { enqueue_multi(nr, s, precision_); };
        r.before_ms = timed(product);
        float bt = 1e30f;
        int border = m_m2m_rows_fast_;
        for (int o : {0, 1}) {
            m_m2m_rows_fast_ = o;
            const float t = timed([&] { run_far_multi(nr, s, 1, precision_); });
            if (t < bt) { bt = t; border = o; }
        }
        m_m2m_rows_fast_ = border;
        bt = 1e30f;
        int bpairs = m_l2l_pairs_;
        for (int q : {1, 2}) {
            bool fits = true;
            for (int p = lmin_; p < lmax_; ++p)
                if (static_cast<size_t>(nth_[p]) * 2 * q * 64 * csize + static_cast<size_t>(nth_[p + 1]) * dn_w_[p] * 16 + 1024 >
                    static_cast<size_t>(dev_smem))
                    fits = false;
            if (!fits) continue;
            m_l2l_pairs_ = q;
            const float t = timed([&] { run_far_multi(nr, s, 3, precision_); });
            if (t < bt) { bt = t; bpairs = q; }
        }
        m_l2l_pairs_ = bpairs;
        r.multi_rows_fast = border;
        r.multi_l2l_pairs = bpairs;
        if (tc_ok_ && precision_ != kFp64)
            for (int bit : {2, 8}) {
                const int st = bit == 2 ? 1 : 3;
                tc_mode_ &= ~bit;
                const float t_cc = timed([&] { run_far_multi(nr, s, st, precision_); });
                tc_mode_ |= bit;
                const float t_tc = timed([&] { run_far_multi(nr, s, st, precision_); });
                if (!(t_tc < t_cc)) tc_mode_ &= ~bit;
            }
        r.after_ms = timed(product);
    }
    r.interp_path = tc_mode();
    r.near_kernel = near_kernel_;
    r.m2l_chunk = m2l_chunk_;
    r.m2m_staged = r.l2l_staged = 0;
    for (int p = lmin_; p < lmax_ && p < 10; ++p) {
        if (m2m_pref_[p]) r.m2m_staged |= 1 << (m2m_pref_[p] == 2 ? 16 + p : p);
        if (l2l_pref_[p]) r.l2l_staged |= 1 << (l2l_pref_[p] == 3 ? 24 + p : l2l_pref_[p] == 2 ? 16 + p : p);
    }
    for (int p = lmin_; p < lmax_; ++p) r.m2m_rows[p] = m2m_rows_[p];
    if (r.multi_rows_fast == 0 && m_m2m_rows_fast_ < 0) r.multi_rows_fast = -1;
    // restore the local patterns, drop captured graphs
    for (size_t i = 0; i < saved.size(); ++i)
        MLFMA_CK(cudaMemcpyAsync(saved[i].first, tmp[i], saved[i].second, cudaMemcpyDeviceToDevice, s));
    MLFMA_CK(cudaStreamSynchronize(s));
    for (void* t : tmp) cudaFree(t);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    drop_graphs();
    ++generation_;
    if (rep) *rep = r;
    MLFMA_CK(cudaGetLastError());
    return {};
}

}  // namespace mlfma
