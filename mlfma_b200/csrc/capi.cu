// C ABI of the operator (include/mlfma_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <complex>
#include <cmath>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include "../../include/mlfma_b200.h"
#include "device.cuh"
#include "gmres.hpp"
#include "plan.hpp"

struct mlfma_op_s {
    mlfma::Plan plan;
    int device = 0;
    int precision = 0;
    std::unique_ptr<mlfma::DeviceOp> dev;
    std::unique_ptr<mlfma::Gmres> gmres;
    std::unique_ptr<mlfma::Gmres> gmres_fixed;  // runs on the library's fixed workspace
    std::unique_ptr<mlfma::GmresMulti> gmres_multi;
    int max_rhs = 1;
    double2* d_xm = nullptr;  // staging for host-buffer calls on many right-hand sides
    double2* d_ym = nullptr;
    double2* d_x = nullptr;  // staging for host-buffer calls
    double2* d_y = nullptr;
    void* d_stage = nullptr;  // small per-call inputs and outputs (directions, rows, far fields); grows only
    size_t stage_bytes = 0;
    mlfma_op_s* inner = nullptr;        // operator of the flexible solve's inner iterations
    std::vector<mlfma_op_s*> outers;    // operators that use this one as their inner operator
    ~mlfma_op_s() {
        if (d_x || d_y || d_xm || d_ym || d_stage) {
            cudaSetDevice(device);
            if (d_x) cudaFree(d_x);
            if (d_y) cudaFree(d_y);
            if (d_xm) cudaFree(d_xm);
            if (d_ym) cudaFree(d_ym);
            if (d_stage) cudaFree(d_stage);
        }
    }
};

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

int from_msg(const std::string& msg) {
    if (msg.empty()) return MLFMA_OK;
    if (msg.rfind("nonfinite", 0) == 0) return fail(MLFMA_ERR_NONFINITE, msg);
    if (msg.rfind("arg:", 0) == 0) return fail(MLFMA_ERR_ARG, msg);
    return fail(MLFMA_ERR_CUDA, msg);
}

// The handle's staging buffer, at least `bytes` long: reallocated (after the
// handle's stream has drained) only when a call needs more than any before.
int ensure_stage(mlfma_handle h, size_t bytes) {
    if (bytes <= h->stage_bytes) return MLFMA_OK;
    bytes = std::max<size_t>(bytes, 2 * h->stage_bytes);
    if (h->d_stage) {
        cudaStreamSynchronize(h->dev->stream());
        cudaFree(h->d_stage);
        h->d_stage = nullptr;
        h->stage_bytes = 0;
    }
    if (cudaMalloc(&h->d_stage, bytes) != cudaSuccess) return fail(MLFMA_ERR_CUDA, "cudaMalloc failed");
    h->stage_bytes = bytes;
    return MLFMA_OK;
}

mlfma::Config to_cfg(const mlfma_config* c) {
    mlfma::Config o;
    o.quad_prec = c->quad_prec;
    o.digits = c->digits;
    o.interp_order = c->interp_order;
    o.over_interp = c->over_interp;
    o.root_leng = c->root_leng;
    o.max_node_srcs = c->max_node_srcs;
    o.max_level = c->max_level;
    o.ref_compat = c->ref_compat;
    o.self_terms = c->self_terms;
    o.device_tree = c->device_tree;
    return o;
}

mlfma::PlaneWave to_pw(const mlfma_planewave* p) {
    mlfma::PlaneWave o;
    o.amplitude = p->amplitude;
    for (int k = 0; k < 3; ++k) {
        o.pol[k] = p->pol[k];
        o.khat[k] = p->khat[k];
    }
    o.wavenum = p->wavenum;
    return o;
}

bool ready(mlfma_handle h) { return h && h->dev; }

}  // namespace

// Used by batch.cu.
mlfma::DeviceOp* mlfma_internal_device(mlfma_handle h) { return h ? h->dev.get() : nullptr; }
int mlfma_internal_fail(int code, const std::string& msg) { return fail(code, msg); }
int mlfma_internal_device_ordinal(mlfma_handle h) { return h ? h->device : -1; }

extern "C" {

const char* mlfma_last_error(void) { return g_err.c_str(); }

int mlfma_config_default(mlfma_config* cfg) {
    if (!cfg) return fail(MLFMA_ERR_ARG, "null config");
    cfg->quad_prec = MLFMA_QUAD_7PT;
    cfg->digits = 3;
    cfg->interp_order = 3;
    cfg->over_interp = 2.0;
    cfg->root_leng = 4.0;
    cfg->max_node_srcs = 64;
    cfg->max_level = 0;
    cfg->ref_compat = 1;
    cfg->device = 0;
    cfg->precision = MLFMA_FP64;
    cfg->self_terms = 0;
    cfg->max_rhs = 1;
    cfg->device_tree = 0;
    return MLFMA_OK;
}

int mlfma_create_dipoles(const mlfma_config* cfg, const mlfma_planewave* pw, int n, const double* pos,
                         const double* mom, mlfma_handle* out) {
    if (!cfg || !pw || !pos || !mom || !out || n <= 0) return fail(MLFMA_ERR_ARG, "null argument or n <= 0");
    try {
        auto h = std::make_unique<mlfma_op_s>();
        h->device = cfg->device;
        h->precision = cfg->precision;
        h->max_rhs = cfg->max_rhs < 1 ? 1 : cfg->max_rhs;
        if (h->max_rhs > 64) return fail(MLFMA_ERR_ARG, "max_rhs must be at most 64");
        if (cfg->device_tree && cudaSetDevice(cfg->device) != cudaSuccess)
            return fail(MLFMA_ERR_CUDA, "cudaSetDevice failed");
        const std::string e = h->plan.build_dipoles(to_cfg(cfg), to_pw(pw), n, pos, mom);
        if (!e.empty()) return fail(MLFMA_ERR_ARG, e);
        *out = h.release();
        return MLFMA_OK;
    } catch (const std::exception& e) {
        return fail(MLFMA_ERR_INTERNAL, e.what());
    }
}

int mlfma_create_rwg(const mlfma_config* cfg, const mlfma_planewave* pw, int nv, const double* verts, int nf,
                     const int* faces, int ne, const int* rwgs, mlfma_handle* out) {
    if (!cfg || !pw || !verts || !faces || !rwgs || !out) return fail(MLFMA_ERR_ARG, "null argument");
    try {
        auto h = std::make_unique<mlfma_op_s>();
        h->device = cfg->device;
        h->precision = cfg->precision;
        h->max_rhs = cfg->max_rhs < 1 ? 1 : cfg->max_rhs;
        if (h->max_rhs > 64) return fail(MLFMA_ERR_ARG, "max_rhs must be at most 64");
        if (cfg->device_tree && cudaSetDevice(cfg->device) != cudaSuccess)
            return fail(MLFMA_ERR_CUDA, "cudaSetDevice failed");
        const std::string e = h->plan.build_rwg(to_cfg(cfg), to_pw(pw), nv, verts, nf, faces, ne, rwgs);
        if (!e.empty()) return fail(MLFMA_ERR_ARG, e);
        *out = h.release();
        return MLFMA_OK;
    } catch (const std::exception& e) {
        return fail(MLFMA_ERR_INTERNAL, e.what());
    }
}

int mlfma_setup(mlfma_handle h) {
    if (!h) return fail(MLFMA_ERR_ARG, "null handle");
    if (h->dev) return fail(MLFMA_ERR_STATE, "already set up");
    try {
        auto dev = std::make_unique<mlfma::DeviceOp>();
        std::string e = dev->setup(h->plan, h->device, h->precision, h->max_rhs);
        if (!e.empty()) return fail(MLFMA_ERR_CUDA, e);
        if (cudaMalloc(&h->d_x, sizeof(double2) * h->plan.n) != cudaSuccess ||
            cudaMalloc(&h->d_y, sizeof(double2) * h->plan.n) != cudaSuccess)
            return fail(MLFMA_ERR_CUDA, "cudaMalloc failed");
        // The fixed workspace of mlfma_gmres_noalloc is created on this device
        // now (first use of its module), not inside a solve.
        e = mlfma::noalloc_workspace_prepare();
        if (!e.empty()) return fail(MLFMA_ERR_CUDA, e);
        h->dev = std::move(dev);
        h->gmres = std::make_unique<mlfma::Gmres>();
        return MLFMA_OK;
    } catch (const std::exception& e) {
        return fail(MLFMA_ERR_INTERNAL, e.what());
    }
}

int mlfma_num_unknowns(mlfma_handle h, int* n) {
    if (!h || !n) return fail(MLFMA_ERR_ARG, "null argument");
    *n = h->plan.n;
    return MLFMA_OK;
}

int mlfma_get_stats(mlfma_handle h, mlfma_stats* st) {
    if (!h || !st) return fail(MLFMA_ERR_ARG, "null argument");
    const mlfma::Plan& p = h->plan;
    std::memset(st, 0, sizeof(*st));
    st->num_nodes = static_cast<int>(p.nodes.size());
    st->num_leaves = static_cast<int>(p.leaves.size());
    st->max_level = p.max_level;
    st->num_levels_far = p.max_level >= p.lmin ? p.max_level - p.lmin + 1 : 0;
    st->list2 = p.n_list2;
    st->list4 = p.n_list4;
    st->near_pairs = p.n_near_pairs;
    st->near_entries = p.near_entries;
    st->pattern_elems = p.pat_elems;
    st->device_bytes = h->dev ? h->dev->bytes_allocated() : 0;
    st->launches_per_matvec = h->dev ? h->dev->launches_per_matvec() : 0;
    return MLFMA_OK;
}

int mlfma_rhs(mlfma_handle h, double* b) {
    if (!h || !b) return fail(MLFMA_ERR_ARG, "null argument");
    h->plan.rhs(reinterpret_cast<mlfma::cplx*>(b));
    return MLFMA_OK;
}

int mlfma_matvec(mlfma_handle h, const double* x, double* y, int accumulate) {
    if (!h || !x || !y) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    const size_t bytes = sizeof(double2) * h->plan.n;
    cudaStream_t s = h->dev->stream();
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(MLFMA_ERR_CUDA, "cudaSetDevice failed");
    if (cudaMemcpyAsync(h->d_x, x, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return fail(MLFMA_ERR_CUDA, "copy of x failed");
    if (accumulate && cudaMemcpyAsync(h->d_y, y, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return fail(MLFMA_ERR_CUDA, "copy of y failed");
    std::string e = h->dev->matvec_device(h->d_x, h->d_y, accumulate != 0, s);
    if (!e.empty()) return fail(MLFMA_ERR_CUDA, e);
    if (cudaMemcpyAsync(y, h->d_y, bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return fail(MLFMA_ERR_CUDA, "copy of y failed");
    const cudaError_t ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return fail(MLFMA_ERR_CUDA, cudaGetErrorString(ce));
    e = h->dev->device_error();
    if (!e.empty()) return fail(MLFMA_ERR_CUDA, e);
    return MLFMA_OK;
}

namespace {
// Device address of the page-locked, mapped host range [p, p + bytes), or null
// when its first or last byte is not in such memory.
void* mapped_range(const void* p, size_t bytes) {
    cudaPointerAttributes a{}, b{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    const char* last = static_cast<const char*>(p) + bytes - 1;
    if (cudaPointerGetAttributes(&b, last) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a.type != cudaMemoryTypeHost || b.type != cudaMemoryTypeHost || !a.devicePointer || !b.devicePointer)
        return nullptr;
    if (static_cast<const char*>(b.devicePointer) != static_cast<const char*>(a.devicePointer) + (bytes - 1))
        return nullptr;
    return a.devicePointer;
}
}  // namespace

int mlfma_matvec_mapped(mlfma_handle h, const double* x, double* y, int accumulate) {
    if (!h || !x || !y) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(MLFMA_ERR_CUDA, "cudaSetDevice failed");
    const size_t bytes = sizeof(double2) * h->plan.n;
    void* dx = mapped_range(x, bytes);
    void* dy = mapped_range(y, bytes);
    if (!dx || !dy) return fail(MLFMA_ERR_ARG, "x and y must be page-locked host memory mapped for the device");
    cudaStream_t s = h->dev->stream();
    std::string e = h->dev->matvec_mapped(static_cast<const double2*>(dx), static_cast<double2*>(dy), accumulate != 0, s);
    if (!e.empty()) return fail(MLFMA_ERR_CUDA, e);
    const cudaError_t ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return fail(MLFMA_ERR_CUDA, cudaGetErrorString(ce));
    e = h->dev->device_error();
    if (!e.empty()) return fail(MLFMA_ERR_CUDA, e);
    return MLFMA_OK;
}

int mlfma_matvec_device(mlfma_handle h, const void* d_x, void* d_y, int accumulate, void* stream) {
    if (!h || !d_x || !d_y) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    std::string e = h->dev->matvec_device(static_cast<const double2*>(d_x), static_cast<double2*>(d_y),
                                          accumulate != 0, static_cast<cudaStream_t>(stream));
    if (!e.empty()) return fail(MLFMA_ERR_CUDA, e);
    return MLFMA_OK;
}

int mlfma_gmres(mlfma_handle h, const double* b, double* x, const mlfma_solver_opts* opts,
                mlfma_solve_info* info) {
    if (!h || !b || !x) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    mlfma::SolveOpts o;
    if (opts) {
        o.max_iter = opts->max_iter;
        o.tol = opts->tol;
        o.restart = opts->restart;
        o.ref_givens = opts->ref_givens;
        o.refine = opts->refine;
        o.inner_tol = opts->inner_tol;
        o.flexible = opts->flexible;
        o.inner_iters = opts->inner_iters;
        o.precond = opts->precond;
    }
    if (o.flexible && h->inner) o.inner = h->inner->dev.get();
    const size_t bytes = sizeof(double2) * h->plan.n;
    cudaStream_t s = h->dev->stream();
    cudaSetDevice(h->device);
    if (cudaMemcpyAsync(h->d_x, b, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return fail(MLFMA_ERR_CUDA, "copy of b failed");
    mlfma::SolveResult r;
    std::string e = h->gmres->solve(*h->dev, h->d_x, h->d_y, o, &r);
    if (!e.empty()) return from_msg(e);
    if (cudaMemcpyAsync(x, h->d_y, bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return fail(MLFMA_ERR_CUDA, "copy of x failed");
    e = h->dev->device_error();
    if (e.empty() && o.inner) e = o.inner->device_error();
    if (!e.empty()) return fail(MLFMA_ERR_CUDA, e);
    if (info) {
        info->iterations = r.iterations;
        info->residual = r.residual;
        info->true_residual = r.true_residual;
        info->seconds = r.seconds;
        info->refinements = r.refinements;
    }
    if (!r.converged) return fail(MLFMA_ERR_NOT_CONVERGED, "iteration limit reached");
    return MLFMA_OK;
}

int mlfma_check_bounded_wait(int device, int* timed_out) {
    if (!timed_out) return fail(MLFMA_ERR_ARG, "null argument");
    if (cudaSetDevice(device) != cudaSuccess) return fail(MLFMA_ERR_CUDA, "cudaSetDevice failed");
    int* d = nullptr;
    if (cudaMalloc(&d, sizeof(int)) != cudaSuccess) return fail(MLFMA_ERR_CUDA, "cudaMalloc failed");
    cudaMemset(d, 0xff, sizeof(int));
    mlfma::launch_wait_runs_out(1ll << 24, d);  // about 8 ms
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(timed_out, d, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(MLFMA_ERR_CUDA, cudaGetErrorString(e));
    return MLFMA_OK;
}

int mlfma_dense_rows(mlfma_handle h, int nrows, const int* rows, const double* x, double* y) {
    if (!h || nrows < 0 || (nrows > 0 && (!rows || !x || !y))) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    if (nrows == 0) return MLFMA_OK;
    const int n = h->plan.n;
    std::vector<int> slot(n), tree(nrows);
    for (int t = 0; t < n; ++t) slot[h->plan.perm[t]] = t;
    for (int i = 0; i < nrows; ++i) {
        if (rows[i] < 0 || rows[i] >= n) return fail(MLFMA_ERR_ARG, "row index out of range");
        tree[i] = slot[rows[i]];
    }
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(MLFMA_ERR_CUDA, "cudaSetDevice failed");
    cudaStream_t s = h->dev->stream();
    const size_t yb = (sizeof(double2) * nrows + 255) & ~static_cast<size_t>(255);
    const int code = ensure_stage(h, yb + sizeof(int) * nrows);
    if (code != MLFMA_OK) return code;
    double2* d_y = static_cast<double2*>(h->d_stage);
    int* d_rows = reinterpret_cast<int*>(static_cast<char*>(h->d_stage) + yb);
    std::string e;
    if (cudaMemcpyAsync(d_rows, tree.data(), sizeof(int) * nrows, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(h->d_x, x, sizeof(double2) * n, cudaMemcpyHostToDevice, s) != cudaSuccess)
        e = "copy failed";
    if (e.empty()) e = h->dev->dense_rows(d_rows, nrows, h->d_x, d_y, s);
    if (e.empty() && (cudaMemcpyAsync(y, d_y, sizeof(double2) * nrows, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                      cudaStreamSynchronize(s) != cudaSuccess))
        e = "copy of y failed";
    if (!e.empty()) return fail(MLFMA_ERR_CUDA, e);
    return MLFMA_OK;
}

int mlfma_dense_block_device(mlfma_handle h, int nrows, const int* rows, void* d_out, long long ld) {
    if (!h || nrows < 0 || (nrows > 0 && (!rows || !d_out))) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    const int n = h->plan.n;
    if (ld < n) return fail(MLFMA_ERR_ARG, "ld must be at least n");
    if (nrows == 0) return MLFMA_OK;
    std::vector<int> slot(n), tree(nrows);
    for (int t = 0; t < n; ++t) slot[h->plan.perm[t]] = t;
    for (int i = 0; i < nrows; ++i) {
        if (rows[i] < 0 || rows[i] >= n) return fail(MLFMA_ERR_ARG, "row index out of range");
        tree[i] = slot[rows[i]];
    }
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(MLFMA_ERR_CUDA, "cudaSetDevice failed");
    cudaStream_t s = h->dev->stream();
    const int code = ensure_stage(h, sizeof(int) * nrows);
    if (code != MLFMA_OK) return code;
    int* d_rows = static_cast<int*>(h->d_stage);
    if (cudaMemcpyAsync(d_rows, tree.data(), sizeof(int) * nrows, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return fail(MLFMA_ERR_CUDA, "copy of rows failed");
    std::string e = h->dev->dense_block(d_rows, nrows, static_cast<double2*>(d_out), ld, s);
    if (!e.empty()) return fail(MLFMA_ERR_CUDA, e);
    const cudaError_t ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return fail(MLFMA_ERR_CUDA, cudaGetErrorString(ce));
    return MLFMA_OK;
}

int mlfma_farfield(mlfma_handle h, const double* x, int ndir, const double* khat, double* out) {
    if (!h || !x || (ndir > 0 && (!khat || !out)) || ndir < 0) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    if (ndir == 0) return MLFMA_OK;
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(MLFMA_ERR_CUDA, "cudaSetDevice failed");
    cudaStream_t s = h->dev->stream();
    const size_t ob = (sizeof(double2) * 3 * ndir + 255) & ~static_cast<size_t>(255);
    const int code = ensure_stage(h, ob + sizeof(double) * 3 * ndir);
    if (code != MLFMA_OK) return code;
    double2* d_o = static_cast<double2*>(h->d_stage);
    double* d_k = reinterpret_cast<double*>(static_cast<char*>(h->d_stage) + ob);
    std::string e;
    if (cudaMemcpyAsync(h->d_x, x, sizeof(double2) * h->plan.n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(d_k, khat, sizeof(double) * 3 * ndir, cudaMemcpyHostToDevice, s) != cudaSuccess)
        e = "copy failed";
    if (e.empty()) e = h->dev->farfield(h->d_x, ndir, d_k, d_o, s);
    if (e.empty() && (cudaMemcpyAsync(out, d_o, sizeof(double2) * 3 * ndir, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                      cudaStreamSynchronize(s) != cudaSuccess))
        e = "copy of the far field failed";
    if (!e.empty()) return fail(MLFMA_ERR_CUDA, e);
    return MLFMA_OK;
}

// For callers that cannot allocate device memory during a solve: the Krylov
// workspace is the library's fixed device array (gmres.cu), never cudaMalloc.
int mlfma_gmres_noalloc(mlfma_handle h, const void* d_b, void* d_x, const mlfma_solver_opts* opts,
                        mlfma_solve_info* info) {
    if (!h || !d_b || !d_x) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    mlfma::SolveOpts o;
    if (opts) {
        o.max_iter = opts->max_iter;
        o.tol = opts->tol;
        o.restart = opts->restart;
        o.ref_givens = opts->ref_givens;
        o.refine = opts->refine;
        o.inner_tol = opts->inner_tol;
        o.flexible = opts->flexible;
        o.inner_iters = opts->inner_iters;
        o.precond = opts->precond;
    }
    if (o.max_iter < 1 || o.restart < 0) return fail(MLFMA_ERR_ARG, "max_iter and restart must be positive");
    if (o.flexible || o.precond)
        return fail(MLFMA_ERR_ARG, "flexible and preconditioned solves need their own workspace (use mlfma_gmres)");
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(MLFMA_ERR_CUDA, "cudaSetDevice failed");
    if (!h->gmres_fixed) h->gmres_fixed = std::make_unique<mlfma::Gmres>();
    const int m = o.restart > 0 ? o.restart : o.max_iter;
    std::string e = h->gmres_fixed->use_static_workspace(
        h->plan.n, m + 1, (o.refine && h->precision != MLFMA_FP64) ? 2 : 0);
    if (!e.empty()) return e.rfind("size:", 0) == 0 ? fail(MLFMA_ERR_ARG, e.substr(5)) : fail(MLFMA_ERR_CUDA, e);
    mlfma::SolveResult r;
    e = h->gmres_fixed->solve(*h->dev, static_cast<const double2*>(d_b), static_cast<double2*>(d_x), o, &r);
    if (!e.empty()) return from_msg(e);
    // a kernel that gave up a bounded wait leaves x invalid (as in mlfma_gmres)
    e = h->dev->device_error();
    if (!e.empty()) return fail(MLFMA_ERR_CUDA, e);
    if (info) {
        info->iterations = r.iterations;
        info->residual = r.residual;
        info->true_residual = r.true_residual;
        info->seconds = r.seconds;
        info->refinements = r.refinements;
    }
    if (!r.converged) return fail(MLFMA_ERR_NOT_CONVERGED, "iteration limit reached");
    return MLFMA_OK;
}

int mlfma_rhs_planewave(mlfma_handle h, const mlfma_planewave* pw, double* b) {
    if (!h || !pw || !b) return fail(MLFMA_ERR_ARG, "null argument");
    if (pw->wavenum != h->plan.pw.wavenum) return fail(MLFMA_ERR_ARG, "wavenumber differs from the operator's");
    h->plan.rhs_for(to_pw(pw), reinterpret_cast<mlfma::cplx*>(b));
    return MLFMA_OK;
}

int mlfma_matvec_multi_device(mlfma_handle h, int nrhs, const void* d_x, void* d_y, int accumulate, void* stream) {
    if (!h || !d_x || !d_y) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    std::string e = h->dev->matvec_multi_device(static_cast<const double2*>(d_x), static_cast<double2*>(d_y), nrhs,
                                                accumulate != 0, static_cast<cudaStream_t>(stream));
    if (!e.empty()) return from_msg(e);
    return MLFMA_OK;
}

static int ensure_multi_staging(mlfma_handle h) {
    if (h->d_xm) return MLFMA_OK;
    const size_t bytes = sizeof(double2) * static_cast<size_t>(h->plan.n) * h->max_rhs;
    if (cudaMalloc(&h->d_xm, bytes) != cudaSuccess || cudaMalloc(&h->d_ym, bytes) != cudaSuccess)
        return fail(MLFMA_ERR_CUDA, "cudaMalloc failed");
    return MLFMA_OK;
}

int mlfma_matvec_multi(mlfma_handle h, int nrhs, const double* x, double* y, int accumulate) {
    if (!h || !x || !y) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    if (nrhs < 1 || nrhs > h->max_rhs) return fail(MLFMA_ERR_ARG, "nrhs must be between 1 and max_rhs");
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(MLFMA_ERR_CUDA, "cudaSetDevice failed");
    int code = ensure_multi_staging(h);
    if (code != MLFMA_OK) return code;
    const size_t bytes = sizeof(double2) * static_cast<size_t>(h->plan.n) * nrhs;
    cudaStream_t s = h->dev->stream();
    if (cudaMemcpyAsync(h->d_xm, x, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return fail(MLFMA_ERR_CUDA, "copy of x failed");
    if (accumulate && cudaMemcpyAsync(h->d_ym, y, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return fail(MLFMA_ERR_CUDA, "copy of y failed");
    std::string e = h->dev->matvec_multi_device(h->d_xm, h->d_ym, nrhs, accumulate != 0, s);
    if (!e.empty()) return from_msg(e);
    if (cudaMemcpyAsync(y, h->d_ym, bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return fail(MLFMA_ERR_CUDA, "copy of y failed");
    const cudaError_t ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return fail(MLFMA_ERR_CUDA, cudaGetErrorString(ce));
    return MLFMA_OK;
}

int mlfma_gmres_multi(mlfma_handle h, int nrhs, const double* b, double* x, const mlfma_solver_opts* opts,
                      mlfma_solve_info* info) {
    if (!h || !b || !x) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    if (nrhs < 1 || nrhs > h->max_rhs) return fail(MLFMA_ERR_ARG, "nrhs must be between 1 and max_rhs");
    mlfma::SolveOpts o;
    if (opts) {
        o.max_iter = opts->max_iter;
        o.tol = opts->tol;
        o.restart = opts->restart;
        o.ref_givens = opts->ref_givens;
        o.refine = opts->refine;
        o.inner_tol = opts->inner_tol;
        o.flexible = opts->flexible;
        o.inner_iters = opts->inner_iters;
        o.precond = opts->precond;
    }
    if (o.precond)
        return fail(MLFMA_ERR_ARG, "preconditioned GMRES runs one right-hand side at a time (mlfma_gmres)");
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(MLFMA_ERR_CUDA, "cudaSetDevice failed");
    int code = ensure_multi_staging(h);
    if (code != MLFMA_OK) return code;
    if (!h->gmres_multi) h->gmres_multi = std::make_unique<mlfma::GmresMulti>();
    const size_t bytes = sizeof(double2) * static_cast<size_t>(h->plan.n) * nrhs;
    cudaStream_t s = h->dev->stream();
    if (cudaMemcpyAsync(h->d_xm, b, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return fail(MLFMA_ERR_CUDA, "copy of b failed");
    std::vector<mlfma::SolveResult> r;
    std::string e = h->gmres_multi->solve(*h->dev, nrhs, h->d_xm, h->d_ym, o, r);
    if (!e.empty()) return from_msg(e);
    if (cudaMemcpyAsync(x, h->d_ym, bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return fail(MLFMA_ERR_CUDA, "copy of x failed");
    bool all = true;
    for (int i = 0; i < nrhs; ++i) {
        if (info) {
            info[i].iterations = r[i].iterations;
            info[i].residual = r[i].residual;
            info[i].true_residual = r[i].true_residual;
            info[i].seconds = r[i].seconds;
            info[i].refinements = r[i].refinements;
        }
        all = all && r[i].converged;
    }
    if (!all) return fail(MLFMA_ERR_NOT_CONVERGED, "iteration limit reached for some right-hand side");
    return MLFMA_OK;
}

int mlfma_time_stages_multi(mlfma_handle h, int nrhs, mlfma_stage_times* t) {
    if (!h || !t) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    mlfma::StageTimes st{};
    std::string e = h->dev->time_stages_multi(nrhs, &st);
    if (!e.empty()) return from_msg(e);
    t->gather = st.gather;
    t->s2m = st.s2m;
    t->m2m = st.m2m;
    t->m2l = st.m2l;
    t->l2l = st.l2l;
    t->l2t = st.l2t;
    t->near_field = st.near;
    t->finish = st.finish;
    t->total = st.total;
    return MLFMA_OK;
}

// ---------------------------------------------------------------- adjoint
// No counterpart in the reference: loads, the adjoint product and solve, and
// the far-field power gradient built on them.

int mlfma_set_loads(mlfma_handle h, const double* z) {
    if (!h) return fail(MLFMA_ERR_ARG, "null handle");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    if (z)
        for (int i = 0; i < 2 * h->plan.n; ++i)
            if (!std::isfinite(z[i])) return fail(MLFMA_ERR_NONFINITE, "nonfinite load");
    std::string e = h->dev->set_loads(reinterpret_cast<const double2*>(z));
    if (!e.empty()) return from_msg(e);
    return MLFMA_OK;
}

int mlfma_matvec_adjoint(mlfma_handle h, const double* x, double* y, int accumulate) {
    if (!h || !x || !y) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    const size_t bytes = sizeof(double2) * h->plan.n;
    cudaStream_t s = h->dev->stream();
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(MLFMA_ERR_CUDA, "cudaSetDevice failed");
    if (cudaMemcpyAsync(h->d_x, x, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return fail(MLFMA_ERR_CUDA, "copy of x failed");
    if (accumulate && cudaMemcpyAsync(h->d_y, y, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return fail(MLFMA_ERR_CUDA, "copy of y failed");
    std::string e = h->dev->matvec_device(h->d_x, h->d_y, accumulate != 0, s, -1, true);
    if (!e.empty()) return from_msg(e);
    if (cudaMemcpyAsync(y, h->d_y, bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return fail(MLFMA_ERR_CUDA, "copy of y failed");
    const cudaError_t ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return fail(MLFMA_ERR_CUDA, cudaGetErrorString(ce));
    return MLFMA_OK;
}

static mlfma::SolveOpts to_opts(const mlfma_solver_opts* opts) {
    mlfma::SolveOpts o;
    if (opts) {
        o.max_iter = opts->max_iter;
        o.tol = opts->tol;
        o.restart = opts->restart;
        o.ref_givens = opts->ref_givens;
        o.refine = opts->refine;
        o.inner_tol = opts->inner_tol;
        o.flexible = opts->flexible;
        o.inner_iters = opts->inner_iters;
        o.precond = opts->precond;
    }
    return o;
}

static void to_info(const mlfma::SolveResult& r, mlfma_solve_info* info) {
    if (!info) return;
    info->iterations = r.iterations;
    info->residual = r.residual;
    info->true_residual = r.true_residual;
    info->seconds = r.seconds;
    info->refinements = r.refinements;
}

// Host b -> host x through the handle's GMRES (adjoint when adj).
static int solve_host(mlfma_handle h, const double* b, double* x, mlfma::SolveOpts o, bool adj,
                      mlfma_solve_info* info) {
    o.adjoint = adj ? 1 : 0;
    if (adj) o.ref_givens = 0;
    const size_t bytes = sizeof(double2) * h->plan.n;
    cudaStream_t s = h->dev->stream();
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(MLFMA_ERR_CUDA, "cudaSetDevice failed");
    if (cudaMemcpyAsync(h->d_x, b, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return fail(MLFMA_ERR_CUDA, "copy of b failed");
    mlfma::SolveResult r;
    std::string e = h->gmres->solve(*h->dev, h->d_x, h->d_y, o, &r);
    if (!e.empty()) return from_msg(e);
    if (cudaMemcpyAsync(x, h->d_y, bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return fail(MLFMA_ERR_CUDA, "copy of x failed");
    e = h->dev->device_error();
    if (!e.empty()) return fail(MLFMA_ERR_CUDA, e);
    to_info(r, info);
    if (!r.converged) return fail(MLFMA_ERR_NOT_CONVERGED, "iteration limit reached");
    return MLFMA_OK;
}

int mlfma_gmres_adjoint(mlfma_handle h, const double* b, double* x, const mlfma_solver_opts* opts,
                        mlfma_solve_info* info) {
    if (!h || !b || !x) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    return solve_host(h, b, x, to_opts(opts), true, info);
}

int mlfma_farfield_adjoint(mlfma_handle h, int ndir, const double* khat, const double* F, double* g) {
    if (!h || ndir < 0 || (ndir > 0 && (!khat || !F)) || !g) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(MLFMA_ERR_CUDA, "cudaSetDevice failed");
    cudaStream_t s = h->dev->stream();
    const int nd = ndir > 0 ? ndir : 1;
    // F, its projection (k_project), the directions
    const size_t fb = (sizeof(double2) * 3 * nd + 255) & ~static_cast<size_t>(255);
    const int code = ensure_stage(h, 2 * fb + sizeof(double) * 3 * nd);
    if (code != MLFMA_OK) return code;
    double2* d_F = static_cast<double2*>(h->d_stage);
    double2* d_P = reinterpret_cast<double2*>(static_cast<char*>(h->d_stage) + fb);
    double* d_k = reinterpret_cast<double*>(static_cast<char*>(h->d_stage) + 2 * fb);
    std::string e;
    if (ndir > 0 && (cudaMemcpyAsync(d_k, khat, sizeof(double) * 3 * ndir, cudaMemcpyHostToDevice, s) != cudaSuccess ||
                     cudaMemcpyAsync(d_F, F, sizeof(double2) * 3 * ndir, cudaMemcpyHostToDevice, s) != cudaSuccess))
        e = "copy failed";
    if (e.empty()) e = h->dev->farfield_adjoint(d_F, ndir, d_k, h->d_y, s, d_P);
    if (e.empty() && (cudaMemcpyAsync(g, h->d_y, sizeof(double2) * h->plan.n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                      cudaStreamSynchronize(s) != cudaSuccess))
        e = "copy of g failed";
    if (!e.empty()) return fail(MLFMA_ERR_CUDA, e);
    return MLFMA_OK;
}

int mlfma_vjp_farfield_power(mlfma_handle h, int nexc, const mlfma_planewave* pws, const double* w, int ndir,
                             const double* khat, const mlfma_solver_opts* opts, double* J, double* grad_loads,
                             double* grad_w, double* currents, mlfma_solve_info* info) {
    if (!h || nexc < 1 || !pws || !w || ndir < 1 || !khat || !J) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    if (h->dev->ref_compat()) return fail(MLFMA_ERR_ARG, "the adjoint needs ref_compat = 0");
    using cd = std::complex<double>;
    const int n = h->plan.n;
    try {
        // b = sum_j w_j b_j
        std::vector<std::vector<cd>> bj(nexc, std::vector<cd>(n));
        std::vector<cd> b(n, cd(0));
        for (int j = 0; j < nexc; ++j) {
            if (pws[j].wavenum != h->plan.pw.wavenum) return fail(MLFMA_ERR_ARG, "wavenumber differs from the operator's");
            h->plan.rhs_for(to_pw(&pws[j]), bj[j].data());
            const cd wj(w[2 * j], w[2 * j + 1]);
            for (int i = 0; i < n; ++i) b[i] += wj * bj[j][i];
        }
        const mlfma::SolveOpts o = to_opts(opts);
        // forward solve A I = b
        std::vector<cd> I(n);
        int code = solve_host(h, reinterpret_cast<const double*>(b.data()), reinterpret_cast<double*>(I.data()), o,
                              false, info);
        if (code != MLFMA_OK) return code;
        // F = M I, J = |F|^2
        std::vector<cd> F(3 * static_cast<size_t>(ndir));
        code = mlfma_farfield(h, reinterpret_cast<const double*>(I.data()), ndir, khat, reinterpret_cast<double*>(F.data()));
        if (code != MLFMA_OK) return code;
        double Jv = 0;
        for (const cd& f : F) Jv += std::norm(f);
        *J = Jv;
        // g = M^H F ; adjoint solve A^H lambda = g
        std::vector<cd> g(n), lam(n);
        code = mlfma_farfield_adjoint(h, ndir, khat, reinterpret_cast<const double*>(F.data()),
                                      reinterpret_cast<double*>(g.data()));
        if (code != MLFMA_OK) return code;
        code = solve_host(h, reinterpret_cast<const double*>(g.data()), reinterpret_cast<double*>(lam.data()), o, true,
                          info ? info + 1 : nullptr);
        if (code != MLFMA_OK) return code;
        // dJ = 2 Re(lambda^H (db - dZ I)):  dJ/dRe z + i dJ/dIm z = -2 lambda conj(I);
        // dJ/dRe w_j + i dJ/dIm w_j = 2 conj(lambda^H b_j)
        if (grad_loads)
            for (int i = 0; i < n; ++i) {
                const cd v = -2.0 * lam[i] * std::conj(I[i]);
                grad_loads[2 * i] = v.real();
                grad_loads[2 * i + 1] = v.imag();
            }
        if (grad_w)
            for (int j = 0; j < nexc; ++j) {
                cd d(0);
                for (int i = 0; i < n; ++i) d += std::conj(lam[i]) * bj[j][i];
                const cd v = 2.0 * std::conj(d);
                grad_w[2 * j] = v.real();
                grad_w[2 * j + 1] = v.imag();
            }
        if (currents) std::memcpy(currents, I.data(), sizeof(cd) * n);
    } catch (const std::exception& e) {
        return fail(MLFMA_ERR_INTERNAL, e.what());
    }
    return MLFMA_OK;
}

int mlfma_autotune(mlfma_handle h, int nrhs, int reps, mlfma_tuning* out) {
    if (!h) return fail(MLFMA_ERR_ARG, "null handle");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    mlfma::TuneReport r{};
    std::string e = h->dev->autotune(nrhs, reps, &r);
    if (!e.empty()) return from_msg(e);
    if (out) {
        std::memset(out, 0, sizeof(*out));
        out->m2l_chunk = r.m2l_chunk;
        for (int i = 0; i < 20 && i < mlfma::kMaxLevels; ++i) out->m2m_rows[i] = r.m2m_rows[i];
        out->multi_m2m_rows_fast = r.multi_rows_fast;
        out->multi_l2l_pairs = r.multi_l2l_pairs;
        out->product_ms_before = r.before_ms;
        out->product_ms_after = r.after_ms;
        out->near_blocks_per_sm = r.near_blocks_per_sm;
        out->interp_path = r.interp_path;
        out->schedule = r.schedule;
        out->m2m_staged = r.m2m_staged;
        out->l2l_staged = r.l2l_staged;
        out->near_kernel = r.near_kernel;
    }
    return MLFMA_OK;
}

int mlfma_set_interp_path(mlfma_handle h, int mode) {
    if (!h) return fail(MLFMA_ERR_ARG, "null handle");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    return from_msg(h->dev->set_tc(mode));
}

int mlfma_set_near_kernel(mlfma_handle h, int kind) {
    if (!h) return fail(MLFMA_ERR_ARG, "null handle");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    return from_msg(h->dev->set_near_kernel(kind));
}

int mlfma_set_schedule(mlfma_handle h, int schedule) {
    if (!h) return fail(MLFMA_ERR_ARG, "null handle");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    return from_msg(h->dev->set_schedule(schedule));
}

int mlfma_set_staged_interp(mlfma_handle h, int mode) {
    if (!h) return fail(MLFMA_ERR_ARG, "null handle");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    return from_msg(h->dev->set_staged(mode));
}

int mlfma_get_interp_path(mlfma_handle h, int* mode) {
    if (!h || !mode) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    *mode = h->dev->tc_mode();
    return MLFMA_OK;
}

int mlfma_get_stream(mlfma_handle h, void** stream) {
    if (!h || !stream) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    *stream = static_cast<void*>(h->dev->stream());
    return MLFMA_OK;
}

int mlfma_time_stages(mlfma_handle h, mlfma_stage_times* t) {
    if (!h || !t) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    mlfma::StageTimes st{};
    std::string e = h->dev->time_stages(&st);
    if (!e.empty()) return fail(MLFMA_ERR_CUDA, e);
    t->gather = st.gather;
    t->s2m = st.s2m;
    t->m2m = st.m2m;
    t->m2l = st.m2l;
    t->l2l = st.l2l;
    t->l2t = st.l2t;
    t->near_field = st.near;
    t->finish = st.finish;
    t->total = st.total;
    return MLFMA_OK;
}

int mlfma_time_levels(mlfma_handle h, int cap, float* ms, int* nlevels) {
    if (!h || !nlevels) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    *nlevels = h->plan.max_level + 1;
    if (!ms) return MLFMA_OK;
    if (cap < 3 * *nlevels) return fail(MLFMA_ERR_ARG, "buffer too small");
    std::vector<float> v;
    std::string e = h->dev->time_levels(v);
    if (!e.empty()) return fail(MLFMA_ERR_CUDA, e);
    std::copy(v.begin(), v.end(), ms);
    return MLFMA_OK;
}

int mlfma_get_traffic(mlfma_handle h, mlfma_traffic* t) {
    if (!h || !t) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    const auto tr = h->dev->traffic();
    t->s2m = tr.s2m;
    t->m2m = tr.m2m;
    t->m2l = tr.m2l;
    t->l2l = tr.l2l;
    t->l2t = tr.l2t;
    t->near_field = tr.near;
    t->total = tr.total;
    return MLFMA_OK;
}

int mlfma_level_info(mlfma_handle h, int level, int* sizes, double* thetas, double* weights, double* phis) {
    if (!h || !sizes) return fail(MLFMA_ERR_ARG, "null argument");
    const mlfma::Plan& p = h->plan;
    if (level < p.lmin || level > p.max_level) return fail(MLFMA_ERR_ARG, "level has no far field");
    const mlfma::Level& L = p.levels[level];
    sizes[0] = L.nth;
    sizes[1] = L.nph;
    sizes[2] = L.L;
    if (thetas) std::memcpy(thetas, L.thetas.data(), sizeof(double) * L.nth);
    if (weights) std::memcpy(weights, L.weights.data(), sizeof(double) * L.nth);
    if (phis) std::memcpy(phis, L.phis.data(), sizeof(double) * L.nph);
    return MLFMA_OK;
}

int mlfma_level_boxes(mlfma_handle h, int level, int* nbox, int* coords) {
    if (!h || !nbox) return fail(MLFMA_ERR_ARG, "null argument");
    const mlfma::Plan& p = h->plan;
    if (level < p.lmin || level > p.max_level) return fail(MLFMA_ERR_ARG, "level has no far field");
    const mlfma::Level& L = p.levels[level];
    *nbox = static_cast<int>(L.boxes.size());
    if (coords)
        for (size_t b = 0; b < L.boxes.size(); ++b) {
            const mlfma::Node& nd = p.nodes[L.boxes[b]];
            coords[3 * b] = nd.ix;
            coords[3 * b + 1] = nd.iy;
            coords[3 * b + 2] = nd.iz;
        }
    return MLFMA_OK;
}

int mlfma_level_patterns(mlfma_handle h, int level, int which, double* out, long long count) {
    if (!h || !out) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    std::string e = h->dev->copy_level(level, which, reinterpret_cast<double2*>(out), count);
    if (!e.empty()) return fail(MLFMA_ERR_ARG, e);
    return MLFMA_OK;
}

int mlfma_level_transl(mlfma_handle h, int level, double* out) {
    if (!h || !out) return fail(MLFMA_ERR_ARG, "null argument");
    const mlfma::Plan& p = h->plan;
    if (level < p.lmin || level > p.max_level) return fail(MLFMA_ERR_ARG, "level has no far field");
    const mlfma::Level& L = p.levels[level];
    std::memcpy(out, L.transl.data(), sizeof(double) * 2 * L.transl.size());
    return MLFMA_OK;
}

int mlfma_level_transl_gpu(mlfma_handle h, int level, double* out) {
    if (!h || !out) return fail(MLFMA_ERR_ARG, "null argument");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    const std::string e = h->dev->copy_transl(level, reinterpret_cast<double2*>(out));
    if (!e.empty()) return fail(e == "level out of range" ? MLFMA_ERR_ARG : MLFMA_ERR_CUDA, e);
    return MLFMA_OK;
}

int mlfma_far_leaves(mlfma_handle h, int* count, int* info, int* perm) {
    if (!h || !count) return fail(MLFMA_ERR_ARG, "null argument");
    const mlfma::Plan& p = h->plan;
    *count = static_cast<int>(p.far_leaves.size());
    if (info)
        for (size_t i = 0; i < p.far_leaves.size(); ++i) {
            const mlfma::FarLeaf& f = p.far_leaves[i];
            info[4 * i] = f.level;
            info[4 * i + 1] = f.box;
            info[4 * i + 2] = f.src0;
            info[4 * i + 3] = f.nsrc;
        }
    if (perm) std::memcpy(perm, p.perm.data(), sizeof(int) * p.perm.size());
    return MLFMA_OK;
}

int mlfma_tree_export(mlfma_handle h, int which, int* out, long long cap, long long* count) {
    if (!h || !count) return fail(MLFMA_ERR_ARG, "null argument");
    if (which < 0 || which > 5) return fail(MLFMA_ERR_ARG, "which must be 0..5");
    const mlfma::Plan& p = h->plan;
    std::vector<int> v;
    if (which == 1) {
        v = p.perm;
    } else {
        for (const mlfma::Node& nd : p.nodes) {
            if (which == 0) {
                v.insert(v.end(), {nd.level, nd.parent, nd.branch});
                v.insert(v.end(), nd.child, nd.child + 8);
                v.insert(v.end(), {nd.leaf ? 1 : 0, nd.src_begin, nd.src_count});
                continue;
            }
            const std::vector<int>& l = which == 2 ? nd.nbors : which == 3 ? nd.near_nbors
                                        : which == 4 ? nd.ilist : nd.leaf_ilist;
            v.push_back(static_cast<int>(l.size()));
            v.insert(v.end(), l.begin(), l.end());
        }
    }
    *count = static_cast<long long>(v.size());
    if (!out) return MLFMA_OK;
    if (cap < *count) return fail(MLFMA_ERR_ARG, "buffer too small");
    std::memcpy(out, v.data(), sizeof(int) * v.size());
    return MLFMA_OK;
}

int mlfma_rwg_patterns_host(mlfma_handle h, double* out, long long count) {
    if (!h || !out) return fail(MLFMA_ERR_ARG, "null argument");
    const mlfma::Plan& p = h->plan;
    if (p.kind != mlfma::kRwg) return fail(MLFMA_ERR_ARG, "not an RWG operator");
    if (count < p.pat_elems * 2) return fail(MLFMA_ERR_ARG, "buffer too small");
    try {
        std::vector<mlfma::cplx> pat;
        p.rwg_patterns_host(pat);
        std::memcpy(out, pat.data(), sizeof(mlfma::cplx) * pat.size());
    } catch (const std::exception& e) {
        return fail(MLFMA_ERR_INTERNAL, e.what());
    }
    return MLFMA_OK;
}

int mlfma_set_inner_operator(mlfma_handle h, mlfma_handle inner) {
    if (!h) return fail(MLFMA_ERR_ARG, "null handle");
    if (!ready(h)) return fail(MLFMA_ERR_STATE, "mlfma_setup has not run");
    if (inner == h) return fail(MLFMA_ERR_ARG, "an operator is not its own inner operator");
    if (inner) {
        if (!ready(inner)) return fail(MLFMA_ERR_STATE, "the inner operator is not set up");
        if (inner->device != h->device) return fail(MLFMA_ERR_ARG, "the inner operator is on another device");
        if (inner->plan.n != h->plan.n || inner->plan.perm != h->plan.perm)
            return fail(MLFMA_ERR_ARG, "the inner operator has other unknowns or another source order (build it "
                                       "from the same sources with the same root_leng, max_node_srcs, max_level)");
    }
    if (h->inner) {
        auto& o = h->inner->outers;
        o.erase(std::remove(o.begin(), o.end(), h), o.end());
    }
    h->inner = inner;
    if (inner) inner->outers.push_back(h);
    return MLFMA_OK;
}

int mlfma_destroy(mlfma_handle h) {
    if (h) {
        if (h->inner) {
            auto& o = h->inner->outers;
            o.erase(std::remove(o.begin(), o.end(), h), o.end());
        }
        for (mlfma_op_s* o : h->outers) o->inner = nullptr;
    }
    delete h;
    return MLFMA_OK;
}

}  // extern "C"
