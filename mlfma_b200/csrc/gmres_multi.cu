// GMRES on many right-hand sides at once (Solver::solve, src/solver.cpp:5-146,
// run for nr independent systems A x_r = b_r that share every product).
//
// Each column has its own Krylov basis, Hessenberg matrix and Givens
// rotations; the columns share the operator launches (one product on nr
// vectors per Arnoldi step), the orthogonalisation launches (CGS2, batched over
// columns) and one host synchronisation per step.  A column that has met its
// tolerance is frozen: its next basis vector is zero, so it costs nothing but
// its share of the batched launches.  Vectors are tree-ordered with the
// right-hand side innermost ([n][nr]), the layout of the many-rhs product.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <string>
#include <vector>

#include "gmres.hpp"

namespace mlfma {

namespace {

constexpr int kThreads = 256;
constexpr int kRowsPerChunk = 2048;

inline int nblk(long long n, int bs) { return static_cast<int>((n + bs - 1) / bs); }

// partial[j][c][r] = sum_{i in chunk c} conj(Q_j[i][r]) w[i][r]
__global__ void k_mdot(const double2* __restrict__ Q, long long ld, const double2* __restrict__ w, int n, int nr,
                       double2* __restrict__ partial, int nchunks) {
    __shared__ double2 red[kThreads];
    const int c = blockIdx.x, j = blockIdx.y;
    const int r = threadIdx.x % kMaxRhs, sub = threadIdx.x / kMaxRhs;  // 4 rows at a time
    const double2* q = Q + static_cast<long long>(j) * ld;
    const int i0 = c * kRowsPerChunk, i1 = min(n, i0 + kRowsPerChunk);
    double2 acc = make_double2(0.0, 0.0);
    if (r < nr)
        for (int i = i0 + sub; i < i1; i += kThreads / kMaxRhs) {
            const double2 a = q[static_cast<long long>(i) * nr + r], b = w[static_cast<long long>(i) * nr + r];
            acc.x = fma(a.x, b.x, fma(a.y, b.y, acc.x));
            acc.y = fma(a.x, b.y, fma(-a.y, b.x, acc.y));
        }
    red[threadIdx.x] = acc;
    __syncthreads();
    if (sub == 0 && r < nr) {
        double2 s = red[r];
        for (int u = 1; u < kThreads / kMaxRhs; ++u) {
            s.x += red[u * kMaxRhs + r].x;
            s.y += red[u * kMaxRhs + r].y;
        }
        partial[(static_cast<long long>(j) * nchunks + c) * nr + r] = s;
    }
}

// h[j][r] (+)= sum_c partial[j][c][r]  (fixed order)
__global__ void k_mreduce(const double2* __restrict__ partial, int nchunks, int ncols, int nr, double2* __restrict__ h,
                          int add) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ncols * nr) return;
    const int j = t / nr, r = t - j * nr;
    double2 s = make_double2(0.0, 0.0);
    for (int c = 0; c < nchunks; ++c) {
        const double2 p = partial[(static_cast<long long>(j) * nchunks + c) * nr + r];
        s.x += p.x;
        s.y += p.y;
    }
    if (add) { h[t].x += s.x; h[t].y += s.y; } else { h[t] = s; }
}

// w[i][r] -= sum_j Q_j[i][r] h[j][r]
__global__ void k_msub_qh(const double2* __restrict__ Q, long long ld, int ncols, const double2* __restrict__ h,
                          double2* __restrict__ w, long long tot, int nr) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= tot) return;
    const int r = static_cast<int>(t % nr);
    double2 v = w[t];
    for (int j = 0; j < ncols; ++j) {
        const double2 q = Q[static_cast<long long>(j) * ld + t];
        const double2 hj = h[j * nr + r];
        v.x -= q.x * hj.x - q.y * hj.y;
        v.y -= q.x * hj.y + q.y * hj.x;
    }
    w[t] = v;
}

// partial[c][r] = sum_{i in chunk c} |w[i][r]|^2
__global__ void k_mnorm2(const double2* __restrict__ w, int n, int nr, double* __restrict__ partial) {
    __shared__ double red[kThreads];
    const int c = blockIdx.x;
    const int r = threadIdx.x % kMaxRhs, sub = threadIdx.x / kMaxRhs;
    const int i0 = c * kRowsPerChunk, i1 = min(n, i0 + kRowsPerChunk);
    double acc = 0.0;
    if (r < nr)
        for (int i = i0 + sub; i < i1; i += kThreads / kMaxRhs) {
            const double2 a = w[static_cast<long long>(i) * nr + r];
            acc = fma(a.x, a.x, fma(a.y, a.y, acc));
        }
    red[threadIdx.x] = acc;
    __syncthreads();
    if (sub == 0 && r < nr) {
        double s = red[r];
        for (int u = 1; u < kThreads / kMaxRhs; ++u) s += red[u * kMaxRhs + r];
        partial[static_cast<long long>(c) * nr + r] = s;
    }
}

// out[r].x = sum_c partial[c][r]
__global__ void k_msum(const double* __restrict__ partial, int nchunks, int nr, double2* __restrict__ out) {
    const int r = threadIdx.x;
    if (r >= nr) return;
    double s = 0.0;
    for (int c = 0; c < nchunks; ++c) s += partial[static_cast<long long>(c) * nr + r];
    out[r] = make_double2(s, 0.0);
}

// out[i][r] = x[i][r] * s[r]
__global__ void k_mscale(const double2* __restrict__ x, const double* __restrict__ s, double2* __restrict__ out,
                         long long tot, int nr) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= tot) return;
    const double f = s[t % nr];
    out[t] = make_double2(x[t].x * f, x[t].y * f);
}

__global__ void k_msub(const double2* __restrict__ b, const double2* __restrict__ y, double2* __restrict__ out,
                       long long tot) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < tot) out[t] = make_double2(b[t].x - y[t].x, b[t].y - y[t].y);
}

__global__ void k_maxpy(const double2* __restrict__ x, double2* __restrict__ y, long long tot) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < tot) y[t] = make_double2(y[t].x + x[t].x, y[t].y + x[t].y);
}

// xt[t][r] = x[r][perm[t]] and back
__global__ void k_mgather(const double2* __restrict__ x, const int* __restrict__ perm, double2* __restrict__ xt, int n,
                          int nr) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<long long>(n) * nr) return;
    const int t = static_cast<int>(i / nr), r = static_cast<int>(i - static_cast<long long>(t) * nr);
    xt[i] = x[static_cast<size_t>(r) * n + perm[t]];
}
__global__ void k_mscatter(const double2* __restrict__ xt, const int* __restrict__ perm, double2* __restrict__ x, int n,
                           int nr) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<long long>(n) * nr) return;
    const int t = static_cast<int>(i / nr), r = static_cast<int>(i - static_cast<long long>(t) * nr);
    x[static_cast<size_t>(r) * n + perm[t]] = xt[i];
}

}  // namespace

#define GMM_CK(call)                                                               \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) return std::string(#call) + ": " + cudaGetErrorString(e_); \
    } while (0)

GmresMulti::~GmresMulti() { release(); }

void GmresMulti::release() {
    for (void* p : {(void*)Q_, (void*)w_, (void*)b_, (void*)x_, (void*)r_, (void*)h_, (void*)y_, (void*)partial_,
                    (void*)npartial_, (void*)scale_, (void*)xo_, (void*)bo_})
        if (p) cudaFree(p);
    Q_ = w_ = b_ = x_ = r_ = h_ = y_ = partial_ = xo_ = bo_ = nullptr;
    npartial_ = scale_ = nullptr;
    for (void* p : {(void*)V_, (void*)Z_})
        if (p) cudaFree(p);
    V_ = Z_ = nullptr;
    n_ = nr_ = cap_ = vcap_ = 0;
}

std::string GmresMulti::ensure(int n, int nr, int ncols) {
    if (n == n_ && nr == nr_ && ncols <= cap_) return {};
    release();
    n_ = n;
    nr_ = nr;
    cap_ = ncols;
    nchunks_ = (n + kRowsPerChunk - 1) / kRowsPerChunk;
    const size_t v = static_cast<size_t>(n) * nr;
    GMM_CK(cudaMalloc(&Q_, sizeof(double2) * v * ncols));
    GMM_CK(cudaMalloc(&w_, sizeof(double2) * v));
    GMM_CK(cudaMalloc(&b_, sizeof(double2) * v));
    GMM_CK(cudaMalloc(&x_, sizeof(double2) * v));
    GMM_CK(cudaMalloc(&r_, sizeof(double2) * v));
    GMM_CK(cudaMalloc(&xo_, sizeof(double2) * v));
    GMM_CK(cudaMalloc(&bo_, sizeof(double2) * v));
    GMM_CK(cudaMalloc(&h_, sizeof(double2) * static_cast<size_t>(ncols + 1) * nr));
    GMM_CK(cudaMalloc(&y_, sizeof(double2) * static_cast<size_t>(ncols + 1) * nr));
    GMM_CK(cudaMalloc(&partial_, sizeof(double2) * static_cast<size_t>(nchunks_) * (ncols + 1) * nr));
    GMM_CK(cudaMalloc(&npartial_, sizeof(double) * static_cast<size_t>(nchunks_) * nr));
    GMM_CK(cudaMalloc(&scale_, sizeof(double) * nr));
    return {};
}

// Column norms of v ([n][nr]) into out[nr].
std::string GmresMulti::norms(const double2* v, cudaStream_t s, std::vector<double>& out) {
    k_mnorm2<<<nchunks_, kThreads, 0, s>>>(v, n_, nr_, npartial_);
    k_msum<<<1, kMaxRhs, 0, s>>>(npartial_, nchunks_, nr_, h_);
    std::vector<double2> t(nr_);
    GMM_CK(cudaMemcpyAsync(t.data(), h_, sizeof(double2) * nr_, cudaMemcpyDeviceToHost, s));
    GMM_CK(cudaStreamSynchronize(s));
    out.resize(nr_);
    for (int r = 0; r < nr_; ++r) out[r] = std::sqrt(t[r].x);
    return {};
}

// One CGS pass over columns 0..ncols-1: h (+)= Q^H w ; w -= Q h_pass.
void GmresMulti::cgs_pass(int ncols, cudaStream_t s, bool add) { cgs_pass_q(Q_, w_, ncols, s, h_, add); }

void GmresMulti::cgs_pass_q(const double2* Q, double2* w, int ncols, cudaStream_t s, double2* h, bool add) {
    const long long ld = static_cast<long long>(n_) * nr_;
    k_mdot<<<dim3(nchunks_, ncols), kThreads, 0, s>>>(Q, ld, w, n_, nr_, partial_, nchunks_);
    k_mreduce<<<nblk(static_cast<long long>(ncols) * nr_, 128), 128, 0, s>>>(partial_, nchunks_, ncols, nr_, y_, 0);
    k_msub_qh<<<nblk(ld, 256), 256, 0, s>>>(Q, ld, ncols, y_, w, ld, nr_);
    k_mreduce<<<nblk(static_cast<long long>(ncols) * nr_, 128), 128, 0, s>>>(partial_, nchunks_, ncols, nr_, h,
                                                                             add ? 1 : 0);
}

// Restarted GMRES on A(prec) x_ = b_ (all columns, x_ = 0 on entry) with
// per-column absolute targets tol_abs[r]; columns with done[r] set are left
// at zero.  iters[r] counts the column's Arnoldi steps.
std::string GmresMulti::cycles(DeviceOp& op, int prec, int restart, int max_iter, const std::vector<double>& bnorm,
                               const std::vector<double>& tol_abs, std::vector<char>& done, std::vector<int>& iters,
                               std::vector<double>& est) {
    using cd = std::complex<double>;
    const int n = n_, nr = nr_;
    const long long ld = static_cast<long long>(n) * nr;
    const int m = restart > 0 ? restart : max_iter;
    cudaStream_t s = op.stream();
    std::string err;
    GMM_CK(cudaMemsetAsync(x_, 0, sizeof(double2) * ld, s));
    std::vector<std::vector<cd>> H(nr), cs(nr), sn(nr), g(nr);
    std::vector<char> active(nr);
    std::vector<int> kr(nr);
    std::vector<double> beta(nr), sc(nr);
    std::vector<double2> hh(static_cast<size_t>(m + 2) * nr);
    int total = 0;
    bool first = true;
    while (total < max_iter) {
        // r = b - A x (first cycle: x = 0, r = b)
        if (first) {
            GMM_CK(cudaMemcpyAsync(r_, b_, sizeof(double2) * ld, cudaMemcpyDeviceToDevice, s));
            beta = bnorm;
        } else {
            op.apply_tree_multi(x_, w_, nr, s, prec);
            k_msub<<<nblk(ld, 256), 256, 0, s>>>(b_, w_, r_, ld);
            err = norms(r_, s, beta);
            if (!err.empty()) return err;
        }
        int nact = 0;
        for (int r = 0; r < nr; ++r) {
            if (!std::isfinite(beta[r])) return "nonfinite:residual";
            if (!done[r] && beta[r] <= tol_abs[r] && !first) { done[r] = 1; est[r] = beta[r] / bnorm[r]; }
            active[r] = !done[r] && beta[r] > 0.0;
            if (!done[r] && beta[r] == 0.0) done[r] = 1;
            sc[r] = active[r] ? 1.0 / beta[r] : 0.0;
            nact += active[r];
            kr[r] = 0;
            if (active[r]) {
                H[r].assign(static_cast<size_t>(m + 1) * m, cd(0));
                cs[r].assign(m, cd(0));
                sn[r].assign(m, cd(0));
                g[r].assign(m + 1, cd(0));
                g[r][0] = beta[r];
            }
        }
        first = false;
        if (nact == 0) break;
        GMM_CK(cudaMemcpyAsync(scale_, sc.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, s));
        k_mscale<<<nblk(ld, 256), 256, 0, s>>>(r_, scale_, Q_, ld, nr);
        int k = 0;
        for (; k < m && total < max_iter && nact > 0; ++k) {
            double2* qk = Q_ + static_cast<long long>(k) * ld;
            op.apply_tree_multi(qk, w_, nr, s, prec);
            cgs_pass(k + 1, s, false);
            cgs_pass(k + 1, s, true);
            k_mnorm2<<<nchunks_, kThreads, 0, s>>>(w_, n, nr, npartial_);
            k_msum<<<1, kMaxRhs, 0, s>>>(npartial_, nchunks_, nr, h_ + static_cast<size_t>(k + 1) * nr);
            GMM_CK(cudaMemcpyAsync(hh.data(), h_, sizeof(double2) * (k + 2) * nr, cudaMemcpyDeviceToHost, s));
            GMM_CK(cudaStreamSynchronize(s));
            ++total;
            for (int r = 0; r < nr; ++r) {
                sc[r] = 0.0;
                if (!active[r]) continue;
                const double hn = std::sqrt(hh[static_cast<size_t>(k + 1) * nr + r].x);
                if (!std::isfinite(hn)) return "nonfinite:Arnoldi";
                std::vector<cd> hc(k + 2);
                for (int i = 0; i <= k; ++i) hc[i] = cd(hh[static_cast<size_t>(i) * nr + r].x, hh[static_cast<size_t>(i) * nr + r].y);
                hc[k + 1] = hn;
                for (int i = 0; i < k; ++i) {  // unitary rotations (true residual norm)
                    const cd a = hc[i], b = hc[i + 1];
                    hc[i] = cs[r][i] * a + sn[r][i] * b;
                    hc[i + 1] = -std::conj(sn[r][i]) * a + cs[r][i] * b;
                }
                const double az = std::abs(hc[k]);
                const double t = std::sqrt(az * az + std::norm(hc[k + 1]));
                cd c, sg;
                if (az == 0.0) { c = 0.0; sg = 1.0; } else { c = az / t; sg = (hc[k] / az) * std::conj(hc[k + 1]) / t; }
                hc[k] = c * hc[k] + sg * hc[k + 1];
                g[r][k + 1] = -std::conj(sg) * g[r][k];
                g[r][k] = c * g[r][k];
                cs[r][k] = c;
                sn[r][k] = sg;
                for (int i = 0; i <= k; ++i) H[r][static_cast<size_t>(k) * (m + 1) + i] = hc[i];
                kr[r] = k + 1;
                ++iters[r];
                est[r] = std::abs(g[r][k + 1]) / bnorm[r];
                if (!(std::abs(g[r][k + 1]) > tol_abs[r]) || hn == 0.0) {
                    active[r] = 0;
                    done[r] = 1;
                    --nact;
                } else {
                    sc[r] = 1.0 / hn;
                }
            }
            if (nact > 0 && k + 1 < m && total < max_iter) {
                // next basis vectors (zero for frozen columns)
                GMM_CK(cudaMemcpyAsync(scale_, sc.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, s));
                k_mscale<<<nblk(ld, 256), 256, 0, s>>>(w_, scale_, Q_ + static_cast<long long>(k + 1) * ld, ld, nr);
            }
        }
        // x += Q y per column, y from the triangular system R y = g.
        int kmax = 0;
        for (int r = 0; r < nr; ++r) kmax = std::max(kmax, kr[r]);
        if (kmax > 0) {
            std::vector<double2> yd(static_cast<size_t>(kmax) * nr, make_double2(0.0, 0.0));
            for (int r = 0; r < nr; ++r) {
                const int kk = kr[r];
                std::vector<cd> yv(kk);
                for (int i = kk - 1; i >= 0; --i) {
                    cd acc = g[r][i];
                    for (int j = i + 1; j < kk; ++j) acc -= H[r][static_cast<size_t>(j) * (m + 1) + i] * yv[j];
                    yv[i] = acc / H[r][static_cast<size_t>(i) * (m + 1) + i];
                }
                for (int i = 0; i < kk; ++i) yd[static_cast<size_t>(i) * nr + r] = make_double2(-yv[i].real(), -yv[i].imag());
            }
            GMM_CK(cudaMemcpyAsync(y_, yd.data(), sizeof(double2) * yd.size(), cudaMemcpyHostToDevice, s));
            k_msub_qh<<<nblk(ld, 256), 256, 0, s>>>(Q_, ld, kmax, y_, x_, ld, nr);
            GMM_CK(cudaStreamSynchronize(s));
        }
        if (restart <= 0) break;
        bool all = true;
        for (int r = 0; r < nr; ++r) all = all && done[r];
        if (all) break;
    }
    return {};
}

std::string GmresMulti::solve(DeviceOp& op, int nr, const double2* d_b_user, double2* d_x_user, const SolveOpts& o,
                              std::vector<SolveResult>& res) {
    const auto t_start = std::chrono::steady_clock::now();
    const int n = op.n();
    if (nr < 1 || nr > op.max_rhs()) return "arg:nrhs must be between 1 and the operator's max_rhs";
    const int m = o.restart > 0 ? o.restart : o.max_iter;
    if (m < 1 || o.max_iter < 1) return "arg:max_iter and restart must be positive";
    if (o.flexible) return solve_flexible(op, nr, d_b_user, d_x_user, o, res);
    std::string err = ensure(n, nr, m + 1);
    if (!err.empty()) return err;
    cudaStream_t s = op.stream();
    const long long ld = static_cast<long long>(n) * nr;
    const bool refine = o.refine && op.precision() != kFp64;
    res.assign(nr, SolveResult{});
    k_mgather<<<nblk(ld, 256), 256, 0, s>>>(d_b_user, op.perm(), bo_, n, nr);
    GMM_CK(cudaMemcpyAsync(b_, bo_, sizeof(double2) * ld, cudaMemcpyDeviceToDevice, s));
    std::vector<double> bnorm;
    err = norms(bo_, s, bnorm);
    if (!err.empty()) return err;
    std::vector<char> done(nr, 0);
    std::vector<int> iters(nr, 0);
    std::vector<double> est(nr, 0.0), tol_abs(nr);
    for (int r = 0; r < nr; ++r) {
        if (!std::isfinite(bnorm[r])) return "nonfinite:right-hand side";
        tol_abs[r] = o.tol * bnorm[r];
        if (bnorm[r] == 0.0) done[r] = 1;
    }
    std::vector<double> rn = bnorm;
    if (!refine) {
        err = cycles(op, -1, o.restart, o.max_iter, bnorm, tol_abs, done, iters, est);
        if (!err.empty()) return err;
        GMM_CK(cudaMemcpyAsync(xo_, x_, sizeof(double2) * ld, cudaMemcpyDeviceToDevice, s));
        op.apply_tree_multi(xo_, w_, nr, s, -1);
        k_msub<<<nblk(ld, 256), 256, 0, s>>>(bo_, w_, r_, ld);
        err = norms(r_, s, rn);
        if (!err.empty()) return err;
    } else {
        // Iterative refinement: FP64 outer residual, mixed inner solves.
        GMM_CK(cudaMemsetAsync(xo_, 0, sizeof(double2) * ld, s));
        std::vector<char> conv(nr, 0);
        for (int r = 0; r < nr; ++r) conv[r] = bnorm[r] == 0.0;
        for (int outer = 0; outer < 20; ++outer) {
            std::vector<char> idone(nr);
            std::vector<double> itol(nr);
            int left = 0;
            for (int r = 0; r < nr; ++r) {
                idone[r] = conv[r];
                const double eta = std::min(0.5, o.inner_tol > 0 ? o.inner_tol : 0.9 * o.tol * bnorm[r] / std::max(rn[r], 1e-300));
                itol[r] = eta * rn[r];
                left += !conv[r];
            }
            if (left == 0) break;
            int maxit = 0;
            for (int r = 0; r < nr; ++r) maxit = std::max(maxit, o.max_iter - iters[r]);
            if (maxit <= 0) break;
            std::vector<int> it(nr, 0);
            err = cycles(op, kMixed, o.restart, maxit, rn, itol, idone, it, est);
            if (!err.empty()) return err;
            bool progress = false;
            for (int r = 0; r < nr; ++r) { iters[r] += it[r]; progress = progress || it[r] > 0; }
            k_maxpy<<<nblk(ld, 256), 256, 0, s>>>(x_, xo_, ld);  // frozen columns have x_ = 0
            op.apply_tree_multi(xo_, w_, nr, s, kFp64);
            k_msub<<<nblk(ld, 256), 256, 0, s>>>(bo_, w_, b_, ld);
            err = norms(b_, s, rn);
            if (!err.empty()) return err;
            for (int r = 0; r < nr; ++r) {
                if (!std::isfinite(rn[r])) return "nonfinite:residual";
                if (!conv[r]) ++res[r].refinements;
                if (rn[r] <= tol_abs[r]) conv[r] = 1;
            }
            if (!progress) break;
        }
    }
    k_mscatter<<<nblk(ld, 256), 256, 0, s>>>(xo_, op.perm(), d_x_user, n, nr);
    GMM_CK(cudaStreamSynchronize(s));
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    for (int r = 0; r < nr; ++r) {
        res[r].iterations = iters[r];
        res[r].true_residual = bnorm[r] > 0 ? rn[r] / bnorm[r] : 0.0;
        res[r].residual = refine ? res[r].true_residual : est[r];
        res[r].converged = bnorm[r] == 0.0 || rn[r] <= tol_abs[r] * (1.0 + 1e-12) || (!refine && done[r]);
        res[r].seconds = secs;
    }
    return {};
}

// Flexible GMRES on many right-hand sides (Gmres::solve_flexible, one column
// at a time there).  Each column r has its own FP64 outer space: basis V_r,
// preconditioned directions Z_r, Hessenberg matrix, unitary rotations and
// residual.  Outer step k solves A z = v_k for every working column at once:
// inner_iters GMRES iterations from zero on the operator's own far field
// (complex float on a mixed operator), through the batched cycles above, so
// the columns share every inner product launch; then w = A z_k in FP64 (the
// batched FP64 product), CGS2 against the column's V, and the columns' Givens
// rotations on the host.  x_r = Z_r y_r exactly after each cycle, and the
// stopping test is the FP64 residual.  A column that meets its tolerance is
// frozen (zero directions) while the others go on; iterations counts a
// column's inner iterations and refinements its outer steps.
std::string GmresMulti::solve_flexible(DeviceOp& op, int nr, const double2* d_b_user, double2* d_x_user,
                                       const SolveOpts& o, std::vector<SolveResult>& res) {
    using cd = std::complex<double>;
    const auto t_start = std::chrono::steady_clock::now();
    const int n = op.n();
    const int mo = o.restart > 0 ? o.restart : o.max_iter;
    const int mi = o.inner_iters > 0 ? o.inner_iters : 20;
    if (mo < 1 || o.max_iter < 1) return "arg:max_iter and restart must be positive";
    if (o.inner && o.inner != &op) return "arg:an inner operator serves the one-right-hand-side flexible solve";
    std::string err = ensure(n, nr, std::max(mi, mo) + 1);
    if (!err.empty()) return err;
    const long long ld = static_cast<long long>(n) * nr;
    if (vcap_ < mo) {
        for (void* p : {(void*)V_, (void*)Z_})
            if (p) cudaFree(p);
        V_ = Z_ = nullptr;
        vcap_ = 0;
        GMM_CK(cudaMalloc(&V_, sizeof(double2) * ld * (mo + 1)));
        GMM_CK(cudaMalloc(&Z_, sizeof(double2) * ld * mo));
        vcap_ = mo;
    }
    cudaStream_t s = op.stream();
    const int prec_in = op.precision();
    res.assign(nr, SolveResult{});
    k_mgather<<<nblk(ld, 256), 256, 0, s>>>(d_b_user, op.perm(), bo_, n, nr);
    std::vector<double> bnorm;
    err = norms(bo_, s, bnorm);
    if (!err.empty()) return err;
    std::vector<double> tol_abs(nr), beta = bnorm, sc(nr);
    std::vector<char> conv(nr, 0), active(nr, 0);
    std::vector<int> iters(nr, 0), outer(nr, 0), kr(nr, 0);
    for (int r = 0; r < nr; ++r) {
        if (!std::isfinite(bnorm[r])) return "nonfinite:right-hand side";
        tol_abs[r] = o.tol * bnorm[r];
        conv[r] = bnorm[r] == 0.0;
    }
    GMM_CK(cudaMemsetAsync(xo_, 0, sizeof(double2) * ld, s));
    GMM_CK(cudaMemcpyAsync(r_, bo_, sizeof(double2) * ld, cudaMemcpyDeviceToDevice, s));  // r = b (x = 0)
    std::vector<std::vector<cd>> H(nr), cs(nr), sn(nr), g(nr);
    std::vector<double2> hh(static_cast<size_t>(mo + 2) * nr);
    for (;;) {
        int nact = 0;
        for (int r = 0; r < nr; ++r) {
            active[r] = !conv[r] && beta[r] > 0.0 && iters[r] < o.max_iter;
            sc[r] = active[r] ? 1.0 / beta[r] : 0.0;
            kr[r] = 0;
            nact += active[r];
            if (active[r]) {
                H[r].assign(static_cast<size_t>(mo + 1) * mo, cd(0));
                cs[r].assign(mo, cd(0));
                sn[r].assign(mo, cd(0));
                g[r].assign(mo + 1, cd(0));
                g[r][0] = beta[r];
            }
        }
        if (nact == 0) break;
        GMM_CK(cudaMemcpyAsync(scale_, sc.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, s));
        k_mscale<<<nblk(ld, 256), 256, 0, s>>>(r_, scale_, V_, ld, nr);  // v_0 = r / beta, zero when frozen
        for (int k = 0; k < mo && nact > 0; ++k) {
            double2* vk = V_ + static_cast<long long>(k) * ld;
            double2* zk = Z_ + static_cast<long long>(k) * ld;
            // inner solves A z = v_k from zero (||v_k|| = 1 in every working column)
            std::vector<char> idone(nr);
            std::vector<double> ib(nr), itol(nr), iest(nr, 0.0);
            std::vector<int> it(nr, 0);
            int maxit = 0;
            for (int r = 0; r < nr; ++r) {
                idone[r] = !active[r];
                ib[r] = active[r] ? 1.0 : 0.0;
                itol[r] = active[r] && o.inner_tol > 0 ? o.inner_tol : 0.0;
                if (active[r]) maxit = std::max(maxit, std::min(mi, o.max_iter - iters[r]));
            }
            GMM_CK(cudaMemcpyAsync(b_, vk, sizeof(double2) * ld, cudaMemcpyDeviceToDevice, s));
            err = cycles(op, prec_in, mi, std::max(1, maxit), ib, itol, idone, it, iest);
            if (!err.empty()) return err;
            GMM_CK(cudaMemcpyAsync(zk, x_, sizeof(double2) * ld, cudaMemcpyDeviceToDevice, s));
            // w = A z_k in FP64, orthogonalised against v_0..v_k of its column
            op.apply_tree_multi(zk, w_, nr, s, kFp64);
            cgs_pass_q(V_, w_, k + 1, s, h_, false);
            cgs_pass_q(V_, w_, k + 1, s, h_, true);
            k_mnorm2<<<nchunks_, kThreads, 0, s>>>(w_, n, nr, npartial_);
            k_msum<<<1, kMaxRhs, 0, s>>>(npartial_, nchunks_, nr, h_ + static_cast<size_t>(k + 1) * nr);
            GMM_CK(cudaMemcpyAsync(hh.data(), h_, sizeof(double2) * (k + 2) * nr, cudaMemcpyDeviceToHost, s));
            GMM_CK(cudaStreamSynchronize(s));
            for (int r = 0; r < nr; ++r) {
                sc[r] = 0.0;
                if (!active[r]) continue;
                iters[r] += it[r];
                ++outer[r];
                const double hn = std::sqrt(hh[static_cast<size_t>(k + 1) * nr + r].x);
                if (!std::isfinite(hn)) return "nonfinite:Arnoldi";
                std::vector<cd> hc(k + 2);
                for (int i = 0; i <= k; ++i)
                    hc[i] = cd(hh[static_cast<size_t>(i) * nr + r].x, hh[static_cast<size_t>(i) * nr + r].y);
                hc[k + 1] = hn;
                for (int i = 0; i < k; ++i) {  // previous unitary rotations
                    const cd a = hc[i], b = hc[i + 1];
                    hc[i] = cs[r][i] * a + sn[r][i] * b;
                    hc[i + 1] = -std::conj(sn[r][i]) * a + cs[r][i] * b;
                }
                const double az = std::abs(hc[k]);
                const double t = std::sqrt(az * az + std::norm(hc[k + 1]));
                cd c, sg;
                if (az == 0.0) { c = 0.0; sg = 1.0; } else { c = az / t; sg = (hc[k] / az) * std::conj(hc[k + 1]) / t; }
                hc[k] = c * hc[k] + sg * hc[k + 1];
                g[r][k + 1] = -std::conj(sg) * g[r][k];
                g[r][k] = c * g[r][k];
                cs[r][k] = c;
                sn[r][k] = sg;
                for (int i = 0; i <= k; ++i) H[r][static_cast<size_t>(k) * (mo + 1) + i] = hc[i];
                kr[r] = k + 1;
                if (!(std::abs(g[r][k + 1]) > tol_abs[r]) || hn == 0.0 || iters[r] >= o.max_iter) {
                    active[r] = 0;
                    --nact;
                } else {
                    sc[r] = 1.0 / hn;
                }
            }
            if (nact > 0 && k + 1 < mo) {
                GMM_CK(cudaMemcpyAsync(scale_, sc.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, s));
                k_mscale<<<nblk(ld, 256), 256, 0, s>>>(w_, scale_, V_ + static_cast<long long>(k + 1) * ld, ld, nr);
            }
        }
        // x += Z y per column, R y = g
        int kmax = 0;
        for (int r = 0; r < nr; ++r) kmax = std::max(kmax, kr[r]);
        if (kmax > 0) {
            std::vector<double2> yd(static_cast<size_t>(kmax) * nr, make_double2(0.0, 0.0));
            for (int r = 0; r < nr; ++r) {
                const int kk = kr[r];
                std::vector<cd> yv(kk);
                for (int i = kk - 1; i >= 0; --i) {
                    cd acc = g[r][i];
                    for (int j = i + 1; j < kk; ++j) acc -= H[r][static_cast<size_t>(j) * (mo + 1) + i] * yv[j];
                    yv[i] = acc / H[r][static_cast<size_t>(i) * (mo + 1) + i];
                }
                for (int i = 0; i < kk; ++i) yd[static_cast<size_t>(i) * nr + r] = make_double2(-yv[i].real(), -yv[i].imag());
            }
            GMM_CK(cudaMemcpyAsync(y_, yd.data(), sizeof(double2) * yd.size(), cudaMemcpyHostToDevice, s));
            k_msub_qh<<<nblk(ld, 256), 256, 0, s>>>(Z_, ld, kmax, y_, xo_, ld, nr);
        }
        // true FP64 residual
        op.apply_tree_multi(xo_, w_, nr, s, kFp64);
        k_msub<<<nblk(ld, 256), 256, 0, s>>>(bo_, w_, r_, ld);
        err = norms(r_, s, beta);
        if (!err.empty()) return err;
        for (int r = 0; r < nr; ++r) {
            if (!std::isfinite(beta[r])) return "nonfinite:residual";
            if (beta[r] <= tol_abs[r]) conv[r] = 1;
        }
        if (o.restart <= 0) break;
    }
    k_mscatter<<<nblk(ld, 256), 256, 0, s>>>(xo_, op.perm(), d_x_user, n, nr);
    GMM_CK(cudaStreamSynchronize(s));
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    for (int r = 0; r < nr; ++r) {
        res[r].iterations = iters[r];
        res[r].refinements = outer[r];
        res[r].true_residual = bnorm[r] > 0 ? beta[r] / bnorm[r] : 0.0;
        res[r].residual = res[r].true_residual;
        res[r].converged = bnorm[r] == 0.0 || beta[r] <= tol_abs[r] * (1.0 + 1e-12);
        res[r].seconds = secs;
    }
    return {};
}

}  // namespace mlfma
