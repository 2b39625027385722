// GMRES on the device around the MLFMA operator (Solver, src/solver.cpp:5-146).
//
// The Krylov basis lives in HBM as (m+1) tree-ordered vectors.  Each Arnoldi
// step orthogonalises with two passes of classical Gram-Schmidt (CGS2): one
// batched Q^H w reduction and one batched w -= Q h update per pass, instead of
// the reference's k+1 sequential modified Gram-Schmidt dot/axpy pairs
// (solver.cpp:59-83); in exact arithmetic both give the same Hessenberg column.
// The small (k+2)-vector column comes back to the host, where the Givens
// rotations and the triangular solve run in FP64.  With ref_givens = 1 and
// restart = 0 the rotations are the reference's complex-symmetric ones
// (Math::givensRotation, src/math.h:168-172; applyGivensRotation and
// updateGvec, solver.cpp:85-113) and the stopping test is |g_{k+1}|/g0
// (solver.cpp:139); otherwise unitary rotations give the true residual norm.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <complex>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "gmres.hpp"

namespace mlfma {

namespace {

constexpr int kDotThreads = 256;
constexpr int kDotChunk = 8192;  // vector elements per partial sum
constexpr int kStepChunk = 1024;  // the same in the device-resident steps (more blocks in flight)
constexpr int kUpdThreads = 128;  // k_step_update block

__device__ __forceinline__ double2 cj_mul_add(double2 a, double2 b, double2 c) {
    return make_double2(fma(a.x, b.x, fma(a.y, b.y, c.x)), fma(a.x, b.y, fma(-a.y, b.x, c.y)));
}

// partial[j][c] = sum_{i in chunk c} conj(Q_j[i]) w[i]
__global__ void k_multi_dot(const double2* __restrict__ Q, long long ld, int ncols,
                            const double2* __restrict__ w, int n, double2* __restrict__ partial,
                            int nchunks) {
    __shared__ double2 red[kDotThreads];
    const int c = blockIdx.x, j = blockIdx.y;
    const double2* q = Q + static_cast<long long>(j) * ld;
    const int i0 = c * kDotChunk, i1 = min(n, i0 + kDotChunk);
    double2 acc = make_double2(0.0, 0.0);
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) acc = cj_mul_add(q[i], w[i], acc);
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red[threadIdx.x].x += red[threadIdx.x + s].x;
            red[threadIdx.x].y += red[threadIdx.x + s].y;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[static_cast<long long>(j) * nchunks + c] = red[0];
}

// h[j] (+)= sum_c partial[j][c]   (fixed order: deterministic)
__global__ void k_reduce_partials(const double2* __restrict__ partial, int nchunks, int ncols,
                                  double2* __restrict__ h, int add) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ncols) return;
    double2 s = make_double2(0.0, 0.0);
    for (int c = 0; c < nchunks; ++c) {
        s.x += partial[static_cast<long long>(j) * nchunks + c].x;
        s.y += partial[static_cast<long long>(j) * nchunks + c].y;
    }
    if (add) { h[j].x += s.x; h[j].y += s.y; } else { h[j] = s; }
}

// w[i] -= sum_j Q_j[i] h[j]
__global__ void k_sub_qh(const double2* __restrict__ Q, long long ld, int ncols,
                         const double2* __restrict__ h, double2* __restrict__ w, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double2 v = w[i];
    for (int j = 0; j < ncols; ++j) {
        const double2 q = Q[static_cast<long long>(j) * ld + i];
        const double2 hj = h[j];
        v.x -= q.x * hj.x - q.y * hj.y;
        v.y -= q.x * hj.y + q.y * hj.x;
    }
    w[i] = v;
}

// partial[c] = sum |w[i]|^2 over chunk c
__global__ void k_norm2(const double2* __restrict__ w, int n, double* __restrict__ partial) {
    __shared__ double red[kDotThreads];
    const int c = blockIdx.x;
    const int i0 = c * kDotChunk, i1 = min(n, i0 + kDotChunk);
    double acc = 0.0;
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) acc = fma(w[i].x, w[i].x, fma(w[i].y, w[i].y, acc));
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[c] = red[0];
}

// out = a * x  (complex scale)
__global__ void k_scale(const double2* __restrict__ x, double2 a, double2* __restrict__ out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double2 v = x[i];
    out[i] = make_double2(a.x * v.x - a.y * v.y, a.x * v.y + a.y * v.x);
}

// out->x = sum of partial[0..n) in a fixed order (one thread)
__global__ void k_sum_into(const double* __restrict__ partial, int n, double2* __restrict__ out) {
    double acc = 0.0;
    for (int c = 0; c < n; ++c) acc += partial[c];
    *out = make_double2(acc, 0.0);
}

// y += x
__global__ void k_axpy1(const double2* __restrict__ x, double2* __restrict__ y, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    y[i] = make_double2(y[i].x + x[i].x, y[i].y + x[i].y);
}

// out = b - y
__global__ void k_sub(const double2* __restrict__ b, const double2* __restrict__ y, double2* __restrict__ out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = make_double2(b[i].x - y[i].x, b[i].y - y[i].y);
}

__global__ void k_gather_perm(const double2* __restrict__ x, const int* __restrict__ perm, double2* __restrict__ xt, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) xt[t] = x[perm[t]];
}
__global__ void k_scatter_perm(const double2* __restrict__ xt, const int* __restrict__ perm, double2* __restrict__ x, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) x[perm[t]] = xt[t];
}

inline int nblk(long long n, int bs) { return static_cast<int>((n + bs - 1) / bs); }

// ---------------------------------------------------------------- device-resident Arnoldi step
// The step index k lives in device memory, so one captured graph serves every
// step of a cycle.
constexpr int kMaxDeviceSteps = 256;  // basis vectors per cycle that the step kernels handle
constexpr int kStepBatch = 8;         // device steps between host reads of the Hessenberg columns
struct StepStateD {
    int k;
    unsigned cnt;
    double hn;
    double w0;  // ||w||^2 before this step's orthogonalisation
    int skip;   // 1: the first CGS pass kept enough of w, the second is skipped
};

// q_k = w (1 / hn) for k > 0 (q_0 is set by the cycle), and the product's input
// xt = q_k (conj(q_k) for the adjoint).
__global__ void k_step_prep(StepStateD* __restrict__ st, double2* __restrict__ Q, const double2* __restrict__ w,
                            double2* __restrict__ xt, int n, int adj) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = st->k;
    double2 q;
    if (k == 0) {
        q = Q[i];
    } else {
        const double hn = st->hn;
        const double2 v = w[i];
        const double a = hn > 0 ? 1.0 / hn : 0.0;
        q = make_double2(a * v.x, a * v.y);
        Q[static_cast<long long>(k) * n + i] = q;
    }
    xt[i] = adj ? make_double2(q.x, -q.y) : q;
}

// One CGS pass, dots: partial[j][c] = sum_{i in chunk c} conj(Q_j[i]) w[i] for
// j <= k.  Block (c, g) reads chunk c of w once (four elements per thread, in
// registers) and forms the dots with the kStepCols columns j = g kStepCols ..
// of group g; the last block to finish sums each j's partials in a fixed order
// into t[j] and into column k of the Hessenberg matrix (pass 0 sets it, pass 1
// adds).
constexpr int kStepCols = 8;
__global__ void __launch_bounds__(kDotThreads)
k_step_dots(StepStateD* __restrict__ st, const double2* __restrict__ Q, int n, const double2* __restrict__ w,
            double2* __restrict__ partial, int nchunks, double2* __restrict__ t, double2* __restrict__ hcols, int ldh,
            int pass, double* __restrict__ wnorm) {
    __shared__ double2 red[kStepCols][kDotThreads];
    __shared__ double wred[kDotThreads / 32];
    __shared__ bool last;
    if (pass == 1 && st->skip) return;  // the whole grid: the second pass is not needed
    const int c = blockIdx.x, j0 = blockIdx.y * kStepCols;
    const int k = st->k;
    constexpr int per = kStepChunk / kDotThreads;  // elements per thread
    if (j0 <= k) {
        const int i0 = c * kStepChunk;
        double2 wv[per];
#pragma unroll
        for (int e = 0; e < per; ++e) {
            const int i = i0 + e * kDotThreads + threadIdx.x;
            wv[e] = i < n ? w[i] : make_double2(0.0, 0.0);
        }
        if (pass == 0 && blockIdx.y == 0) {  // ||chunk of w||^2, for the reorthogonalisation test
            double nn = 0.0;
#pragma unroll
            for (int e = 0; e < per; ++e) nn = fma(wv[e].x, wv[e].x, fma(wv[e].y, wv[e].y, nn));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) nn += __shfl_xor_sync(0xffffffffu, nn, o);
            if ((threadIdx.x & 31) == 0) wred[threadIdx.x >> 5] = nn;
            __syncthreads();
            if (threadIdx.x == 0) {
                double a = 0.0;
                for (int q = 0; q < kDotThreads / 32; ++q) a += wred[q];
                wnorm[c] = a;
            }
        }
#pragma unroll
        for (int jj = 0; jj < kStepCols; ++jj) {
            const int j = j0 + jj;
            double2 acc = make_double2(0.0, 0.0);
            if (j <= k) {
                const double2* q = Q + static_cast<long long>(j) * n;
                double2 qv[per];
#pragma unroll
                for (int e = 0; e < per; ++e) {
                    const int i = i0 + e * kDotThreads + threadIdx.x;
                    qv[e] = i < n ? q[i] : make_double2(0.0, 0.0);
                }
#pragma unroll
                for (int e = 0; e < per; ++e) acc = cj_mul_add(qv[e], wv[e], acc);
            }
            red[jj][threadIdx.x] = acc;
        }
        __syncthreads();
        // warp jj sums column jj's kDotThreads values: eight per lane, then a butterfly
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (warp < kStepCols && j0 + warp <= k) {
            double2 a = make_double2(0.0, 0.0);
#pragma unroll
            for (int e = 0; e < kDotThreads / 32; ++e) {
                const double2 v = red[warp][e * 32 + lane];
                a.x += v.x;
                a.y += v.y;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                a.x += __shfl_xor_sync(0xffffffffu, a.x, o);
                a.y += __shfl_xor_sync(0xffffffffu, a.y, o);
            }
            if (lane == 0) partial[static_cast<long long>(j0 + warp) * nchunks + c] = a;
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&st->cnt, 1u) == gridDim.x * gridDim.y - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    double2* h = hcols + static_cast<long long>(k) * ldh;
    for (int jj = threadIdx.x; jj <= k; jj += blockDim.x) {
        double2 sum = make_double2(0.0, 0.0);
        for (int cc = 0; cc < nchunks; ++cc) {
            const double2 p = __ldcg(partial + static_cast<long long>(jj) * nchunks + cc);
            sum.x += p.x;
            sum.y += p.y;
        }
        t[jj] = sum;
        h[jj] = pass ? make_double2(h[jj].x + sum.x, h[jj].y + sum.y) : sum;
    }
    if (threadIdx.x == 0) {
        if (pass == 0) {
            double a = 0.0;
            for (int cc = 0; cc < nchunks; ++cc) a += __ldcg(wnorm + cc);
            st->w0 = a;
        }
        st->cnt = 0;
    }
}

// One CGS pass, update: w -= sum_{j <= k} Q_j t[j].  The second pass also
// forms ||w||^2 (block partials, the last block sums them in a fixed order):
// h[k+1] = (||w||^2, 0), hn = ||w||, and the step index moves on.
__global__ void k_step_update(StepStateD* __restrict__ st, const double2* __restrict__ Q, int n,
                              const double2* __restrict__ t, double2* __restrict__ w, double* __restrict__ npart,
                              double2* __restrict__ hcols, int ldh, int pass) {
    __shared__ double red[kUpdThreads];
    __shared__ bool last;
    if (pass == 1 && st->skip) return;  // the whole grid
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = st->k;
    double nn = 0.0;
    if (i < n) {
        // four independent partial sums over the basis vectors, then in order
        double2 u[4] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0),
                        make_double2(0.0, 0.0)};
        int j = 0;
        for (; j + 3 <= k; j += 4) {
            double2 q[4], h[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                q[a] = Q[static_cast<long long>(j + a) * n + i];
                h[a] = t[j + a];
            }
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                u[a].x += q[a].x * h[a].x - q[a].y * h[a].y;
                u[a].y += q[a].x * h[a].y + q[a].y * h[a].x;
            }
        }
        for (; j <= k; ++j) {
            const double2 q = Q[static_cast<long long>(j) * n + i];
            const double2 hj = t[j];
            u[0].x += q.x * hj.x - q.y * hj.y;
            u[0].y += q.x * hj.y + q.y * hj.x;
        }
        double2 v = w[i];
        v.x -= (u[0].x + u[1].x) + (u[2].x + u[3].x);
        v.y -= (u[0].y + u[1].y) + (u[2].y + u[3].y);
        w[i] = v;
        nn = fma(v.x, v.x, v.y * v.y);
    }
    red[threadIdx.x] = nn;
    __syncthreads();
    for (int s2 = blockDim.x / 2; s2 > 0; s2 >>= 1) {
        if (threadIdx.x < s2) red[threadIdx.x] += red[threadIdx.x + s2];
        __syncthreads();
    }
    if (threadIdx.x == 0) npart[blockIdx.x] = red[0];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&st->cnt, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double acc = 0.0;
    for (int b = 0; b < static_cast<int>(gridDim.x); ++b) acc += __ldcg(npart + b);
    st->cnt = 0;
    // Twice is enough: a second pass only when the first one cancelled more
    // than half of ||w||^2 (||w_1|| <= ||w_0|| / sqrt 2).
    if (pass == 0) {
        st->skip = acc > 0.5 * st->w0 ? 1 : 0;
        if (!st->skip) return;
    }
    hcols[static_cast<long long>(k) * ldh + k + 1] = make_double2(acc, 0.0);
    st->hn = sqrt(acc);
    st->k = k + 1;
}

}  // namespace

#define GM_CK(call)                                                                \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) return std::string(#call) + ": " + cudaGetErrorString(e_); \
    } while (0)

// extra = 2: also the two vectors of iterative refinement.
std::string Gmres::ensure(int n, int ncols, int extra) {
    if (external_)
        return (n == n_ && ncols <= cap_ && extra <= extra_) ? std::string()
                                                             : std::string("fixed workspace set up for another size");
    if (n == n_ && ncols <= cap_ && extra <= extra_) return {};
    release();
    n_ = n;
    cap_ = ncols;
    extra_ = extra;
    nchunks_ = (n + kDotChunk - 1) / kDotChunk;
    GM_CK(cudaMalloc(&Q_, sizeof(double2) * static_cast<size_t>(n) * ncols));
    GM_CK(cudaMalloc(&w_, sizeof(double2) * n));
    GM_CK(cudaMalloc(&b_, sizeof(double2) * n));
    GM_CK(cudaMalloc(&x_, sizeof(double2) * n));
    GM_CK(cudaMalloc(&r_, sizeof(double2) * n));
    GM_CK(cudaMalloc(&h_, sizeof(double2) * (ncols + 1)));
    GM_CK(cudaMalloc(&y_, sizeof(double2) * (ncols + 1)));
    GM_CK(cudaMalloc(&partial_, sizeof(double2) * static_cast<size_t>(nchunks_) * (ncols + 1)));
    GM_CK(cudaMalloc(&npartial_, sizeof(double) * nchunks_));
    GM_CK(cudaMalloc(&tq_, sizeof(double2) * n));
    if (extra >= 2) {
        GM_CK(cudaMalloc(&xo_, sizeof(double2) * n));
        GM_CK(cudaMalloc(&bo_, sizeof(double2) * n));
    }
    if (ncols <= kMaxDeviceSteps + 1) {
        GM_CK(cudaMalloc(&st_, sizeof(StepStateD)));
        GM_CK(cudaMalloc(&hcols_, sizeof(double2) * static_cast<size_t>(ncols) * (ncols + 1)));
        GM_CK(cudaMalloc(&tco_, sizeof(double2) * (ncols + 1)));
        GM_CK(cudaMalloc(&npart2_, sizeof(double) * nblk(n, kUpdThreads)));
        nstep_ = (n + kStepChunk - 1) / kStepChunk;
        GM_CK(cudaMalloc(&spartial_, sizeof(double2) * static_cast<size_t>(nstep_) * (ncols + 1)));
        GM_CK(cudaMalloc(&swnorm_, sizeof(double) * nstep_));
    }
    return {};
}

void Gmres::release_steps() {
    if (sgx_) cudaGraphExecDestroy(sgx_);
    if (sg_) cudaGraphDestroy(sg_);
    sgx_ = nullptr;
    sg_ = nullptr;
    sg_op_ = nullptr;
    for (void* p : {st_, (void*)hcols_, (void*)tco_, (void*)npart2_, (void*)spartial_, (void*)swnorm_})
        if (p) cudaFree(p);
    swnorm_ = nullptr;
    st_ = nullptr;
    hcols_ = nullptr;
    tco_ = nullptr;
    npart2_ = nullptr;
    spartial_ = nullptr;
}

// The captured Arnoldi step for this operator, precision and direction
// (recaptured when any of them, the operator's generation or the workspace
// changes).
std::string Gmres::step_graph(DeviceOp& op, int prec) {
    const int adj = adj_ ? 1 : 0;
    const int pc = pc_ ? 1 : 0;
    if (sgx_ && sg_op_ == &op && sg_prec_ == prec && sg_adj_ == adj && sg_gen_ == op.generation() && sg_q_ == Q_ &&
        sg_pc_ == pc)
        return {};
    if (sgx_) cudaGraphExecDestroy(sgx_);
    if (sg_) cudaGraphDestroy(sg_);
    sgx_ = nullptr;
    sg_ = nullptr;
    cudaStream_t s = op.stream();
    StepStateD* st = static_cast<StepStateD*>(st_);
    const int n = n_, ldh = cap_ + 1;
    GM_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    if (pc) {  // the product's input is M^{-1} q_k
        k_step_prep<<<nblk(n, 256), 256, 0, s>>>(st, Q_, w_, tq_, n, 0);
        op.bj_apply(tq_, op.input_buffer(), s);
    } else {
        k_step_prep<<<nblk(n, 256), 256, 0, s>>>(st, Q_, w_, op.input_buffer(), n, adj);
    }
    op.enqueue_apply_from_input(w_, s, prec, adj_);
    for (int pass = 0; pass < 2; ++pass) {
        k_step_dots<<<dim3(nstep_, (cap_ + kStepCols - 1) / kStepCols), kDotThreads, 0, s>>>(st, Q_, n, w_, spartial_,
                                                                                          nstep_, tco_, hcols_, ldh,
                                                                                          pass, swnorm_);
        k_step_update<<<nblk(n, kUpdThreads), kUpdThreads, 0, s>>>(st, Q_, n, tco_, w_, npart2_, hcols_, ldh, pass);
    }
    const cudaError_t ce = cudaStreamEndCapture(s, &sg_);
    if (ce != cudaSuccess) return std::string("step capture: ") + cudaGetErrorString(ce);
    GM_CK(cudaGraphInstantiate(&sgx_, sg_, cudaGraphInstantiateFlagUseNodePriority));
    sg_op_ = &op;
    sg_prec_ = prec;
    sg_adj_ = adj;
    sg_gen_ = op.generation();
    sg_q_ = Q_;
    sg_pc_ = pc;
    return {};
}

void Gmres::release() {
    release_steps();
    if (!external_)
        for (void* p : {(void*)Q_, (void*)w_, (void*)b_, (void*)x_, (void*)r_, (void*)h_, (void*)y_,
                        (void*)partial_, (void*)npartial_, (void*)xo_, (void*)bo_, (void*)tq_})
            if (p) cudaFree(p);
    Q_ = w_ = b_ = x_ = r_ = h_ = y_ = partial_ = xo_ = bo_ = tq_ = nullptr;
    npartial_ = nullptr;
    n_ = cap_ = extra_ = 0;
}

Gmres::~Gmres() {
    release();
    release_outer();
}

std::string Gmres::ensure_outer(int n, int ncols) {
    if (n == on_ && ncols <= ocap_) return {};
    release_outer();
    on_ = n;
    ocap_ = ncols;
    const int nch = (n + kDotChunk - 1) / kDotChunk;
    GM_CK(cudaMalloc(&V_, sizeof(double2) * static_cast<size_t>(n) * (ncols + 1)));
    GM_CK(cudaMalloc(&Z_, sizeof(double2) * static_cast<size_t>(n) * ncols));
    GM_CK(cudaMalloc(&wo_, sizeof(double2) * n));
    GM_CK(cudaMalloc(&xf_, sizeof(double2) * n));
    GM_CK(cudaMalloc(&bf_, sizeof(double2) * n));
    GM_CK(cudaMalloc(&ho_, sizeof(double2) * (ncols + 2)));
    GM_CK(cudaMalloc(&to_, sizeof(double2) * (ncols + 2)));
    GM_CK(cudaMalloc(&po_, sizeof(double2) * static_cast<size_t>(nch) * (ncols + 2)));
    return {};
}

void Gmres::release_outer() {
    for (void* p : {(void*)V_, (void*)Z_, (void*)wo_, (void*)xf_, (void*)bf_, (void*)ho_, (void*)to_, (void*)po_})
        if (p) cudaFree(p);
    V_ = Z_ = wo_ = xf_ = bf_ = ho_ = to_ = po_ = nullptr;
    on_ = ocap_ = 0;
}

void Gmres::apply(DeviceOp& op, const double2* x, double2* y, cudaStream_t s, int prec) {
    if (external_) op.apply_tree_direct(x, y, s, prec, adj_); else op.apply_tree(x, y, s, prec, adj_);
}

// ------------------------------------------------------------ fixed workspace
// Some callers cannot allocate device memory while they solve: code that runs
// with a device memory budget fixed at start-up, or under an allocator policy
// that forbids cudaMalloc outside initialisation.  For them the library keeps
// one fixed GMRES workspace in device memory that is part of this file's
// module: kNoAllocWorkspace complex doubles (32 MiB) for the Krylov basis and
// work vectors, and kNoAllocNorm doubles for norm partial sums.  CUDA loads
// modules lazily, so the arrays are created on a device when the module is
// first used there; mlfma_setup forces that (noalloc_workspace_prepare) on the
// operator's device, and the memory stays until the process exits.  Every
// solve shares the arrays and they keep the previous solve's contents (every
// element is written before it is read); two solves that overlap on the GPU
// race on them.
constexpr size_t kNoAllocWorkspace = size_t(1) << 21;
constexpr int kNoAllocNorm = 4096;
static __device__ __align__(256) double2 g_noalloc_ws[kNoAllocWorkspace];
static __device__ __align__(256) double g_noalloc_norm[kNoAllocNorm];

namespace {
// Device addresses of the arrays, looked up once per device (with that device
// current); host code only sees host-side stand-ins for them.
std::string noalloc_addresses(double2** ws, double** nws) {
    static std::mutex mu;
    static std::map<int, std::pair<double2*, double*>> addr;
    int dev = 0;
    GM_CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    auto it = addr.find(dev);
    if (it == addr.end()) {
        double2* w = nullptr;
        double* nw = nullptr;
        GM_CK(cudaGetSymbolAddress(reinterpret_cast<void**>(&w), g_noalloc_ws));
        GM_CK(cudaGetSymbolAddress(reinterpret_cast<void**>(&nw), g_noalloc_norm));
        it = addr.emplace(dev, std::make_pair(w, nw)).first;
    }
    *ws = it->second.first;
    *nws = it->second.second;
    return {};
}
}  // namespace

std::string noalloc_workspace_prepare() {
    double2* ws = nullptr;
    double* nws = nullptr;
    return noalloc_addresses(&ws, &nws);
}

size_t noalloc_workspace_need(int n, int ncols, int extra) {
    const size_t nchunks = (static_cast<size_t>(n) + kDotChunk - 1) / kDotChunk;
    return static_cast<size_t>(n) * ncols + (4 + extra) * static_cast<size_t>(n) + 2 * static_cast<size_t>(ncols + 1) +
           nchunks * (ncols + 1);
}

std::string Gmres::use_static_workspace(int n, int ncols, int extra) {
    double2* ws = nullptr;
    double* nws = nullptr;
    std::string err = noalloc_addresses(&ws, &nws);
    if (!err.empty()) return err;
    const int nchunks = (n + kDotChunk - 1) / kDotChunk;
    const size_t need = noalloc_workspace_need(n, ncols, extra);
    if (need > kNoAllocWorkspace || nchunks > kNoAllocNorm) {
        // need = n (m + 5 + extra) + (m + 2)(2 + ceil(n / 8192)), m = ncols - 1
        return "size:the solve needs " + std::to_string(need) + " complex values = N x (m + " +
               std::to_string(5 + extra) + ") + (m + 2) x (2 + ceil(N / 8192)) with N = " + std::to_string(n) +
               ", m = " + std::to_string(ncols - 1) +
               " (restart, or max_iter without restart); the fixed workspace holds 2097152";
    }
    if (!external_) release();
    external_ = true;
    n_ = n;
    cap_ = ncols;
    extra_ = extra;
    nchunks_ = nchunks;
    double2* p = ws;
    Q_ = p; p += static_cast<size_t>(n) * ncols;
    w_ = p; p += n;
    b_ = p; p += n;
    x_ = p; p += n;
    r_ = p; p += n;
    h_ = p; p += ncols + 1;
    y_ = p; p += ncols + 1;
    if (extra >= 2) {
        xo_ = p; p += n;
        bo_ = p; p += n;
    } else {
        xo_ = bo_ = nullptr;
    }
    partial_ = p;
    npartial_ = nws;
    return {};
}

std::string Gmres::norm(const double2* v, cudaStream_t s, double* out) {
    k_norm2<<<nchunks_, kDotThreads, 0, s>>>(v, n_, npartial_);
    std::vector<double> p(nchunks_);
    GM_CK(cudaMemcpyAsync(p.data(), npartial_, sizeof(double) * nchunks_, cudaMemcpyDeviceToHost, s));
    GM_CK(cudaStreamSynchronize(s));
    double acc = 0;
    for (double v2 : p) acc += v2;
    *out = std::sqrt(acc);
    return {};
}

// One CGS pass: h (+)= Q_{0..k}^H w ; w -= Q_{0..k} h_pass
std::string Gmres::cgs_pass(int ncols, cudaStream_t s, bool add) {
    dim3 grid(nchunks_, ncols);
    k_multi_dot<<<grid, kDotThreads, 0, s>>>(Q_, n_, ncols, w_, n_, partial_, nchunks_);
    // h_pass -> y_ (scratch), then accumulate into h_
    k_reduce_partials<<<nblk(ncols, 128), 128, 0, s>>>(partial_, nchunks_, ncols, y_, 0);
    k_sub_qh<<<nblk(n_, 256), 256, 0, s>>>(Q_, n_, ncols, y_, w_, n_);
    if (add) {
        k_reduce_partials<<<nblk(ncols, 128), 128, 0, s>>>(partial_, nchunks_, ncols, h_, 1);
    } else {
        GM_CK(cudaMemcpyAsync(h_, y_, sizeof(double2) * ncols, cudaMemcpyDeviceToDevice, s));
    }
    GM_CK(cudaGetLastError());
    return {};
}

// Restarted GMRES(m) on A(prec) x_ = b_ with x_ = 0 on entry (Solver::solve,
// src/solver.cpp:116-146, when restart = 0).  One host synchronisation per
// Arnoldi step: the new Hessenberg column and the norm of the orthogonalised
// vector come back in one copy.
std::string Gmres::cycles(DeviceOp& op, int prec, const SolveOpts& o, double bnorm, double tol_abs, int max_iter,
                          bool refg, int* iters, double* resid, bool* conv) {
    using cd = std::complex<double>;
    const int n = n_;
    const int m = o.restart > 0 ? o.restart : max_iter;
    cudaStream_t s = op.stream();
    std::string err;
    int total = 0;
    bool converged = false;
    double last = 0;
    std::vector<cd> H(static_cast<size_t>(m + 1) * m), cs(m), sn(m), g(m + 1);
    std::vector<double2> hcol(m + 2);
    GM_CK(cudaMemsetAsync(x_, 0, sizeof(double2) * n, s));
    while (total < max_iter && !converged) {
        // r = b - A x  (x = 0 on the first cycle: r = b, as the reference)
        double beta;
        if (total == 0) {
            GM_CK(cudaMemcpyAsync(r_, b_, sizeof(double2) * n, cudaMemcpyDeviceToDevice, s));
            beta = bnorm;
        } else {
            if (pc_) {  // x_ holds u with x = M^{-1} u
                op.bj_apply(x_, tq_, s);
                apply(op, tq_, w_, s, prec);
            } else {
                apply(op, x_, w_, s, prec);
            }
            k_sub<<<nblk(n, 256), 256, 0, s>>>(b_, w_, r_, n);
            err = norm(r_, s, &beta);
            if (!err.empty()) return err;
            if (!std::isfinite(beta)) return "nonfinite:residual";
            if (beta <= tol_abs) { converged = true; last = beta / bnorm; break; }
        }
        k_scale<<<nblk(n, 256), 256, 0, s>>>(r_, make_double2(1.0 / beta, 0.0), Q_, n);
        std::fill(g.begin(), g.end(), cd(0));
        g[0] = beta;
        // Givens rotations of Hessenberg column k (hc[0..k], hc[k+1] = the new
        // vector's norm); true when the cycle ends here.
        auto absorb = [&](int k, std::vector<cd>& hc) -> bool {
            const double hn = std::abs(hc[k + 1]);
            for (int i = 0; i < k; ++i) {
                const cd a = hc[i], b = hc[i + 1];
                if (refg) {
                    hc[i] = cs[i] * a + sn[i] * b;
                    hc[i + 1] = -sn[i] * a + cs[i] * b;
                } else {
                    hc[i] = cs[i] * a + sn[i] * b;
                    hc[i + 1] = -std::conj(sn[i]) * a + cs[i] * b;
                }
            }
            cd c, sgn;
            if (refg) {
                const cd t = std::sqrt(hc[k] * hc[k] + hc[k + 1] * hc[k + 1]);
                c = hc[k] / t;
                sgn = hc[k + 1] / t;
                hc[k] = c * hc[k] + sgn * hc[k + 1];
                g[k + 1] = -sgn * g[k];
                g[k] = c * g[k];
            } else {
                const double az = std::abs(hc[k]);
                const double t = std::sqrt(az * az + std::norm(hc[k + 1]));
                if (az == 0.0) {
                    c = 0.0;
                    sgn = 1.0;
                } else {
                    c = az / t;
                    sgn = (hc[k] / az) * std::conj(hc[k + 1]) / t;
                }
                hc[k] = c * hc[k] + sgn * hc[k + 1];
                g[k + 1] = -std::conj(sgn) * g[k];
                g[k] = c * g[k];
            }
            hc[k + 1] = 0.0;
            cs[k] = c;
            sn[k] = sgn;
            for (int i = 0; i <= k; ++i) H[static_cast<size_t>(k) * (m + 1) + i] = hc[i];
            ++total;
            last = std::abs(g[k + 1]) / bnorm;
            if (!(std::abs(g[k + 1]) > tol_abs) || hn == 0.0) {
                converged = true;
                return true;
            }
            return false;
        };
        int k = 0;
        const bool device_steps = !external_ && st_ && m + 1 <= cap_ && m <= kMaxDeviceSteps;
        if (device_steps) {
            // batches of device-resident steps; the host takes the new columns once per batch
            err = step_graph(op, prec);
            if (!err.empty()) return err;
            GM_CK(cudaMemsetAsync(st_, 0, sizeof(StepStateD), s));
            const int ldh = cap_ + 1;
            std::vector<double2> cols;
            bool stop = false;
            while (!stop && k < m && total < max_iter) {
                const int batch = std::min(kStepBatch, std::min(m - k, max_iter - total));
                for (int b = 0; b < batch; ++b) GM_CK(cudaGraphLaunch(sgx_, s));
                cols.resize(static_cast<size_t>(batch) * ldh);
                GM_CK(cudaMemcpyAsync(cols.data(), hcols_ + static_cast<size_t>(k) * ldh,
                                      sizeof(double2) * cols.size(), cudaMemcpyDeviceToHost, s));
                GM_CK(cudaStreamSynchronize(s));
                for (int b = 0; b < batch && !stop; ++b, ++k) {
                    const double2* col = cols.data() + static_cast<size_t>(b) * ldh;
                    const double hn = std::sqrt(col[k + 1].x);
                    if (!std::isfinite(hn)) return "nonfinite:Arnoldi";
                    std::vector<cd> hc(k + 2);
                    for (int i = 0; i <= k; ++i) hc[i] = cd(col[i].x, col[i].y);
                    hc[k + 1] = hn;
                    stop = absorb(k, hc);
                }
            }
        } else {
            for (; k < m && total < max_iter; ++k) {
                double2* qk = Q_ + static_cast<long long>(k) * n;
                if (pc_) {  // w = A M^{-1} q_k
                    op.bj_apply(qk, tq_, s);
                    apply(op, tq_, w_, s, prec);
                } else {
                    apply(op, qk, w_, s, prec);  // w = A q_k
                }
                err = cgs_pass(k + 1, s, false);
                if (!err.empty()) return err;
                err = cgs_pass(k + 1, s, true);
                if (!err.empty()) return err;
                // ||w||^2 into h_[k+1].x, then h_[0..k+1] to the host in one copy.
                k_norm2<<<nchunks_, kDotThreads, 0, s>>>(w_, n, npartial_);
                k_sum_into<<<1, 1, 0, s>>>(npartial_, nchunks_, h_ + k + 1);
                GM_CK(cudaMemcpyAsync(hcol.data(), h_, sizeof(double2) * (k + 2), cudaMemcpyDeviceToHost, s));
                GM_CK(cudaStreamSynchronize(s));
                const double hn = std::sqrt(hcol[k + 1].x);
                if (!std::isfinite(hn)) return "nonfinite:Arnoldi";
                std::vector<cd> hc(k + 2);
                for (int i = 0; i <= k; ++i) hc[i] = cd(hcol[i].x, hcol[i].y);
                hc[k + 1] = hn;
                if (hn > 0) {
                    double2* qn = Q_ + static_cast<long long>(k + 1) * n;
                    k_scale<<<nblk(n, 256), 256, 0, s>>>(w_, make_double2(1.0 / hn, 0.0), qn, n);
                }
                if (absorb(k, hc)) {
                    ++k;
                    break;
                }
            }
        }
        // Solve the k x k upper-triangular system R y = g (solver.cpp:143-145).
        std::vector<cd> yv(k);
        for (int i = k - 1; i >= 0; --i) {
            cd acc = g[i];
            for (int j = i + 1; j < k; ++j) acc -= H[static_cast<size_t>(j) * (m + 1) + i] * yv[j];
            yv[i] = acc / H[static_cast<size_t>(i) * (m + 1) + i];
        }
        std::vector<double2> yd(k);
        for (int i = 0; i < k; ++i) yd[i] = make_double2(-yv[i].real(), -yv[i].imag());
        GM_CK(cudaMemcpyAsync(y_, yd.data(), sizeof(double2) * k, cudaMemcpyHostToDevice, s));
        // x -= Q (-y)  ==  x += Q y
        k_sub_qh<<<nblk(n, 256), 256, 0, s>>>(Q_, n, k, y_, x_, n);
        GM_CK(cudaStreamSynchronize(s));
        if (o.restart <= 0) break;  // unrestarted: one cycle (the reference)
    }
    if (pc_) {  // back from the preconditioned space: x = M^{-1} u
        op.bj_apply(x_, tq_, s);
        GM_CK(cudaMemcpyAsync(x_, tq_, sizeof(double2) * n, cudaMemcpyDeviceToDevice, s));
        GM_CK(cudaStreamSynchronize(s));
    }
    *iters = total;
    *resid = last;
    *conv = converged;
    return {};
}

std::string Gmres::solve(DeviceOp& op, const double2* d_b_user, double2* d_x_user, const SolveOpts& o,
                         SolveResult* res) {
    if (o.adjoint && op.ref_compat()) return "arg:the adjoint needs ref_compat = 0";
    adj_ = o.adjoint != 0;
    pc_ = o.precond != 0;
    if (o.inner) {
        if (!o.flexible) return "arg:an inner operator serves the flexible solve";
        if (adj_) return "arg:the flexible solve with an inner operator serves forward solves";
        if (o.inner->n() != op.n()) return "arg:the inner operator has another number of unknowns";
    }
    if (pc_) {
        if (adj_) return "arg:the block-Jacobi preconditioner serves forward solves";
        if (external_) return "arg:the preconditioned solve needs its own workspace (use mlfma_gmres)";
        const std::string e = (o.inner ? *o.inner : op).bj_prepare();
        if (!e.empty()) return e;
    }
    if (o.flexible) {
        if (external_) return "arg:the flexible solve needs its own workspace (use mlfma_gmres)";
        return solve_flexible(op, d_b_user, d_x_user, o, res);
    }
    if (o.refine && op.precision() != kFp64) return solve_refined(op, d_b_user, d_x_user, o, res);
    const auto t_start = std::chrono::steady_clock::now();
    const int n = op.n();
    const int m = o.restart > 0 ? o.restart : o.max_iter;
    if (m < 1 || o.max_iter < 1) return "max_iter and restart must be positive";
    std::string err = ensure(n, m + 1, 0);
    if (!err.empty()) return err;
    cudaStream_t s = op.stream();
    const int* perm = op.perm();
    k_gather_perm<<<nblk(n, 256), 256, 0, s>>>(d_b_user, perm, b_, n);
    double bnorm = 0;
    err = norm(b_, s, &bnorm);
    if (!err.empty()) return err;
    if (!std::isfinite(bnorm)) return "nonfinite:right-hand side";
    res->iterations = 0;
    res->residual = 0;
    if (bnorm == 0.0) {
        GM_CK(cudaMemsetAsync(d_x_user, 0, sizeof(double2) * n, s));
        GM_CK(cudaStreamSynchronize(s));
        res->true_residual = 0;
        res->converged = true;
        return {};
    }
    bool converged = false;
    err = cycles(op, -1, o, bnorm, o.tol * bnorm, o.max_iter, o.ref_givens != 0, &res->iterations, &res->residual,
                 &converged);
    if (!err.empty()) return err;
    // True residual.
    apply(op, x_, w_, s);
    k_sub<<<nblk(n, 256), 256, 0, s>>>(b_, w_, r_, n);
    double rn;
    err = norm(r_, s, &rn);
    if (!err.empty()) return err;
    res->true_residual = rn / bnorm;
    k_scatter_perm<<<nblk(n, 256), 256, 0, s>>>(x_, perm, d_x_user, n);
    GM_CK(cudaStreamSynchronize(s));
    res->converged = converged;
    res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    return {};
}

// Mixed-precision iterative refinement: the outer loop keeps the solution and
// its residual r = b - A x in FP64 (FP64 far field); each inner solve runs
// GMRES on the mixed operator for the correction d in A d = r, to a residual
// target of 0.9 of the remaining gap, and x += d.  The mixed far field differs
// from the FP64 one by float rounding (about 1e-8 relative on the product),
// so one inner solve normally reaches the target and the FP64 residual only
// confirms it.
std::string Gmres::solve_refined(DeviceOp& op, const double2* d_b_user, double2* d_x_user, const SolveOpts& o,
                                 SolveResult* res) {
    const auto t_start = std::chrono::steady_clock::now();
    const int n = op.n();
    const int m = o.restart > 0 ? o.restart : o.max_iter;
    if (m < 1 || o.max_iter < 1) return "max_iter and restart must be positive";
    std::string err = ensure(n, m + 1, 2);
    if (!err.empty()) return err;
    cudaStream_t s = op.stream();
    const int* perm = op.perm();
    k_gather_perm<<<nblk(n, 256), 256, 0, s>>>(d_b_user, perm, bo_, n);
    GM_CK(cudaMemsetAsync(xo_, 0, sizeof(double2) * n, s));
    double bnorm = 0;
    err = norm(bo_, s, &bnorm);
    if (!err.empty()) return err;
    if (!std::isfinite(bnorm)) return "nonfinite:right-hand side";
    *res = SolveResult{};
    if (bnorm == 0.0) {
        GM_CK(cudaMemsetAsync(d_x_user, 0, sizeof(double2) * n, s));
        GM_CK(cudaStreamSynchronize(s));
        res->converged = true;
        return {};
    }
    GM_CK(cudaMemcpyAsync(b_, bo_, sizeof(double2) * n, cudaMemcpyDeviceToDevice, s));
    double rn = bnorm;
    bool converged = false;
    const int kMaxOuter = 20;
    while (res->iterations < o.max_iter && res->refinements < kMaxOuter) {
        // Inner target: residual of the correction system at most eta * ||r||;
        // the mixed product is within about 1e-8 of the FP64 one, so aiming at
        // 0.9 of the gap normally lands under tol on the FP64 residual.
        double eta = o.inner_tol > 0 ? o.inner_tol : 0.9 * o.tol * bnorm / rn;
        eta = std::min(eta, 0.5);
        int it = 0;
        double est = 0;
        bool c = false;
        err = cycles(op, kMixed, o, rn, eta * rn, o.max_iter - res->iterations, false, &it, &est, &c);
        if (!err.empty()) return err;
        res->iterations += it;
        // x += d ; r = b - A64 x  (FP64)
        k_axpy1<<<nblk(n, 256), 256, 0, s>>>(x_, xo_, n);
        apply(op, xo_, w_, s, kFp64);
        k_sub<<<nblk(n, 256), 256, 0, s>>>(bo_, w_, b_, n);
        ++res->refinements;
        err = norm(b_, s, &rn);
        if (!err.empty()) return err;
        if (!std::isfinite(rn)) return "nonfinite:residual";
        res->residual = rn / bnorm;
        if (rn <= o.tol * bnorm) { converged = true; break; }
        if (it == 0) break;  // no progress possible
    }
    res->true_residual = rn / bnorm;
    k_scatter_perm<<<nblk(n, 256), 256, 0, s>>>(xo_, perm, d_x_user, n);
    GM_CK(cudaStreamSynchronize(s));
    res->converged = converged;
    res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    return {};
}

// Flexible GMRES (FGMRES(m), right preconditioning that may change at every
// step): the outer Krylov space, its products, the Hessenberg matrix, the
// unitary Givens rotations and the residual are FP64; the preconditioner of
// outer step j is an inner GMRES of `inner_iters` iterations from zero on
// A z = v_j on the operator's own far field (complex float on a mixed
// operator), so every inner solve's result z_j enters the solution
// x = x0 + Z y exactly, and the inner precision only changes how good a
// preconditioner it is.  The outer space keeps what restarted GMRES(m) throws
// away at each restart; the stopping test is the FP64 residual.
std::string Gmres::solve_flexible(DeviceOp& op, const double2* d_b_user, double2* d_x_user, const SolveOpts& o,
                                  SolveResult* res) {
    using cd = std::complex<double>;
    const auto t_start = std::chrono::steady_clock::now();
    const int n = op.n();
    const int mo = o.restart > 0 ? o.restart : o.max_iter;
    const int mi = o.inner_iters > 0 ? o.inner_iters : 20;
    if (mo < 1 || o.max_iter < 1) return "max_iter and restart must be positive";
    std::string err = ensure(n, mi + 1, 0);
    if (!err.empty()) return err;
    err = ensure_outer(n, mo);
    if (!err.empty()) return err;
    cudaStream_t s = op.stream();
    const int* perm = op.perm();
    const int nch = nchunks_;
    // inner solves: on the inner operator when one is given (its own stream;
    // the two streams meet at host synchronisations around each inner solve)
    DeviceOp& iop = o.inner ? *o.inner : op;
    const bool two_streams = iop.stream() != op.stream();
    const int prec_in = iop.precision();
    k_gather_perm<<<nblk(n, 256), 256, 0, s>>>(d_b_user, perm, bf_, n);
    GM_CK(cudaMemsetAsync(xf_, 0, sizeof(double2) * n, s));
    double bnorm = 0;
    err = norm(bf_, s, &bnorm);
    if (!err.empty()) return err;
    if (!std::isfinite(bnorm)) return "nonfinite:right-hand side";
    *res = SolveResult{};
    if (bnorm == 0.0) {
        GM_CK(cudaMemsetAsync(d_x_user, 0, sizeof(double2) * n, s));
        GM_CK(cudaStreamSynchronize(s));
        res->converged = true;
        return {};
    }
    const double tol_abs = o.tol * bnorm;
    // CGS2 of w against the first ncols outer basis vectors: h (device) = V^H w
    // summed over both passes, w orthogonalised in place.
    auto cgs2 = [&](int ncols) {
        const dim3 grid(nch, ncols);
        for (int pass = 0; pass < 2; ++pass) {
            k_multi_dot<<<grid, kDotThreads, 0, s>>>(V_, n, ncols, wo_, n, po_, nch);
            k_reduce_partials<<<nblk(ncols, 128), 128, 0, s>>>(po_, nch, ncols, to_, 0);
            k_sub_qh<<<nblk(n, 256), 256, 0, s>>>(V_, n, ncols, to_, wo_, n);
            k_reduce_partials<<<nblk(ncols, 128), 128, 0, s>>>(po_, nch, ncols, ho_, pass);
        }
    };
    std::vector<cd> H(static_cast<size_t>(mo + 1) * mo), cs(mo), sn(mo), g(mo + 1);
    std::vector<double2> hcol(mo + 2);
    double beta = bnorm;
    bool converged = false;
    SolveOpts oi = o;
    oi.restart = mi;
    oi.flexible = 0;
    GM_CK(cudaMemcpyAsync(r_, bf_, sizeof(double2) * n, cudaMemcpyDeviceToDevice, s));  // r = b (x = 0)
    while (res->iterations < o.max_iter && !converged) {
        k_scale<<<nblk(n, 256), 256, 0, s>>>(r_, make_double2(1.0 / beta, 0.0), V_, n);
        std::fill(g.begin(), g.end(), cd(0));
        g[0] = beta;
        int k = 0;
        for (; k < mo && res->iterations < o.max_iter; ++k) {
            double2* vk = V_ + static_cast<size_t>(k) * n;
            double2* zk = Z_ + static_cast<size_t>(k) * n;
            // inner solve A z = v_k from zero (||v_k|| = 1)
            GM_CK(cudaMemcpyAsync(b_, vk, sizeof(double2) * n, cudaMemcpyDeviceToDevice, s));
            if (two_streams) GM_CK(cudaStreamSynchronize(s));
            int it = 0;
            double est = 0;
            bool c = false;
            err = cycles(iop, prec_in, oi, 1.0, o.inner_tol > 0 ? o.inner_tol : 0.0,
                         std::min(mi, o.max_iter - res->iterations), false, &it, &est, &c);
            if (!err.empty()) return err;
            if (two_streams) GM_CK(cudaStreamSynchronize(iop.stream()));
            res->iterations += it;
            GM_CK(cudaMemcpyAsync(zk, x_, sizeof(double2) * n, cudaMemcpyDeviceToDevice, s));
            // w = A z_k in FP64, orthogonalised against v_0..v_k
            apply(op, zk, wo_, s, kFp64);
            ++res->refinements;
            cgs2(k + 1);
            k_norm2<<<nch, kDotThreads, 0, s>>>(wo_, n, npartial_);
            k_sum_into<<<1, 1, 0, s>>>(npartial_, nch, ho_ + k + 1);
            GM_CK(cudaMemcpyAsync(hcol.data(), ho_, sizeof(double2) * (k + 2), cudaMemcpyDeviceToHost, s));
            GM_CK(cudaStreamSynchronize(s));
            const double hn = std::sqrt(hcol[k + 1].x);
            if (!std::isfinite(hn)) return "nonfinite:Arnoldi";
            std::vector<cd> hc(k + 2);
            for (int i = 0; i <= k; ++i) hc[i] = cd(hcol[i].x, hcol[i].y);
            hc[k + 1] = hn;
            if (hn > 0)
                k_scale<<<nblk(n, 256), 256, 0, s>>>(wo_, make_double2(1.0 / hn, 0.0), V_ + static_cast<size_t>(k + 1) * n, n);
            for (int i = 0; i < k; ++i) {  // previous unitary rotations
                const cd a = hc[i], b = hc[i + 1];
                hc[i] = cs[i] * a + sn[i] * b;
                hc[i + 1] = -std::conj(sn[i]) * a + cs[i] * b;
            }
            const double az = std::abs(hc[k]);
            const double t = std::sqrt(az * az + std::norm(hc[k + 1]));
            cd cr, sr;
            if (az == 0.0) {
                cr = 0.0;
                sr = 1.0;
            } else {
                cr = az / t;
                sr = (hc[k] / az) * std::conj(hc[k + 1]) / t;
            }
            hc[k] = cr * hc[k] + sr * hc[k + 1];
            g[k + 1] = -std::conj(sr) * g[k];
            g[k] = cr * g[k];
            cs[k] = cr;
            sn[k] = sr;
            for (int i = 0; i <= k; ++i) H[static_cast<size_t>(k) * (mo + 1) + i] = hc[i];
            res->residual = std::abs(g[k + 1]) / bnorm;
            if (!(std::abs(g[k + 1]) > tol_abs) || hn == 0.0) {
                ++k;
                break;
            }
        }
        // x += Z y, R y = g
        std::vector<cd> yv(k);
        for (int i = k - 1; i >= 0; --i) {
            cd acc = g[i];
            for (int j = i + 1; j < k; ++j) acc -= H[static_cast<size_t>(j) * (mo + 1) + i] * yv[j];
            yv[i] = acc / H[static_cast<size_t>(i) * (mo + 1) + i];
        }
        std::vector<double2> yd(k);
        for (int i = 0; i < k; ++i) yd[i] = make_double2(-yv[i].real(), -yv[i].imag());
        GM_CK(cudaMemcpyAsync(to_, yd.data(), sizeof(double2) * k, cudaMemcpyHostToDevice, s));
        k_sub_qh<<<nblk(n, 256), 256, 0, s>>>(Z_, n, k, to_, xf_, n);
        // true FP64 residual
        apply(op, xf_, wo_, s, kFp64);
        k_sub<<<nblk(n, 256), 256, 0, s>>>(bf_, wo_, r_, n);
        err = norm(r_, s, &beta);
        if (!err.empty()) return err;
        if (!std::isfinite(beta)) return "nonfinite:residual";
        res->true_residual = beta / bnorm;
        if (beta <= tol_abs) converged = true;
    }
    k_scatter_perm<<<nblk(n, 256), 256, 0, s>>>(xf_, perm, d_x_user, n);
    GM_CK(cudaStreamSynchronize(s));
    res->converged = converged;
    res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    return {};
}

}  // namespace mlfma
