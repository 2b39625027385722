// Many independent operators of uneven size (mlfma_batch_*): one CUDA graph
// holds every operator's product as a parallel branch, so a single graph
// launch applies all of them; solves run every operator's GMRES at once, one
// host thread per operator, each on its operator's own streams.  No
// counterpart in the reference (one problem per process there).
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mlfma_b200.h"
#include "device.cuh"

// Defined in capi.cu.
mlfma::DeviceOp* mlfma_internal_device(mlfma_handle h);
int mlfma_internal_fail(int code, const std::string& msg);
int mlfma_internal_device_ordinal(mlfma_handle h);

struct mlfma_batch_s {
    std::vector<mlfma_handle> ops;
    std::vector<long long> off;  // start of each operator's vector in the packed layout
    long long total = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    double2* d_x = nullptr;
    double2* d_y = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~mlfma_batch_s() {
        cudaSetDevice(device);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (d_x) cudaFree(d_x);
        if (d_y) cudaFree(d_y);
        if (fork) cudaEventDestroy(fork);
        for (cudaEvent_t e : join)
            if (e) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

#define B_CK(call)                                                                                          \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess)                                                                              \
            return mlfma_internal_fail(MLFMA_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Records every operator's product, reading d_x and writing d_y (packed), as
// parallel branches forked from and joined back into b->stream.
int capture(mlfma_batch_s* b) {
    B_CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaEventRecord(b->fork, b->stream);
    for (size_t i = 0; i < b->ops.size(); ++i) {
        mlfma::DeviceOp* d = mlfma_internal_device(b->ops[i]);
        cudaStreamWaitEvent(d->stream(), b->fork, 0);
        d->enqueue_matvec(b->d_x + b->off[i], b->d_y + b->off[i], d->stream());
        cudaEventRecord(b->join[i], d->stream());
        cudaStreamWaitEvent(b->stream, b->join[i], 0);
        cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(b->stream, &st);
        if (st != cudaStreamCaptureStatusActive) {
            const cudaError_t le = cudaGetLastError();
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(b->stream, &g);
            if (g) cudaGraphDestroy(g);
            return mlfma_internal_fail(MLFMA_ERR_CUDA, "capture of operator " + std::to_string(i) +
                                                           " failed: " + cudaGetErrorString(le));
        }
    }
    B_CK(cudaStreamEndCapture(b->stream, &b->graph));
    B_CK(cudaGraphInstantiate(&b->exec, b->graph, cudaGraphInstantiateFlagUseNodePriority));
    return MLFMA_OK;
}

}  // namespace

extern "C" {

int mlfma_batch_create(int nops, const mlfma_handle* ops, mlfma_batch* out) {
    if (nops < 1 || !ops || !out) return mlfma_internal_fail(MLFMA_ERR_ARG, "null argument or nops < 1");
    auto b = std::make_unique<mlfma_batch_s>();
    for (int i = 0; i < nops; ++i) {
        if (!ops[i] || !mlfma_internal_device(ops[i])) return mlfma_internal_fail(MLFMA_ERR_STATE, "operator not set up");
        for (int j = 0; j < i; ++j)
            if (ops[j] == ops[i]) return mlfma_internal_fail(MLFMA_ERR_ARG, "an operator appears twice in the batch");
        const int dev = mlfma_internal_device_ordinal(ops[i]);
        if (i == 0) b->device = dev;
        if (dev != b->device) return mlfma_internal_fail(MLFMA_ERR_ARG, "operators on different devices");
        b->ops.push_back(ops[i]);
        b->off.push_back(b->total);
        b->total += mlfma_internal_device(ops[i])->n();
    }
    B_CK(cudaSetDevice(b->device));
    B_CK(cudaDeviceSynchronize());  // every operator idle before its streams join the capture
    B_CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    B_CK(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    b->join.assign(b->ops.size(), nullptr);
    for (auto& e : b->join) B_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    B_CK(cudaMalloc(&b->d_x, sizeof(double2) * b->total));
    B_CK(cudaMalloc(&b->d_y, sizeof(double2) * b->total));
    const int code = capture(b.get());
    if (code != MLFMA_OK) return code;
    *out = b.release();
    return MLFMA_OK;
}

int mlfma_batch_size(mlfma_batch b, long long* total) {
    if (!b || !total) return mlfma_internal_fail(MLFMA_ERR_ARG, "null argument");
    *total = b->total;
    return MLFMA_OK;
}

int mlfma_batch_matvec_device(mlfma_batch b, const void* d_x, void* d_y, void* stream) {
    if (!b || !d_x || !d_y) return mlfma_internal_fail(MLFMA_ERR_ARG, "null argument");
    B_CK(cudaSetDevice(b->device));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : b->stream;
    const size_t bytes = sizeof(double2) * b->total;
    B_CK(cudaMemcpyAsync(b->d_x, d_x, bytes, cudaMemcpyDeviceToDevice, s));
    B_CK(cudaGraphLaunch(b->exec, s));
    B_CK(cudaMemcpyAsync(d_y, b->d_y, bytes, cudaMemcpyDeviceToDevice, s));
    return MLFMA_OK;
}

int mlfma_batch_matvec(mlfma_batch b, const double* x, double* y) {
    if (!b || !x || !y) return mlfma_internal_fail(MLFMA_ERR_ARG, "null argument");
    B_CK(cudaSetDevice(b->device));
    const size_t bytes = sizeof(double2) * b->total;
    B_CK(cudaMemcpyAsync(b->d_x, x, bytes, cudaMemcpyHostToDevice, b->stream));
    B_CK(cudaGraphLaunch(b->exec, b->stream));
    B_CK(cudaMemcpyAsync(y, b->d_y, bytes, cudaMemcpyDeviceToHost, b->stream));
    B_CK(cudaStreamSynchronize(b->stream));
    return MLFMA_OK;
}

int mlfma_batch_gmres(mlfma_batch b, const double* rhs, double* x, const mlfma_solver_opts* opts,
                      mlfma_solve_info* info) {
    if (!b || !rhs || !x) return mlfma_internal_fail(MLFMA_ERR_ARG, "null argument");
    const size_t n = b->ops.size();
    std::vector<int> codes(n, MLFMA_OK);
    std::vector<std::string> msgs(n);
    std::vector<std::thread> th;
    for (size_t i = 0; i < n; ++i)
        th.emplace_back([&, i] {
            const long long o = b->off[i];
            codes[i] = mlfma_gmres(b->ops[i], rhs + 2 * o, x + 2 * o, opts, info ? info + i : nullptr);
            if (codes[i] != MLFMA_OK) msgs[i] = mlfma_last_error();
        });
    for (auto& t : th) t.join();
    int worst = MLFMA_OK;
    std::string msg;
    for (size_t i = 0; i < n; ++i)
        if (codes[i] != MLFMA_OK && (worst == MLFMA_OK || worst == MLFMA_ERR_NOT_CONVERGED)) {
            worst = codes[i];
            msg = "operator " + std::to_string(i) + ": " + msgs[i];
        }
    if (worst != MLFMA_OK) return mlfma_internal_fail(worst, msg);
    return MLFMA_OK;
}

int mlfma_batch_destroy(mlfma_batch b) {
    delete b;
    return MLFMA_OK;
}

}  // extern "C"
