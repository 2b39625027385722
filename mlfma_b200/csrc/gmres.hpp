// Device GMRES driver (see gmres.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "device.cuh"

namespace mlfma {

struct SolveOpts {
    int max_iter = 500;
    double tol = 1e-6;
    int restart = 0;     // 0: no restart (reference)
    int ref_givens = 1;  // complex-symmetric rotations of the reference
    int refine = 0;      // mixed operator: inner GMRES on the mixed far field,
                         // outer loop on the FP64 residual
    double inner_tol = 0;  // refinement: inner relative target (0 = automatic)
    int adjoint = 0;       // solve A^H x = b (operator set up with ref_compat = 0)
    int flexible = 0;      // FGMRES: FP64 outer Krylov space over inner GMRES solves
    int inner_iters = 0;   // flexible: iterations per inner solve (0 = 20)
    int precond = 0;       // 1: leaf block-Jacobi right preconditioner (DeviceOp::bj_*)
    DeviceOp* inner = nullptr;  // flexible: operator of the inner solves (same
                                // unknowns and source order), null = the outer one
};

struct SolveResult {
    int iterations = 0;
    double residual = 0;
    double true_residual = 0;
    double seconds = 0;
    bool converged = false;
    int refinements = 0;   // outer FP64 residual evaluations (refinement only)
};

class Gmres {
public:
    Gmres() = default;
    ~Gmres();
    Gmres(const Gmres&) = delete;
    Gmres& operator=(const Gmres&) = delete;

    // b and x are device vectors in the caller's source order.
    std::string solve(DeviceOp& op, const double2* d_b_user, double2* d_x_user, const SolveOpts& o,
                      SolveResult* res);

    // Point this solver at the library's fixed device workspace instead of
    // allocating (see mlfma_gmres_noalloc); products then run without graph
    // capture.  Fails if n and ncols do not fit.
    // extra = 2 reserves the two vectors of iterative refinement.
    std::string use_static_workspace(int n, int ncols, int extra = 0);

private:
    void apply(DeviceOp& op, const double2* x, double2* y, cudaStream_t s, int prec = -1);
    // Restarted GMRES on A(prec) x_ = b_ from x_ = 0 until the estimated
    // residual norm is at most tol_abs or max_iter iterations have run.
    std::string cycles(DeviceOp& op, int prec, const SolveOpts& o, double bnorm, double tol_abs, int max_iter,
                       bool refg, int* iters, double* resid, bool* conv);
    std::string solve_refined(DeviceOp& op, const double2* d_b_user, double2* d_x_user, const SolveOpts& o,
                              SolveResult* res);
    std::string solve_flexible(DeviceOp& op, const double2* d_b_user, double2* d_x_user, const SolveOpts& o,
                               SolveResult* res);
    std::string ensure_outer(int n, int ncols);
    void release_outer();
    bool external_ = false;   // workspace not owned (static device array)
    bool adj_ = false;        // products with A^H (SolveOpts::adjoint)
    std::string ensure(int n, int ncols, int extra);
    void release();
    std::string norm(const double2* v, cudaStream_t s, double* out);
    std::string cgs_pass(int ncols, cudaStream_t s, bool add);

    // Device-resident Arnoldi steps (allocated workspace, restart <= kMaxDeviceSteps):
    // one step = a captured graph (next basis vector, product, CGS2, norm)
    // that reads the step index from device memory; the host takes the new
    // Hessenberg columns once per batch of steps.
    std::string step_graph(DeviceOp& op, int prec);
    void release_steps();
    void* st_ = nullptr;         // step index, block counter, last norm (device)
    double2* hcols_ = nullptr;   // [cap_][cap_ + 1]: Hessenberg column k at k (cap_ + 1)
    double2* tco_ = nullptr;     // [cap_]: coefficients of the current CGS pass
    double* npart2_ = nullptr;   // norm partials, one per update block
    double2* spartial_ = nullptr;  // dot partials of the device steps, [columns][nstep_]
    int nstep_ = 0;                // their chunks of the vector
    double* swnorm_ = nullptr;     // ||w||^2 partials of the device steps, [nstep_]
    cudaGraph_t sg_ = nullptr;
    cudaGraphExec_t sgx_ = nullptr;
    const DeviceOp* sg_op_ = nullptr;
    int sg_prec_ = -1, sg_adj_ = -1, sg_gen_ = -1, sg_pc_ = -1;
    bool pc_ = false;            // right preconditioning in this solve
    double2* tq_ = nullptr;      // preconditioner scratch vector
    const double2* sg_q_ = nullptr;

    int n_ = 0, cap_ = 0, extra_ = 0, nchunks_ = 0;
    double2* Q_ = nullptr;
    double2* w_ = nullptr;
    double2* b_ = nullptr;
    double2* x_ = nullptr;
    double2* r_ = nullptr;
    double2* h_ = nullptr;
    double2* y_ = nullptr;
    double2* partial_ = nullptr;
    double* npartial_ = nullptr;
    double2* xo_ = nullptr;   // refinement: accumulated solution
    double2* bo_ = nullptr;   // refinement: right-hand side
    // Flexible GMRES: outer basis V (ncols + 1), preconditioned directions Z
    // (ncols), outer work vector, Hessenberg column and dot partials.
    int on_ = 0, ocap_ = 0;
    double2 *V_ = nullptr, *Z_ = nullptr, *wo_ = nullptr, *ho_ = nullptr, *to_ = nullptr, *po_ = nullptr;
    double2 *xf_ = nullptr, *bf_ = nullptr;
};

// The fixed workspace of Gmres::use_static_workspace: makes sure it exists on
// the current device (CUDA creates a module's device arrays when the module is
// first used on a device) and looks up its address; mlfma_setup calls it.
std::string noalloc_workspace_prepare();
// Complex values the fixed workspace must hold for a solve of n unknowns with
// ncols basis vectors (restart + 1) and `extra` refinement vectors.
size_t noalloc_workspace_need(int n, int ncols, int extra);

// GMRES on nr right-hand sides sharing every product (gmres_multi.cu).
class GmresMulti {
public:
    GmresMulti() = default;
    ~GmresMulti();
    GmresMulti(const GmresMulti&) = delete;
    GmresMulti& operator=(const GmresMulti&) = delete;

    // b and x: nr device vectors one after another, caller order ([nr][n]).
    // Unitary Givens rotations (ref_givens is ignored); restart as in Gmres;
    // refine on a mixed operator: FP64 outer residual, mixed inner solves.
    std::string solve(DeviceOp& op, int nr, const double2* d_b_user, double2* d_x_user, const SolveOpts& o,
                      std::vector<SolveResult>& res);

private:
    // opts.flexible: FGMRES(restart) per column, FP64 outer spaces, each outer
    // step's inner solves run together (inner_iters GMRES iterations on the
    // operator's own far field, complex float on a mixed operator).
    std::string solve_flexible(DeviceOp& op, int nr, const double2* d_b_user, double2* d_x_user, const SolveOpts& o,
                               std::vector<SolveResult>& res);
    void cgs_pass_q(const double2* Q, double2* w, int ncols, cudaStream_t s, double2* h, bool add);
    std::string ensure(int n, int nr, int ncols);
    void release();
    std::string norms(const double2* v, cudaStream_t s, std::vector<double>& out);
    void cgs_pass(int ncols, cudaStream_t s, bool add);
    std::string cycles(DeviceOp& op, int prec, int restart, int max_iter, const std::vector<double>& bnorm,
                       const std::vector<double>& tol_abs, std::vector<char>& done, std::vector<int>& iters,
                       std::vector<double>& est);

    int n_ = 0, nr_ = 0, cap_ = 0, nchunks_ = 0;
    double2 *Q_ = nullptr, *w_ = nullptr, *b_ = nullptr, *x_ = nullptr, *r_ = nullptr;
    double2 *h_ = nullptr, *y_ = nullptr, *partial_ = nullptr, *xo_ = nullptr, *bo_ = nullptr;
    double *npartial_ = nullptr, *scale_ = nullptr;
    double2 *V_ = nullptr, *Z_ = nullptr;  // flexible: outer bases ([mo + 1] and [mo] vectors of [n][nr])
    int vcap_ = 0;                         // their capacity (outer steps)
};

}  // namespace mlfma
