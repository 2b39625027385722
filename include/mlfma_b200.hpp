// C++ wrapper over the C ABI (mlfma_b200.h) with the reference's entry-point
// names, for host code that drove the reference's FMM::Node / Solver protocol.
//
//   reference (ellilu11/MLFMA)                     this wrapper
//   Node::initStatic + root ctor + buildLists      mlfma_b200::Operator::dipoles / rwg
//     + Node::buildTables (src/mlfma.cpp:21-55)
//   Leaf::buildNearRads + resizeCoeffs             Operator::setup()
//     + Leaf::buildRadPats (src/mlfma.cpp:42-62)
//   Solver::evalRvec: rvec += A lvec               Operator::evalRvec(lvec, rvec)
//     (src/solver.cpp:41-57)
//   Solver(srcs, root, maxIter, EPS, ...).solve()  Solver(op, maxIter, EPS).solve()
//     (src/solver.cpp:5-146)
//
// Errors become std::runtime_error carrying the ABI's message, like the
// reference's own std::runtime_error on bad input (src/fileio.h).
#pragma once

#include <complex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "mlfma_b200.h"

namespace mlfma_b200 {

using cplx = std::complex<double>;

inline void check(int code) {
    if (code != MLFMA_OK) throw std::runtime_error(std::string("mlfma_b200: ") + mlfma_last_error());
}

class Operator {
public:
    static Operator dipoles(const mlfma_config& cfg, const mlfma_planewave& pw, const std::vector<double>& pos,
                            const std::vector<double>& mom) {
        mlfma_handle h = nullptr;
        check(mlfma_create_dipoles(&cfg, &pw, static_cast<int>(pos.size() / 3), pos.data(), mom.data(), &h));
        return Operator(h);
    }
    static Operator rwg(const mlfma_config& cfg, const mlfma_planewave& pw, const std::vector<double>& verts,
                        const std::vector<int>& faces, const std::vector<int>& rwgs) {
        mlfma_handle h = nullptr;
        check(mlfma_create_rwg(&cfg, &pw, static_cast<int>(verts.size() / 3), verts.data(),
                               static_cast<int>(faces.size() / 3), faces.data(), static_cast<int>(rwgs.size() / 4),
                               rwgs.data(), &h));
        return Operator(h);
    }
    Operator(Operator&& o) noexcept : h_(std::exchange(o.h_, nullptr)) {}
    Operator& operator=(Operator&& o) noexcept {
        if (this != &o) {
            if (h_) mlfma_destroy(h_);
            h_ = std::exchange(o.h_, nullptr);
        }
        return *this;
    }
    Operator(const Operator&) = delete;
    Operator& operator=(const Operator&) = delete;
    ~Operator() {
        if (h_) mlfma_destroy(h_);
    }

    void setup() { check(mlfma_setup(h_)); }

    int numSrcs() const {
        int n = 0;
        check(mlfma_num_unknowns(h_, &n));
        return n;
    }

    // -V, the reference's initial lvec (src/solver.cpp:31-32).
    std::vector<cplx> rhs() const {
        std::vector<cplx> b(numSrcs());
        check(mlfma_rhs(h_, reinterpret_cast<double*>(b.data())));
        return b;
    }

    // rvec += A lvec, as Solver::evalRvec does.
    void evalRvec(const std::vector<cplx>& lvec, std::vector<cplx>& rvec) {
        check(mlfma_matvec(h_, reinterpret_cast<const double*>(lvec.data()), reinterpret_cast<double*>(rvec.data()), 1));
    }

    // Many right-hand sides at once: Y = A X for the rows of X (nrhs x n).
    std::vector<cplx> evalRvecMulti(int nrhs, const std::vector<cplx>& X) {
        std::vector<cplx> Y(X.size());
        check(mlfma_matvec_multi(h_, nrhs, reinterpret_cast<const double*>(X.data()),
                                 reinterpret_cast<double*>(Y.data()), 0));
        return Y;
    }

    // -V for another incident plane wave of the same wavenumber.
    std::vector<cplx> rhs(const mlfma_planewave& pw) const {
        std::vector<cplx> b(numSrcs());
        check(mlfma_rhs_planewave(h_, &pw, reinterpret_cast<double*>(b.data())));
        return b;
    }

    // y = A^H x (operators set up with ref_compat = 0).
    std::vector<cplx> evalAdjoint(const std::vector<cplx>& x) {
        std::vector<cplx> y(x.size());
        check(mlfma_matvec_adjoint(h_, reinterpret_cast<const double*>(x.data()), reinterpret_cast<double*>(y.data()), 0));
        return y;
    }

    // Diagonal impedance loads z (n complex) added to the operator.
    void setLoads(const std::vector<cplx>& z) { check(mlfma_set_loads(h_, reinterpret_cast<const double*>(z.data()))); }

    // (A x)[rows] with every interaction evaluated directly in FP64: the dense
    // reference for sampled rows (rows: caller-order indices).
    std::vector<cplx> denseRows(const std::vector<int>& rows, const std::vector<cplx>& x) {
        std::vector<cplx> y(rows.size());
        check(mlfma_dense_rows(h_, static_cast<int>(rows.size()), rows.data(), reinterpret_cast<const double*>(x.data()),
                               reinterpret_cast<double*>(y.data())));
        return y;
    }

    // Launch shapes timed on this operator (nrhs = 1: one-vector product).
    mlfma_tuning autotune(int nrhs = 1, int reps = 5) {
        mlfma_tuning t{};
        check(mlfma_autotune(h_, nrhs, reps, &t));
        return t;
    }

    // The one-vector product's schedule: the bits mlfma_tuning.schedule reports.
    void setSchedule(int schedule) { check(mlfma_set_schedule(h_, schedule)); }

    // evalRvec on page-locked host buffers the device addresses directly
    // (cudaHostAlloc / cudaMallocHost / cudaHostRegister memory of n values).
    void evalRvecMapped(const cplx* lvec, cplx* rvec, bool accumulate = false) {
        check(mlfma_matvec_mapped(h_, reinterpret_cast<const double*>(lvec), reinterpret_cast<double*>(rvec),
                                  accumulate ? 1 : 0));
    }

    // nrhs systems at once (B: nrhs x n, caller order), GMRES or, with
    // opts.flexible, FGMRES per system; infos may be null.
    std::vector<cplx> solveMulti(int nrhs, const std::vector<cplx>& B, const mlfma_solver_opts& opts,
                                 std::vector<mlfma_solve_info>* infos = nullptr) {
        std::vector<cplx> X(B.size());
        std::vector<mlfma_solve_info> inf(static_cast<size_t>(nrhs));
        const int code = mlfma_gmres_multi(h_, nrhs, reinterpret_cast<const double*>(B.data()),
                                           reinterpret_cast<double*>(X.data()), &opts, inf.data());
        if (code != MLFMA_OK && code != MLFMA_ERR_NOT_CONVERGED) check(code);
        if (infos) *infos = inf;
        return X;
    }

    mlfma_handle handle() const { return h_; }

private:
    explicit Operator(mlfma_handle h) : h_(h) {}
    mlfma_handle h_ = nullptr;
};

class Solver {
public:
    Solver(Operator& op, int maxIter, double EPS) : op_(op) {
        opts_.max_iter = maxIter;
        opts_.tol = EPS;
        opts_.restart = 0;
        opts_.ref_givens = 1;
    }
    // Unrestarted GMRES from lvec = -V; returns the currents (Solver::solve).
    std::vector<cplx> solve() {
        const std::vector<cplx> b = op_.rhs();
        currents_.assign(b.size(), cplx(0));
        const int code = mlfma_gmres(op_.handle(), reinterpret_cast<const double*>(b.data()),
                                     reinterpret_cast<double*>(currents_.data()), &opts_, &info_);
        if (code != MLFMA_OK && code != MLFMA_ERR_NOT_CONVERGED) check(code);
        return currents_;
    }
    const mlfma_solve_info& info() const { return info_; }
    const std::vector<cplx>& getCurrents() const { return currents_; }

private:
    Operator& op_;
    mlfma_solver_opts opts_{};
    mlfma_solve_info info_{};
    std::vector<cplx> currents_;
};

}  // namespace mlfma_b200
