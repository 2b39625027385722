/*
 * mlfma_b200: C ABI of the B200 MLFMA operator and GMRES solver.
 *
 * The reference (ellilu11/MLFMA) has no foreign-function interface; its
 * operator API is a C++ object protocol driven from main() with global
 * state.  Each entry point below replaces one step of that protocol; the
 * reference file:line it stands in for is given beside it.
 *
 * Conventions:
 *   - every call returns an int status (MLFMA_OK or MLFMA_ERR_*); nothing throws
 *     across the boundary; mlfma_last_error() gives a message (per thread);
 *   - complex vectors are interleaved (re, im) doubles, length 2*N, in the
 *     caller's source order (the order sources were passed in);
 *   - host buffers are caller-owned; device state is owned by the handle;
 *   - a handle is used from one thread at a time; many handles may coexist.
 */
#ifndef MLFMA_B200_H
#define MLFMA_B200_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
    MLFMA_OK = 0,
    MLFMA_ERR_ARG = 1,            /* invalid argument or input geometry */
    MLFMA_ERR_CUDA = 2,           /* CUDA runtime error (no device, launch failure, ...) */
    MLFMA_ERR_STATE = 3,          /* call out of order (e.g. matvec before setup) */
    MLFMA_ERR_NOT_CONVERGED = 4,  /* solver hit its iteration limit */
    MLFMA_ERR_NONFINITE = 5,      /* NaN or Inf in an input or the solver state */
    MLFMA_ERR_INTERNAL = 6
};

enum { MLFMA_DIPOLE = 0, MLFMA_RWG = 1 };

/* Precision enum of the reference (src/config.h:7): triangle quadrature rule. */
enum { MLFMA_QUAD_1PT = 0, MLFMA_QUAD_3PT = 1, MLFMA_QUAD_7PT = 2, MLFMA_QUAD_13PT = 3 };

typedef struct mlfma_op_s* mlfma_handle;

/* Operator configuration.  The first six fields are the reference Config
 * (src/config.h:50-73) with the same meaning; the rest are extensions. */
typedef struct {
    int quad_prec;       /* MLFMA_QUAD_*; RWG only */
    int digits;          /* excess-bandwidth digits of the angular sampling */
    int interp_order;    /* Lagrange half-width: 2*interp_order points */
    double over_interp;  /* psi oversampling of the transfer functions */
    double root_leng;    /* side of the root box, centred at the origin */
    int max_node_srcs;   /* a box splits while it holds more sources than this */
    int max_level;       /* >0: do not split below this level (0 = reference rule) */
    int ref_compat;      /* 1: reproduce the reference's stale-local rule (default) */
    int device;          /* CUDA device ordinal */
    int precision;       /* MLFMA_FP64 (default) or MLFMA_MIXED: far field in complex
                            float with float accumulation, near field and vectors in
                            complex double */
    int self_terms;      /* 0: the reference's operator (zero diagonal, coincident
                            triangles skipped, src/sources/dipole.h:65,
                            src/sources/rwg.cpp:97,113-116).  1: dipoles get a unit
                            diagonal; RWG pairs whose triangles share a vertex are
                            integrated in mixed-potential form with the 1/R
                            singularity of the source triangle in closed form
                            (symmetrised, FP64) */
    int max_rhs;         /* most right-hand sides of one product (1..64; mlfma_matvec_multi,
                            mlfma_gmres_multi); > 1 reserves their device work space */
    int device_tree;     /* 1: build the octree and its lists on the device (Morton keys,
                            radix sort, one thread per box for the lists): the same
                            boxes, numbering, source order and lists as the host build
                            (Stem ctor, src/fmm/stem.cpp:3-26; src/fmm/nbor.cpp:10-644;
                            Node::buildInteractionList, src/fmm/node.cpp:61-84); trees
                            deeper than 21 levels fall back to the host build */
} mlfma_config;

enum { MLFMA_FP64 = 0, MLFMA_MIXED = 1 };

/* Incident plane wave (src/excite.h:6-28; file format src/fileio.h:8-27). */
typedef struct {
    double amplitude;
    double pol[3];
    double khat[3];
    double wavenum;
} mlfma_planewave;

typedef struct {
    int num_nodes, num_leaves, max_level, num_levels_far;
    long long list2, list4, near_pairs, near_entries, pattern_elems;
    long long device_bytes;
    int launches_per_matvec;  /* kernels this library launches per matvec */
} mlfma_stats;

/* Per-stage device time of one matvec, ms (the reference's ClockTimes stages,
 * src/clock.h:8-17, plus the near field). */
typedef struct {
    float gather, s2m, m2m, m2l, l2l, l2t, near_field, finish, total;
} mlfma_stage_times;

/* Algorithmic HBM bytes of one matvec per stage (roofline accounting). */
typedef struct {
    double s2m, m2m, m2l, l2l, l2t, near_field, total;
} mlfma_traffic;

typedef struct {
    int max_iter;        /* iteration limit (reference: 500, src/mlfma.cpp:69) */
    double tol;          /* relative residual target (reference: 1e-6, src/mlfma.cpp:70) */
    int restart;         /* 0 = no restart (reference), else GMRES(restart) */
    int ref_givens;      /* 1: complex-symmetric Givens of the reference (src/math.h:168-172) */
    int refine;          /* MLFMA_MIXED operators: 1 = iterative refinement (inner GMRES on the
                            mixed operator, outer residual r = b - A x in FP64, x += correction;
                            stops on the FP64 residual); 0 = GMRES on the mixed operator alone.
                            Ignored by MLFMA_FP64 operators. */
    double inner_tol;    /* refinement: inner relative residual target (0 = automatic); flexible:
                            an inner solve stops early below this relative residual (0 = never) */
    int flexible;        /* 1: flexible GMRES (FGMRES(restart), restart 0 = max_iter outer steps):
                            outer Krylov space, products and residual in FP64; each outer step's
                            preconditioner is inner_iters GMRES iterations from zero on the
                            operator's own far field (the complex-float one on a mixed operator).
                            iterations counts inner products, refinements outer products.
                            No counterpart in the reference. */
    int inner_iters;     /* flexible: GMRES iterations per inner solve (0 = 20) */
    int precond;         /* 1: leaf block-Jacobi right preconditioner (each leaf's diagonal block of
                            A, loads included, inverted on the GPU; with flexible = 1 it
                            preconditions the inner solves).  Forward solves; no counterpart in
                            the reference. */
} mlfma_solver_opts;

typedef struct {
    int iterations;
    double residual;       /* final |g_{k+1}| / g0 estimate */
    double true_residual;  /* ||b - A x|| / ||b||, recomputed */
    double seconds;
    int refinements;       /* FP64 residual evaluations of iterative refinement (0 otherwise) */
} mlfma_solve_info;

/* Fill *cfg with the defaults (digits 3, order 3, overInterp 2, rootLeng 4, 64 per box). */
int mlfma_config_default(mlfma_config* cfg);

/* Dipole sources: pos and mom are n x 3 (row-major).  Builds the host plan:
 * tree, lists, angular grids and tables (replaces Node::initStatic,
 * src/fmm/node.cpp:13-26, the Stem/Leaf constructors, src/mlfma.cpp:26-30,
 * buildLists, src/fmm/stem.cpp:48-57, and Node::buildTables,
 * src/fmm/node.cpp:46-56, after importDipoles, src/fileio.h:110-131). */
int mlfma_create_dipoles(const mlfma_config* cfg, const mlfma_planewave* pw, int n,
                         const double* pos, const double* mom, mlfma_handle* out);

/* RWG sources on a triangle mesh: verts nv x 3, faces nf x 3, rwgs ne x 4
 * (v0, v1, t+, t-), 0-based (importRWG, src/fileio.h:174-202, then the same
 * setup steps as mlfma_create_dipoles). */
int mlfma_create_rwg(const mlfma_config* cfg, const mlfma_planewave* pw, int nv, const double* verts,
                     int nf, const int* faces, int ne, const int* rwgs, mlfma_handle* out);

/* The reference's text formats (no GPU needed).  Errors: MLFMA_ERR_ARG with
 * "Unable to find file" or "Unable to parse line" in mlfma_last_error(), the
 * reference's messages.  Each line is parsed as the reference parses it: the
 * values it needs are read and the rest of the line ignored; a line without
 * them (a blank line included) is an error.
 * Plane wave: the first line holds amplitude, pol (3), khat (3), wavenumber
 * (importPlaneWave, src/fileio.h:8-27). */
int mlfma_read_planewave(const char* path, mlfma_planewave* pw);
/* Dipoles: one line per dipole, position (3) and moment (3) (importDipoles,
 * src/fileio.h:110-131), then as mlfma_create_dipoles. */
int mlfma_create_dipoles_from_file(const mlfma_config* cfg, const mlfma_planewave* pw, const char* path,
                                   mlfma_handle* out);
/* RWG mesh: vertices (x y z per line), faces (three 0-based vertex indices),
 * rwgs (v0 v1 t+ t-) (importVertices, importTriangles, importRWG,
 * src/fileio.h:134-202), then as mlfma_create_rwg. */
int mlfma_create_rwg_from_files(const mlfma_config* cfg, const mlfma_planewave* pw, const char* vertices_path,
                                const char* faces_path, const char* rwgs_path, mlfma_handle* out);
/* Solution file: one complex current per line as "(re,im)", 15 significant
 * digits, scientific (Solver::printSols, src/solver.cpp:149-165; the caller
 * chooses the path).  x: n interleaved complex values. */
int mlfma_write_solution(const char* path, int n, const double* x);

/* Upload to the GPU and assemble radiation patterns and near-field blocks
 * there (Leaf::buildNearRads, src/fmm/leaf.cpp:108-180; root->resizeCoeffs;
 * Leaf::buildRadPats, src/fmm/leaf.cpp:185-207). */
int mlfma_setup(mlfma_handle h);

int mlfma_num_unknowns(mlfma_handle h, int* n);
int mlfma_get_stats(mlfma_handle h, mlfma_stats* st);

/* b = -V, the GMRES right-hand side (Solver ctor, src/solver.cpp:31-32;
 * Source::buildVoltage, src/sources/dipole.h:29-32, src/sources/rwg.h:18-21). */
int mlfma_rhs(mlfma_handle h, double* b);

/* y = A x (accumulate = 0) or y += A x (accumulate = 1), host buffers
 * (Solver::evalRvec, src/solver.cpp:41-57: rvec += A lvec).  Copies in and
 * out through the handle's stream. */
int mlfma_matvec(mlfma_handle h, const double* x, double* y, int accumulate);

/* Same on device buffers (cudaStream_t passed as void*, NULL = handle's stream).
 * Asynchronous with respect to the host.  The product runs as one CUDA graph
 * (captured on the first call) between a gather and a scatter kernel, using
 * the handle's internal work buffers: products on one handle must not overlap
 * on the GPU (issue them on one stream, or order the streams). */
int mlfma_matvec_device(mlfma_handle h, const void* d_x, void* d_y, int accumulate, void* stream);

/* mlfma_matvec (Solver::evalRvec, src/solver.cpp:41-57) on page-locked host
 * buffers that the device addresses directly (cudaHostAlloc / cudaMallocHost
 * memory, or cudaHostRegister'd memory, each covering the n complex values):
 * no separate copies; the gather kernel reads x and the final kernel writes y
 * across the bus, each in one contiguous run per warp.  Returns when y is
 * complete.  MLFMA_ERR_ARG when the first or the last value of x or y is not
 * in such memory. */
int mlfma_matvec_mapped(mlfma_handle h, const double* x, double* y, int accumulate);

/* Solve A x = b with GMRES on the device; b and x host buffers (Solver::solve,
 * src/solver.cpp:116-146).  x is overwritten (initial guess 0).  On a mixed
 * operator with opts->refine = 1 the answer meets tol on the FP64 residual. */
int mlfma_gmres(mlfma_handle h, const double* b, double* x, const mlfma_solver_opts* opts,
                mlfma_solve_info* info);

/* Operator of the inner iterations of flexible solves (opts->flexible) on h:
 * the outer FGMRES space and its products stay on h's FP64 far field, each
 * outer step is preconditioned by opts->inner_iters GMRES iterations on
 * `inner` instead of on h.  `inner` is a set-up operator on the same device
 * with the same unknowns in the same source order (the same sources, root_leng,
 * max_node_srcs and max_level); it may use fewer digits, a lower
 * interpolation order or mixed precision, which makes each inner product
 * cheaper.  NULL detaches it; destroying either handle detaches it too. */
int mlfma_set_inner_operator(mlfma_handle h, mlfma_handle inner);

/* Far field of the currents x (host, n complex, caller order) along ndir unit
 * directions khat (host, ndir x 3): out (host, ndir x 3 complex) =
 * C k (I - khat khat^T) sum_n x_n f_n(k khat), the sum of Node::printFarSols
 * (src/fmm/node.cpp:147-178) for any direction list (the reference prints it
 * on the root's angular grid).  Allocates device scratch for the directions. */
int mlfma_farfield(mlfma_handle h, const double* x, int ndir, const double* khat, double* out);

/* Self-check of the failure path of the kernels' bounded waits (the
 * near-field kernel waits on mbarriers for its bulk copies; every wait gives
 * up after about a second and raises the operator's error word, which the
 * synchronous calls report, instead of hanging).  Runs one wait on a barrier nothing arrives
 * on, limited to about 8 ms, on `device`; *timed_out = 1 when it ran out and
 * the kernel returned.  No GPU fault is involved; the context stays usable. */
int mlfma_check_bounded_wait(int device, int* timed_out);

/* Rows of the operator evaluated densely: y[i] = (A x)[rows[i]] with every
 * interaction computed directly in FP64 (O(N) work per row; the near-field
 * entry of every pair, diagonal loads not included).  The dense FP64
 * reference for the relative error of an MLFMA product or of a solution's
 * residual on sampled rows.  rows: caller-order indices; x (n) and y (nrows)
 * interleaved complex.  No counterpart in the reference. */
int mlfma_dense_rows(mlfma_handle h, int nrows, const int* rows, const double* x, double* y);

/* The same operator's entries themselves: d_out[i * ld + j] = A[rows[i]][j]
 * (caller order, j < n, ld >= n) in a DEVICE buffer, every interaction
 * evaluated directly in FP64 (diagonal loads not included).  A dense reference
 * for the adjoint and the solution (all rows of a 30,720-unknown operator are
 * 15 GB).  Returns when written.  No counterpart in the reference (its direct
 * path, src/mlfma.cpp:84-107, applies the entries without keeping them). */
int mlfma_dense_block_device(mlfma_handle h, int nrows, const int* rows, void* d_out, long long ld);

/* GMRES that allocates no device memory.  No counterpart in the reference.
 * mlfma_gmres allocates its Krylov basis with cudaMalloc on first use; a
 * caller that cannot allocate device memory during a solve (a fixed memory
 * budget reserved at start-up, an allocator policy that forbids cudaMalloc
 * after initialisation) calls this instead.  Same algorithm and options as
 * mlfma_gmres; b and x are DEVICE buffers of n complex values in the caller's
 * source order; the solve runs on the handle's stream and returns when done.
 * The workspace is one fixed array in device memory that is part of the
 * library (32 MiB).  CUDA creates it on a device when the library's solver
 * module is first used there; mlfma_setup does that on the operator's device,
 * so the 32 MiB are taken at setup (not during a solve, and not merely by
 * loading the library) and held until the process exits.  A solve of n
 * unknowns with m = restart (max_iter when restart is 0) needs
 * n (m + 5) + (m + 2)(2 + ceil(n / 8192)) complex values, n (m + 7) + ... with
 * refinement on a mixed operator; more than 2,097,152 gives MLFMA_ERR_ARG with
 * the count in mlfma_last_error().  All calls share the array and it keeps the
 * last call's contents, so calls that overlap on the GPU race. */
int mlfma_gmres_noalloc(mlfma_handle h, const void* d_b, void* d_x, const mlfma_solver_opts* opts,
                        mlfma_solve_info* info);

/* b = -V for another incident plane wave of the operator's wavenumber (the
 * Solver ctor's right-hand side, src/solver.cpp:31-32, with
 * Source::buildVoltage, src/sources/dipole.h:29-32, src/sources/rwg.h:18-21,
 * evaluated for pw).  Many incident directions give the right-hand sides of
 * mlfma_gmres_multi. */
int mlfma_rhs_planewave(mlfma_handle h, const mlfma_planewave* pw, double* b);

/* Y = A X (accumulate = 0) or Y += A X for nrhs vectors at once (1 <= nrhs <=
 * max_rhs): Solver::evalRvec, src/solver.cpp:41-57, applied to many lvec.
 * x and y hold the nrhs vectors one after another (nrhs x n complex, caller
 * order).  Every coefficient of the operator is read once per call, and the
 * per-leaf products become small complex GEMMs.  Host buffers. */
int mlfma_matvec_multi(mlfma_handle h, int nrhs, const double* x, double* y, int accumulate);
/* Same on device buffers (stream as in mlfma_matvec_device). */
int mlfma_matvec_multi_device(mlfma_handle h, int nrhs, const void* d_x, void* d_y, int accumulate, void* stream);

/* GMRES on nrhs right-hand sides sharing every product (Solver::solve,
 * src/solver.cpp:116-146, for many b): each system has its own Krylov basis
 * and Givens rotations (unitary; ref_givens is ignored) and stops on its own
 * tolerance.  b and x: nrhs x n complex host buffers, caller order; info:
 * nrhs records (may be NULL).  refine as in mlfma_gmres.  flexible = 1:
 * FGMRES(restart) per right-hand side with FP64 outer spaces, each outer
 * step's inner solves (inner_iters iterations on the operator's own far
 * field) run for all right-hand sides together; iterations counts a system's
 * inner iterations, refinements its outer steps.  precond and an inner
 * operator serve mlfma_gmres only. */
int mlfma_gmres_multi(mlfma_handle h, int nrhs, const double* b, double* x, const mlfma_solver_opts* opts,
                      mlfma_solve_info* info);
/* Per-stage CUDA-event time of one product on nrhs right-hand sides. */
int mlfma_time_stages_multi(mlfma_handle h, int nrhs, mlfma_stage_times* t);

/* ---- Adjoint and gradients (no counterpart in the reference).  The
 * operator must be set up with ref_compat = 0: the reference's stale-local
 * rule makes the product depend on earlier products, and such a map has no
 * adjoint.  The transposed product is the exact transpose of the discrete
 * MLFMA pipeline (conjugated and plain patterns swap ends, interpolation and
 * anterpolation swap with the octant shifts moved to the other grid,
 * translations use the negated offsets); the stored near field is symmetric
 * to rounding and is reused. */

/* Diagonal loads added to the operator: A x + z .* x (surface-impedance loads
 * per unknown, in ohms, like the entries of A = C k Z).  z: n complex, caller
 * order; NULL removes them.  Applies to every later product and solve. */
int mlfma_set_loads(mlfma_handle h, const double* z);

/* y = A^H x (accumulate = 0) or y += A^H x, host buffers. */
int mlfma_matvec_adjoint(mlfma_handle h, const double* x, double* y, int accumulate);

/* Solve A^H x = b with GMRES (unitary Givens rotations); as mlfma_gmres. */
int mlfma_gmres_adjoint(mlfma_handle h, const double* b, double* x, const mlfma_solver_opts* opts,
                        mlfma_solve_info* info);

/* g = M^H F: the adjoint of mlfma_farfield (M: currents -> far field along
 * khat), for F (ndir x 3 complex); g: n complex, caller order. */
int mlfma_farfield_adjoint(mlfma_handle h, int ndir, const double* khat, const double* F, double* g);

/* Far-field power objective and its gradient by one forward and one adjoint
 * solve.  Excitation b = sum_j w_j b_j over nexc incident plane waves (b_j as
 * mlfma_rhs_planewave; w: nexc complex weights); currents I solve
 * (A + diag(z)) I = b with the loads z of mlfma_set_loads; J = sum over the
 * ndir directions khat of |F|^2, F = mlfma_farfield(I).  Outputs: *J;
 * grad_loads[n] = dJ/dRe z_n + i dJ/dIm z_n; grad_w[nexc] likewise for the
 * weights; currents[n] = I (each may be NULL); info[2] = forward and adjoint
 * solve records (may be NULL). */
int mlfma_vjp_farfield_power(mlfma_handle h, int nexc, const mlfma_planewave* pws, const double* w, int ndir,
                             const double* khat, const mlfma_solver_opts* opts, double* J, double* grad_loads,
                             double* grad_w, double* currents, mlfma_solve_info* info);

/* Launch shapes chosen by mlfma_autotune (no counterpart in the reference). */
typedef struct {
    int m2l_chunk;             /* one-vector translation: directions per thread block */
    int m2m_rows[20];          /* one-vector interpolation: parent theta rows per block, by parent level */
    int multi_m2m_rows_fast;   /* many-rhs interpolation grid: 1 rows fastest, 0 parents fastest */
    int multi_l2l_pairs;       /* many-rhs anterpolation: column pairs per block */
    float product_ms_before;   /* one product (nrhs right-hand sides) before and after, ms */
    float product_ms_after;
    int near_blocks_per_sm;    /* one-vector near field: persistent blocks per SM (it runs beside the far field) */
    int interp_path;           /* interpolation/anterpolation kernels chosen (see mlfma_set_interp_path) */
    int schedule;              /* one-vector product: bit 0 translation lists staged in shared memory,
                                  bit 1 near field started after aggregation, bit 2 two side streams
                                  for the finer levels' translations, bit 3 the far-field chain's
                                  kernels launched as programmatic dependent launches (each kernel's
                                  blocks scheduled while its predecessor drains) */
    int m2m_staged;            /* one-vector interpolation, transition p+1 -> p: bit p = children summed
                                  first in shared memory, bit 16 + p = the same with column-stationary
                                  phi passes; neither = one interpolation per child */
    int l2l_staged;            /* one-vector anterpolation, transition p -> p+1: bit p = parent's local
                                  pattern staged in shared memory, bit 16 + p = the same with
                                  column-stationary phi passes, bit 24 + p = the persistent prefetching
                                  kernel */
    int near_kernel;           /* one-vector near field: 0 one tile per thread block (row and column
                                  threads), 1 one tile per warp from shared memory, 2 one tile per
                                  warp from global memory (see mlfma_set_near_kernel) */
} mlfma_tuning;

/* Autotuner: times the candidate launch shapes of the stages on this operator
 * (reps timed launches each, CUDA events on the handle's stream) and keeps
 * the fastest.  nrhs = 1 tunes the one-vector product; 2 <= nrhs <= max_rhs the
 * many-rhs product at that width.  Results are unchanged up to rounding; the
 * operator's state (the reference's stale locals) is preserved.  Call outside
 * any stream capture; out may be NULL. */
int mlfma_autotune(mlfma_handle h, int nrhs, int reps, mlfma_tuning* out);

/* Interpolation (M2M; Stem::buildMpoleCoeffs + addInterpCoeffs,
 * src/fmm/stem.cpp:72-184) and anterpolation (L2L; getShiftedLocalCoeffs +
 * addAnterpCoeffs, stem.cpp:109-244) of the complex-float far field on the
 * tensor cores: every box of a level at once as separable theta and phi
 * contractions (tcgen05 MMAs, split-precision 3xTF32, FP32 accumulation),
 * children shifted and summed before the interpolation.  mode bit 0: M2M of
 * the one-vector product, bit 1: M2M of the many-right-hand-side product,
 * bit 2: L2L of the one-vector product, bit 3: L2L of the many-rhs product;
 * 0 = the CUDA-core kernels (the default); mlfma_autotune times both kernel
 * families stage by stage and keeps the faster.  Products of the FP64 far
 * field and transposed products always use the CUDA-core kernels.
 * MLFMA_ERR_ARG when the operator has no complex-float far field or a grid
 * exceeds the kernels' shared memory.  Results agree with the CUDA-core
 * kernels to float rounding. */
int mlfma_set_interp_path(mlfma_handle h, int mode);
int mlfma_get_interp_path(mlfma_handle h, int* mode);
/* CUDA-core interpolation kernels of the one-vector product, on every level
 * transition where their shared memory fits: bit 0, M2M with the children
 * shifted and summed on the child grid first (one interpolation per parent,
 * all taps from shared memory; rounding-level differences from the per-child
 * kernel); bit 1, L2L with the parent's shifted local pattern staged in shared
 * memory (the same arithmetic in the same order); bit 2, their phi passes
 * column-stationary (a thread keeps one output column's stencil in registers
 * and walks the rows); bit 3, L2L as a persistent kernel that prefetches the
 * next pair's inputs with asynchronous copies while it computes one.  Modes 1 and 2 are on after setup; mlfma_autotune
 * chooses per transition (mlfma_tuning.m2m_staged/l2l_staged). */
int mlfma_set_staged_interp(mlfma_handle h, int mode);
/* Near-field kernel of the one-vector product (Leaf::evalPairSols,
 * evalNearNonNborSols, evalSelfSols, src/fmm/leaf.cpp:318-383; each stored block
 * applied as Z and Z^T, tiles streamed by bulk copies): kind 0, one tile per
 * thread block (row threads and column threads; the default); kind 1, one
 * tile per warp, each entry read from shared memory once and the row sums
 * formed by a warp reduce-scatter; kind 2, one tile per warp with the entries
 * loaded straight from global memory into registers (no shared-memory stage).
 * Same partial sums, other rounding order; mlfma_autotune tries all three. */
int mlfma_set_near_kernel(mlfma_handle h, int kind);

/* The one-vector product's schedule, as mlfma_tuning.schedule reports it (no
 * counterpart in the reference, which runs the stages one after another on
 * one thread): bit 0 translation lists staged in shared memory, bit 1 near
 * field started after aggregation, bit 2 two side streams for the finer
 * levels' translations, bit 3 the far-field chain's kernels launched as
 * programmatic dependent launches.  Results are unchanged up to rounding
 * order (bit 3 changes nothing).  MLFMA_ERR_ARG outside 0..15. */
int mlfma_set_schedule(mlfma_handle h, int schedule);

/* ---- Many independent operators of uneven size (no counterpart in the
 * reference, which holds one problem per process).  A batch refers to set-up
 * operators on one device (it does not own them; destroy it first).  Vectors
 * are packed: operator 0's n0 values, then operator 1's, ... (caller order
 * within each). */
typedef struct mlfma_batch_s* mlfma_batch;

/* One CUDA graph holds every operator's product as a parallel branch, so one
 * graph launch applies all of them.  The operators' own products must not
 * overlap a batch product on the GPU (they share work buffers), and the graph
 * keeps the launch shapes the operators had at creation: run mlfma_autotune
 * on them first. */
int mlfma_batch_create(int nops, const mlfma_handle* ops, mlfma_batch* out);
/* Total length of the packed vectors. */
int mlfma_batch_size(mlfma_batch b, long long* total);
/* y = blockdiag(A_0, A_1, ...) x: host buffers, or device buffers on stream
 * (NULL = the batch's own stream; asynchronous). */
int mlfma_batch_matvec(mlfma_batch b, const double* x, double* y);
int mlfma_batch_matvec_device(mlfma_batch b, const void* d_x, void* d_y, void* stream);
/* Every operator's GMRES at once (one host thread each, each on its
 * operator's streams); info: one record per operator (may be NULL).  Returns
 * the worst status. */
int mlfma_batch_gmres(mlfma_batch b, const double* rhs, double* x, const mlfma_solver_opts* opts,
                      mlfma_solve_info* info);
int mlfma_batch_destroy(mlfma_batch b);

/* The handle's own CUDA stream (cudaStream_t as void*), on which mlfma_matvec
 * and mlfma_gmres run; callers may record events on it. */
int mlfma_get_stream(mlfma_handle h, void** stream);

/* CUDA-event time of each stage of one matvec on the handle's stream. */
int mlfma_time_stages(mlfma_handle h, mlfma_stage_times* t);
/* CUDA-event time (ms) of each level's far-field launches, one at a time on
 * the handle's stream: for level l, ms[3l] the interpolation into l (M2M from
 * l + 1), ms[3l + 1] the translation at l, ms[3l + 2] the anterpolation out of
 * l (L2L to l + 1); 0 where a level has none.  *nlevels = max level + 1; ms ==
 * NULL only asks for it; cap >= 3 * *nlevels. */
int mlfma_time_levels(mlfma_handle h, int cap, float* ms, int* nlevels);
int mlfma_get_traffic(mlfma_handle h, mlfma_traffic* t);

/* Diagnostics: angular grid of a level (sizes: nth, nph, L) and the
 * outgoing (which = 0) or local (which = 1) patterns of every box of a level
 * after the last matvec, as [box][dir][2] complex, plus each box's integer
 * coordinates (3 ints per box). */
int mlfma_level_info(mlfma_handle h, int level, int* sizes, double* thetas, double* weights,
                     double* phis);
int mlfma_level_boxes(mlfma_handle h, int level, int* nbox, int* coords);
int mlfma_level_patterns(mlfma_handle h, int level, int which, double* out, long long count);
/* Transfer functions of a level: 316 x ndir complex in the order of
 * Math::getINodeDistVecs (src/math.cpp:106-122). */
int mlfma_level_transl(mlfma_handle h, int level, double* out);
/* The same table as the operator uses it: built on the GPU at setup
 * (Tables::getAlpha, getInterpPsi, buildTranslationTable,
 * src/fmm/tables.cpp:90-220), complex double, same layout. */
int mlfma_level_transl_gpu(mlfma_handle h, int level, double* out);

/* Far-field leaves in tree order: count, then per leaf (level, box, first
 * source in tree order, source count) and the tree-order -> caller-order
 * permutation (n ints). */
int mlfma_far_leaves(mlfma_handle h, int* count, int* info, int* perm);
/* The octree and its lists, for inspection: which = 0 gives 14 ints per node
 * in node order (level, parent, branch, child[8], leaf, src_begin, src_count),
 * 1 the source order (perm[tree slot] = caller index), 2..5 per node the
 * length and then the node ids of its equal-or-greater neighbours, list 1
 * (near leaves), list 2 and list 4.  *count receives the ints needed; out ==
 * NULL only asks for it. */
int mlfma_tree_export(mlfma_handle h, int which, int* out, long long cap, long long* count);
/* Reference-rounded RWG radiation patterns computed on the host, laid out as
 * the device array: per far leaf, per source, per direction, 2 complex. */
int mlfma_rwg_patterns_host(mlfma_handle h, double* out, long long count);

int mlfma_destroy(mlfma_handle h);

const char* mlfma_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* MLFMA_B200_H */
