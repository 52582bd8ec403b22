/*
 * prism_solve.h -- C ABI of the B200 solve phase for PrisPack.
 *
 * One handle = one square CSR operator A resident on one CUDA device, an
 * optional preconditioner M built on the host and uploaded once, and the
 * device workspace of the Krylov solvers.  Every handle owns one CUDA stream;
 * a handle is not thread-safe (the reference's preconditioner objects are not
 * either: they keep per-object scratch vectors).  No C++ exception crosses
 * this boundary; every entry point returns a prism_status and, on failure,
 * leaves a message for prism_last_error() (per calling thread).
 *
 * Index and value types follow HOST::CSRMatrix<double>
 * (include/MatrixClass/CSRMatrix.h:19-30 of the reference): uint32 row
 * offsets and column indices, sorted columns within each row, double values.
 *
 * Entry points and the reference interface each one replaces:
 *   prism_create / prism_destroy      HOST::CSRMatrix<double> ctor/dtor
 *                                     (include/MatrixClass/CSRMatrix.h:57)
 *   prism_spmv*                       CSRMatrix::MatPVec
 *                                     (include/MatrixClass/CSRMatrix.h:360-395)
 *   prism_set_precond_ic              IncompleteCholesky(A, threshold) + setup()
 *                                     (source/Preconditioner/IncompleteCholesky.cpp:11-246)
 *   prism_set_precond_ildlt           IncompleteLDLT(A, tol) + setup()
 *                                     (source/Preconditioner/IncompleteLDLT.cpp:39-186)
 *   prism_set_precond_ilut            IncompleteLU(A, lfill, tol) + setup()
 *                                     (source/Preconditioner/IncompleteLU.cpp:12-266)
 *   prism_apply*                      BasePrecondition::MInvSolve(vecIN, vecOUT)
 *                                     (include/Preconditioner/BasePreconditon.h:110-128,
 *                                      TriangularPrecondition::MInvSolve :307-358)
 *   prism_solve* (PRISM_SOLVER_FCG,   CG<double>::solve
 *                 PRISM_SOLVER_CG)    (source/Solver/CG.cpp:34-83)
 *   prism_solve* (PRISM_SOLVER_FGMRES,GMRES<double>::solve + setRestart
 *                 PRISM_SOLVER_GMRES) (source/Solver/GMRES.cpp:60-221)
 *   prism_laplacian_*                 generateLaplacianCSR
 *                                     (include/MatrixClass/ModelProblem.h:45-52,
 *                                      source/MatrixClass/ModelProblem.cpp:68-133)
 *   prism_mtx_read*                   HOST::ReadMtxTools::loadMatrix / loadRightHand
 *                                     (source/utils/TestTools/ReadMtxTools.cpp:50-453)
 */
#ifndef PRISM_SOLVE_H
#define PRISM_SOLVE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum prism_status {
    PRISM_OK = 0,
    PRISM_ERR_ARG = 1,            /* bad argument, size or pointer */
    PRISM_ERR_CUDA = 2,           /* a CUDA runtime call failed */
    PRISM_ERR_ZERO_PIVOT = 3,     /* ILUT/ILDLT |pivot| < 1e-15 (reference throws) */
    PRISM_ERR_NOT_SPD = 4,        /* IC met a non-positive pivot (reference prints and returns) */
    PRISM_ERR_NOT_READY = 5,      /* apply/solve before a preconditioner was set up */
    PRISM_ERR_TIMEOUT = 6,        /* a bounded device-side wait ran out (SpTRSV row flags) */
    PRISM_ERR_NONFINITE = 7,      /* NaN/Inf met in a Krylov scalar */
    PRISM_ERR_ALLOC = 8,          /* host or device allocation failed */
    PRISM_ERR_UNSUPPORTED = 9,    /* option not available for this preconditioner/solver */
    PRISM_ERR_BAD_MATRIX = 10     /* CSR structure invalid (row offsets, column range, order) */
} prism_status;

typedef enum prism_precision {
    PRISM_FP64 = 0,               /* factor values stored in double (<double,double> instantiation) */
    PRISM_FP32 = 1,               /* factor values stored in float  (<float,double> instantiation) */
    PRISM_FP32_APPLY = 2          /* float factor values and single-precision arithmetic inside the
                                     triangular sweeps of the streamed kernel (right-hand side and
                                     1/diag rounded to float, products and sums in float, results
                                     widened to double); everything outside the sweeps, and sweeps
                                     the streamed layout does not fit or block solves run, stays in
                                     double.  No reference counterpart: the reference's float
                                     instantiation computes in double. */
} prism_precision;

typedef enum prism_precond_kind {
    PRISM_PRECOND_NONE = 0,
    PRISM_PRECOND_IC = 1,         /* PreconditionIC    (BasePreconditon.h:12-19) */
    PRISM_PRECOND_ILUT = 2,       /* PreconditionILUT  */
    PRISM_PRECOND_ILDLT = 3,      /* PreconditionILDLT */
    PRISM_PRECOND_GMSLR = 4,      /* PreconditionGMSLR */
    PRISM_PRECOND_AMSED = 5       /* PreconditionAMSED */
} prism_precond_kind;

typedef enum prism_solver_kind {
    PRISM_SOLVER_FCG = 0,         /* CG with CGType FlexibleCG (CG.h:14-18) */
    PRISM_SOLVER_CG = 1,          /* CG with CGType NormalCG: M^{-1} only at step 0 (CG.cpp:48,65) */
    PRISM_SOLVER_FGMRES = 2,      /* GMRES with FlexibleGMRES */
    PRISM_SOLVER_GMRES = 3        /* GMRES with NormalGMRES (no preconditioner applied, GMRES.cpp:164) */
} prism_solver_kind;

typedef enum prism_launch_mode {
    PRISM_LAUNCH_AUTO = 0,        /* GMRES: each restart cycle runs as one CUDA graph whose loop over the
                                     Arnoldi steps ends on the device (one host read per cycle), with
                                     plain launches where the runtime cannot build that graph */
    PRISM_LAUNCH_STREAM = 1       /* plain launches, one host read per Arnoldi step */
} prism_launch_mode;

typedef struct prism_solve_opts {
    int32_t solver;               /* prism_solver_kind */
    double tol;                   /* relative residual tolerance (CG.cpp:59, GMRES.cpp:194) */
    uint32_t max_iter;            /* CG: maxIter (CG.cpp:57); GMRES: 500 as MAX_ITER_NUM_SOLVER (config.h:25) */
    uint32_t restart;             /* GMRES restart m; 0 = no restart (setRestart(false, .)) */
    const double* x_ref;          /* optional reference solution (device pointer for the *_device calls,
                                     host pointer for the host-buffer calls; NULL: none): the solve then
                                     reports its forward error against it.  Ignored by the adjoint, block
                                     and batch solves.  No reference counterpart. */
    int32_t launch_mode;          /* prism_launch_mode (GMRES solvers; CG ignores it).  No reference
                                     counterpart. */
} prism_solve_opts;

typedef struct prism_solve_stats {
    int32_t num_iter;             /* getNumIter(): CG m+1 (CG.cpp:81); GMRES k*m+m_final (GMRES.cpp:218) */
    int32_t converged;            /* getConvergence() */
    double final_error;           /* getError(): recursive residual (CG) / Givens estimate (GMRES) */
    double true_rel_residual;     /* ||b - A x||_2 / ||b||_2 recomputed in FP64 at exit */
    uint32_t precond_applies;     /* number of M^{-1} applications performed */
    uint32_t spmv_count;          /* number of A x products performed */
    double device_ms;             /* device time of the solve (CUDA events on the handle's stream) */
    double forward_error;         /* ||x - x_ref||_2 / ||x_ref||_2 in FP64 when opts.x_ref is given, else -1
                                     (measured after the solve, outside device_ms) */
    uint32_t host_syncs;          /* times the host waited for the device between the solve's first
                                     and last device operation (CG: once per iteration; GMRES: once
                                     per restart cycle with the cycle graph, once per Arnoldi step
                                     with plain launches; block and batch solves: 0, not counted) */
    uint32_t graph_nodes;         /* GMRES: nodes of the captured Arnoldi step replayed by the cycle
                                     graph (0: plain launches) */
} prism_solve_stats;

typedef struct prism_handle_s* prism_handle;

/* ---- diagnostics ------------------------------------------------------- */
const char* prism_last_error(void);
int32_t prism_version(void);
/* number of kernel launches issued by this library in this process (all handles) */
uint64_t prism_kernel_launch_count(void);

/* Failure-detection self test of the bounded device waits: runs, on one warp,
 * a two-row triangular sweep whose first row waits for a value nothing
 * produces.  The wait gives up after wait_ns (<= 2 s) and the kernel returns
 * with status PRISM_ERR_TIMEOUT, which is stored in *device_status; the call
 * then runs a valid sweep to show the context is still usable.  No reference
 * counterpart (the reference has no device-side waits). */
int32_t prism_selftest_wait_timeout(int32_t device, uint64_t wait_ns, int32_t* device_status);

/* Host self test of the streamed round layout of the triangular sweep kernel:
 * builds the sweep of the gather-form CSR (row r lists its dependencies and
 * coefficients; lower != 0: dependencies precede the row, else follow it),
 * with diag (may be null for op 2), op = 0: (in - s)/d, 1: (in - s)*d,
 * 2: in - s, 3: in/d - s, factor values in `precision`, cuts it into
 * num_ctas slabs of rows_per_cta rows (rows_per_cta = 0: the slab boundaries
 * the device layout chooses), and replays the kernel's decoding of every
 * record on the host into out.  PRISM_ERR_ARG with the reason when the
 * layout is inconsistent.  No reference counterpart (the reference solves
 * sequentially, IncompleteLDLT.cpp:188-233). */
int32_t prism_selftest_stream_layout(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
                                     const double* diag, int32_t op, int32_t lower, int32_t precision,
                                     uint32_t num_ctas, uint32_t rows_per_cta, const double* in, double* out);
/* The same with rounds cut short where their record would exceed
 * max_round_bytes (0: no cap), as the device layout does when four of its
 * largest records do not fit the ring; *record_bytes (may be NULL) receives
 * the largest record of the layout. */
int32_t prism_selftest_stream_layout_capped(uint32_t n, const uint32_t* rowptr, const uint32_t* col,
                                            const double* val, const double* diag, int32_t op, int32_t lower,
                                            int32_t precision, uint32_t num_ctas, uint32_t rows_per_cta,
                                            uint32_t max_round_bytes, const double* in, double* out,
                                            uint32_t* record_bytes);

/* The low-rank correction of an AMSED / MSLR level on a block of k <= 64
 * right-hand sides, alone on `device` with host arrays: Y += W (H o (W^T X)),
 * W column-major nrem x rank (rank <= 128), H of length rank, X and Y
 * interleaved (X[i * k + c]).  tensor != 0: W, X and the intermediate
 * T = H o (W^T X) rounded to BF16 (through float, round to nearest even),
 * both products on the tensor cores with FP32 accumulation, Y updated in FP64
 * (the block apply's path with FP32 factor values); tensor == 0: FP64
 * throughout (the path with FP64 factor values).  Reference:
 * AMSEDPrecondition.cpp:1557-1574 (DenseMatrix::transposeVec / MatVec,
 * DenseMatrix.cpp:208-267), one column at a time. */
int32_t prism_lowrank_block_run(int32_t device, uint32_t nrem, uint32_t rank, uint32_t k, const double* W,
                                const double* H, const double* X, double* Y, int32_t tensor);

/* The summation order of the streamed sweep kernel, for checking its
 * arithmetic against the oracle.  For a gather-form triangular sweep given as
 * for prism_selftest_stream_layout (row r lists its dependencies on one side
 * of the diagonal) laid out in at most num_ctas slabs: for each row r,
 * [eptr[r], eptr[r+1]) of edep/ecoef are its "early" positions and
 * [kptr[r], kptr[r+1]) of kdep/kcoef its "late" ones, in the order the kernel
 * sums them (dependency row, or 0xFFFFFFFF for a padding position with
 * coefficient 0).  The kernel's sum of row r is
 *   c_i = fma chains over early positions p = 4g + i  (c_i = fma(coef, x, c_i)),
 *   s = (c0 + c1) + (c2 + c3), then s = fma(coef, x, s) over the late positions,
 * in float for PRISM_FP32_APPLY, else in double; then op 0/1: (in - s) * d,
 * 2: in - s, 3: in * d - s with d = 1 / diag (ops 0, 3) or diag (op 1).
 * eptr and kptr (n + 1 each) are always filled; edep/ecoef/kdep/kcoef may be
 * NULL (sizes only).  No reference counterpart (the reference sums each row
 * in stored order, IncompleteLDLT.cpp:188-233). */
int32_t prism_stream_sweep_order(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
                                 const double* diag, int32_t op, int32_t lower, int32_t precision, uint32_t num_ctas,
                                 uint32_t* eptr, uint32_t* edep, double* ecoef, uint32_t* kptr, uint32_t* kdep,
                                 double* kcoef);
/* Runs the streamed sweep kernel alone on `device` for the same sweep and
 * slabs as prism_stream_sweep_order (host in and out): out = T^{-1} in. */
/* Wavefront pairing of a gather-form sweep (host only): the same solve in
 * about half as many wavefronts.  A row on an odd wavefront 2R+1 has its
 * dependencies on wavefront 2R substituted by their own rows, so the paired
 * sweep T' (prow/pcol/pval, gather form, the rows' dependencies in increasing
 * order) and the right-hand side map M (mptr/mdep/mcoef) satisfy
 *   T^{-1} b = T'^{-1} b',  b'_r = b_r - sum m b_dep, in stored order, one
 * fused multiply-add each, in double.  *pnnz and *mnnz receive the sizes; pass
 * NULL arrays to query them.  The values are computed in double and rounded to
 * the precision's value type (float unless PRISM_FP64).  No reference
 * counterpart: the reference's sweeps run row by row. */
int32_t prism_stream_sweep_pair(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
                                const double* diag, int32_t op, int32_t lower, int32_t precision, uint64_t* pnnz,
                                uint32_t* prow, uint32_t* pcol, double* pval, uint64_t* mnnz, uint32_t* mptr,
                                uint32_t* mdep, double* mcoef);
int32_t prism_stream_sweep_run(int32_t device, uint32_t n, const uint32_t* rowptr, const uint32_t* col,
                               const double* val, const double* diag, int32_t op, int32_t lower, int32_t precision,
                               uint32_t num_ctas, const double* in, double* out);

/* True residual norms of k right-hand sides without any allocation.  No
 * counterpart in the reference (its solvers only report the recursive
 * residual, source/Solver/CG.cpp:58).  For callers that cannot let a library
 * call cudaMalloc/cudaFree: a framework whose pool allocator owns the device
 * memory, a process at the edge of device memory, or a loop on a
 * latency-sensitive stream that a cudaMalloc/cudaFree synchronization would
 * stall.  Computes, for c < k,
 *   norms_d[2c]   = || b_c - A x_c ||_2,   norms_d[2c+1] = || b_c ||_2,
 * with A given as device CSR arrays (rowptr_d[n+1], col_d[nnz], val_d[nnz])
 * and x, b as k column-major columns of leading dimension ld (ignored for
 * k = 1).  All pointers are caller-owned device memory on `device`; the
 * kernel is queued on `stream` (a cudaStream_t, NULL = legacy default) and the
 * call returns without synchronizing.  Scratch is a fixed 151,808-byte
 * __device__ array per device, so 1 <= k <= 16; larger k is rejected with
 * PRISM_ERR_ARG.  Calls that may overlap on the same device (unordered
 * streams, other threads) race on that scratch: order them.  The first call
 * on a device sets up the scratch address; make it before any stream capture
 * begins.  On success nothing is allocated. */
int32_t prism_residual_norms_noalloc(int32_t device, uint32_t n, const uint32_t* rowptr_d, const uint32_t* col_d,
                                     const double* val_d, const double* x_d, const double* b_d, uint32_t k,
                                     uint64_t ld, double* norms_d, void* stream);

/* ---- model problems (host) --------------------------------------------- */
/* sizes of generateLaplacianCSR(nx,ny,nz,...): n = nx*ny*nz, nnz exact */
int32_t prism_laplacian_dims(int32_t nx, int32_t ny, int32_t nz, uint32_t* n, uint32_t* nnz);
/* fills caller buffers (rowptr[n+1], col[nnz], val[nnz]) exactly as
 * generateLaplacianCOO + transCOO2CSR (ModelProblem.cpp:68-133, MatrixTools.h:16-62) */
int32_t prism_laplacian_fill(int32_t nx, int32_t ny, int32_t nz, double alphax, double alphay,
                             double alphaz, double shift, uint32_t* rowptr, uint32_t* col, double* val);

/* ---- Matrix Market files (host) ------------------------------------------
 * HOST::ReadMtxTools::loadMatrix / loadRightHand
 * (source/utils/TestTools/ReadMtxTools.cpp:50-453) restated: a "coordinate"
 * real file (complex: part 0 the real part, part 1 the imaginary part, each
 * with its own pattern; pattern and integer files are refused), entries with
 * |value| <= 10 * DBL_EPSILON not stored, indices shifted by `base` (1 for
 * Matrix Market), "symmetric" files expanded to the full matrix and
 * "skew-symmetric" ones mirrored with the opposite sign, each row ordered by
 * column (transCOO2CSR, include/MatrixClass/MatrixTools.h:16-62).  Pass NULL
 * arrays to get the sizes first.  prism_mtx_read_dense reads an "array" real
 * file (right-hand sides), rows x cols values in column order. */
int32_t prism_mtx_read(const char* path, int32_t base, int32_t part, uint32_t* rows, uint32_t* cols, uint64_t* nnz,
                       uint32_t* rowptr, uint32_t* col, double* val);
int32_t prism_mtx_read_dense(const char* path, uint32_t* rows, uint32_t* cols, double* values);

/* ---- operator ------------------------------------------------------------ */
/* Copies the host CSR to device `device`.  The structure is validated
 * (monotone offsets, columns < n, strictly increasing within a row). */
int32_t prism_create(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
                     int32_t device, prism_handle* out);
int32_t prism_destroy(prism_handle h);
/* Makes the handle issue its work on `stream` (a cudaStream_t) instead of its own stream. */
int32_t prism_set_stream(prism_handle h, void* stream);
int32_t prism_dims(prism_handle h, uint32_t* n, uint64_t* nnz);

/* y = A x on device pointers / host pointers */
int32_t prism_spmv_device(prism_handle h, const double* x_d, double* y_d);
int32_t prism_spmv(prism_handle h, const double* x, double* y);
/* The shape of the handle's SpMV kernel, which prism_create chose by timing each
 * shape on A (PRISM_SPMV_SHAPE = 0..5 names one instead): lanes that share a
 * row and rows each group of lanes takes per pass.  The shape decides only the
 * order of each row's sum.  No reference counterpart (CSRMatrix::MatPVec,
 * include/MatrixClass/CSRMatrix.h:360-395, runs one row per thread). */
int32_t prism_spmv_shape(prism_handle h, int32_t* lanes_per_row, int32_t* rows_per_pass);

/* ---- preconditioners (host setup, bit-exact with the reference; then uploaded) -- */
int32_t prism_set_precond_none(prism_handle h);
int32_t prism_set_precond_ic(prism_handle h, double threshold, int32_t precision);
int32_t prism_set_precond_ildlt(prism_handle h, double tol, int32_t precision);
int32_t prism_set_precond_ilut(prism_handle h, uint32_t lfill, double tol, int32_t precision);
/* getPreconditionNonZeroCount() (BasePreconditon.h:134-136) */
int32_t prism_precond_nnz(prism_handle h, uint64_t* mnnz);
int32_t prism_precond_type(prism_handle h, int32_t* kind);

/* Factor export for parity checks.  which = 0: first stored triangle
 * (IC/ILDLT: L^T by rows; ILUT: L), which = 1: second (ILUT: U).
 * diag receives ILDLT D / ILUT Dinv (may be NULL).  Pass NULL arrays to
 * query sizes only. */
int32_t prism_precond_factor(prism_handle h, int32_t which, uint32_t* n, uint64_t* nnz,
                             uint32_t* rowptr, uint32_t* col, double* val, double* diag);
/* Dependency depth of each triangular sweep (number of wavefronts of the
 * exact integer level schedule): sweep 0 = lower, 1 = upper. */
int32_t prism_precond_levels(prism_handle h, int32_t sweep, uint32_t* num_levels);

/* ---- host-only factors ----------------------------------------------------------
 * The same incomplete factorisations without a device: for callers that
 * build once and attach to several handles, and for host-side parity checks.
 * kind: PRISM_PRECOND_IC (tol = threshold), PRISM_PRECOND_ILUT (lfill, tol),
 * PRISM_PRECOND_ILDLT (tol). */
typedef struct prism_factor_s* prism_factor;
int32_t prism_factor_create(int32_t kind, uint32_t n, const uint32_t* rowptr, const uint32_t* col,
                            const double* val, double tol, uint32_t lfill, int32_t precision,
                            prism_factor* out);
int32_t prism_factor_destroy(prism_factor f);
/* same layout as prism_precond_factor */
int32_t prism_factor_get(prism_factor f, int32_t which, uint32_t* n, uint64_t* nnz, uint32_t* rowptr,
                         uint32_t* col, double* val, double* diag);
/* getPreconditionNonZeroCount() and the wavefront counts of the two sweeps */
int32_t prism_factor_info(prism_factor f, uint64_t* mnnz, uint32_t* lower_levels, uint32_t* upper_levels);
/* attaches a host factor (built for a matrix of the same size) to a handle */
int32_t prism_set_precond_factor(prism_handle h, prism_factor f);

/* ---- AMSED / MSLR (AMSEDPrecondition, include/Preconditioner/AMSEDPrecondition.h:87-540) ----
 * HID ordering by recursive bisection (the METIS calls of MetisTools.h:105-267
 * are replaced by a deterministic level-structure bisection), per-subdomain
 * RCM (vendored genrcm), ILDLT blocks, ICT on the last level, low-rank
 * correction from the classic generalized Lanczos process. */
typedef struct prism_amsed_opts {
    int32_t levels;           /* levelNum (m_nlev_setup) */
    int32_t lanczos_steps;    /* lanczosSteps (AMSED_MSTEPS = 30) */
    int32_t low_rank;         /* lowRankSize (AMSED_RANK = 16): cap of the MSLR (basic) rank */
    double eig_bound;         /* eigCorrectBound (AMSED_EIGVAL_CORRECTION = 0.8) */
    int32_t lowrank_type;     /* 0 AMSEDBasic (MSLR), 1 AMSEDEigenvalueDeflation */
    int32_t lanczos_type;     /* 0 UseClassicLanczos, 1 UseRestartLanczos (Krylov-Schur, up to 3 restarts) */
    int32_t reorder;          /* 0 MatrixReorderNo, 2 MatrixReorderRCM (AMD is not provided) */
    double factor_tol;        /* AMSED_FACTOR_TOLRANCE = 1e-3 */
    uint32_t minsep;          /* AMSED_MINSEP = 3 */
    uint64_t seed;            /* seed of the Lanczos start vector (the reference draws std::random_device) */
} prism_amsed_opts;
void prism_amsed_default_opts(prism_amsed_opts* o);
int32_t prism_set_precond_amsed(prism_handle h, const prism_amsed_opts* o, int32_t precision);
int32_t prism_factor_create_amsed(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
                                  const prism_amsed_opts* o, int32_t precision, prism_factor* out);
/* structure export for parity checks (arrays may be NULL to query sizes) */
int32_t prism_amsed_info(prism_factor f, uint32_t* nlev, uint32_t* lev_ptr, uint32_t* ncomps, uint32_t* ranks,
                         uint64_t* mnnz);
int32_t prism_amsed_perm(prism_factor f, uint32_t* pperm);
int32_t prism_amsed_dom_ptr(prism_factor f, int32_t level, uint32_t* dom_ptr);
/* block factor of (level, block): ILDLT unit L^T + D, or (last level, block 0) IC L^T */
int32_t prism_amsed_block(prism_factor f, int32_t level, int32_t block, uint32_t* n, uint64_t* nnz,
                          uint32_t* rowptr, uint32_t* col, double* val, double* diag);
/* which = 0: E (level rows x C columns), 1: C block (AMSED), 2: F (GMSLR) */
int32_t prism_amsed_coupling(prism_factor f, int32_t level, int32_t which, uint32_t* nrows, uint64_t* nnz,
                             uint32_t* rowptr, uint32_t* col, double* val);
int32_t prism_amsed_lowrank(prism_factor f, int32_t level, uint32_t* rank, uint32_t* nrem, double* W, double* H);

/* ---- GMSLR (GMSLRPrecondition, include/Preconditioner/GMSLRPrecondition.h:45-411) ----
 * Same HID ordering and level structure as AMSED; ILUT(lfill = 20, factor_tol)
 * blocks on every level (factor_tol default 1e-2 = GMSLR_FACTOR_TOLRANCE) and
 * the coupling x2 -= F x1 with F = A(C rows, B columns).  Options reuse
 * prism_amsed_opts (levels, lanczos_steps, low_rank, reorder, factor_tol,
 * minsep); the structure exports above apply, prism_amsed_coupling with
 * which = 2 returns F, and ranks report min(lanczos_steps, low_rank). */
void prism_gmslr_default_opts(prism_amsed_opts* o);
int32_t prism_set_precond_gmslr(prism_handle h, const prism_amsed_opts* o, int32_t precision);
int32_t prism_factor_create_gmslr(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
                                  const prism_amsed_opts* o, int32_t precision, prism_factor* out);
/* ILUT factor of (level, block): which = 0 L, 1 U; dinv receives the inverse pivots */
int32_t prism_gmslr_block(prism_factor f, int32_t level, int32_t block, int32_t which, uint32_t* n,
                          uint64_t* nnz, uint32_t* rowptr, uint32_t* col, double* val, double* dinv);

/* out = M^{-1} in (in == out allowed) */
int32_t prism_apply_device(prism_handle h, const double* in_d, double* out_d);
int32_t prism_apply(prism_handle h, const double* in, double* out);

/* One triangular sweep alone (IC/ILUT/ILDLT: sweep 0 = lower, 1 = upper;
 * AMSED: sweep 2*level + 0/1 = lower/upper sweep of that HID level's
 * block-diagonal factor, whose rows are numbered from the level's first row),
 * on device vectors,
 * for timing the sweep kernel by itself (the preconditioner apply is
 * prism_apply_device).  prepare = 1: mark out_d pending (the sweep's readiness
 * encoding) then sweep; 0: sweep only (the caller marked out_d already);
 * 2: mark out_d pending only.  prism_precond_sweep_info reports the sweep's
 * rows, stored non-zeros, bytes per stored value, wavefront count and the
 * kernel the setup-time autotuner kept (1: level-ordered grid-wide sweep,
 * 2: slab-blocked sweep with shared-memory dependencies). */
int32_t prism_precond_sweep_device(prism_handle h, int32_t sweep, const double* in_d, double* out_d,
                                   int32_t prepare);
int32_t prism_precond_sweep_info(prism_handle h, int32_t sweep, uint32_t* n, uint64_t* nnz,
                                 uint32_t* value_bytes, uint32_t* num_levels, uint32_t* kernel);

/* The summation order of one of the handle's sweeps (numbered as for
 * prism_precond_sweep_device) when it runs the streamed kernel, in the form of
 * prism_stream_sweep_order, rows numbered as the sweep's, together with the
 * sweep itself: diag (n, may be NULL) its per-row diagonal as stored (d of the
 * sum's last step is 1 / diag for ops 0 and 3), *op and *lower (may be NULL).
 * *n receives the sweep's rows; pass NULL eptr and kptr to query it alone.
 * PRISM_ERR_UNSUPPORTED when the sweep runs another kernel.  No reference
 * counterpart; for checking the kernel against the oracle. */
int32_t prism_precond_sweep_order(prism_handle h, int32_t sweep, uint32_t* n, uint32_t* eptr, uint32_t* edep,
                                  double* ecoef, uint32_t* kptr, uint32_t* kdep, double* kcoef, double* diag,
                                  int32_t* op, int32_t* lower);
/* The right-hand side map of a streamed sweep the autotuner kept paired (see
 * prism_stream_sweep_pair; the order above is then the paired sweep's):
 * *paired 1 or 0, *mnnz its entries (0 when not paired), mptr (n + 1), mdep and
 * mcoef filled when not NULL. */
int32_t prism_precond_sweep_rhs_map(prism_handle h, int32_t sweep, int32_t* paired, uint64_t* mnnz, uint32_t* mptr,
                                    uint32_t* mdep, double* mcoef);

/* ---- solvers ------------------------------------------------------------- */
/* x is the in/out initial guess, as BaseSolver::solve (BaseSolver.h:16). */
int32_t prism_solve_device(prism_handle h, const prism_solve_opts* opts, const double* b_d, double* x_d,
                           prism_solve_stats* stats);
int32_t prism_solve(prism_handle h, const prism_solve_opts* opts, const double* b, double* x,
                    prism_solve_stats* stats);

/* ---- new values on the same pattern, and the adjoint solve ---------------
 * prism_update_values*: A's values replaced (same rowptr/col); the
 * preconditioner is kept as it was until a prism_set_precond_* call sets it
 * up again or prism_refactor recomputes it (a solve stays exact with a stale
 * preconditioner, only slower).  No reference counterpart: the reference
 * builds a new CSRMatrix.
 *
 * prism_refactor: the IC / ILDLT factor recomputed on the device for A's
 * current values, on the factor's own pattern (no new fill, no dropping), in
 * the operation order of the host factorisation (IncompleteCholesky::setup,
 * IncompleteCholesky.cpp:96-246; IncompleteLDLT::setup,
 * IncompleteLDLT.cpp:39-186), which the host recorded when it built the
 * factor: with the values the factor was built from, the result is the host
 * factor bit for bit.  The new values go into every device layout of the
 * preconditioner's sweeps.  PRISM_ERR_NOT_SPD / PRISM_ERR_ZERO_PIVOT as the
 * host factorisation reports them; PRISM_ERR_UNSUPPORTED for ILUT, AMSED and
 * GMSLR.
 *
 * prism_adjoint_solve*: the backward pass of x = A^{-1} b for a scalar loss L
 * with g = dL/dx:  lambda = A^{-T} g  (= dL/db), solved with the handle's
 * solver and preconditioner from a zero guess, and, when grad_val is not
 * null, dL/dA on A's stored pattern:  grad_val[k] = -lambda[i] x[j] for the
 * k-th stored entry (i, j).  A must equal A^T exactly (checked once per set
 * of values; PRISM_ERR_UNSUPPORTED otherwise).  No reference counterpart. */
int32_t prism_update_values(prism_handle h, const double* val);
int32_t prism_update_values_device(prism_handle h, const double* val_d);
int32_t prism_refactor(prism_handle h);
int32_t prism_adjoint_solve_device(prism_handle h, const prism_solve_opts* opts, const double* g_d, const double* x_d,
                                   double* lambda_d, double* grad_val_d, prism_solve_stats* stats);
int32_t prism_adjoint_solve(prism_handle h, const prism_solve_opts* opts, const double* g, const double* x,
                            double* lambda, double* grad_val, prism_solve_stats* stats);

/* ---- blocks of right-hand sides ----------------------------------------
 * k (1..64) right-hand sides that share A and M, stored column-major with
 * leading dimension ld >= n (ignored when k = 1).  Each column is solved with
 * the recurrence of CG<double>::solve (source/Solver/CG.cpp:34-83), the same
 * one prism_solve runs for it alone; a column stops changing once it has
 * converged, and stats[c] (k entries) reports its own iteration count, error
 * and true residual.  The reference solves one right-hand side per call; a
 * block here shares every sweep's dependency latency among its k columns.
 * Block solves use FCG / CG (PRISM_ERR_UNSUPPORTED otherwise) and an IC /
 * ILDLT / ILUT preconditioner or none. */
int32_t prism_apply_batched_device(prism_handle h, uint32_t k, const double* in_d, double* out_d, uint64_t ld);
int32_t prism_solve_batched_device(prism_handle h, const prism_solve_opts* opts, uint32_t k, const double* B_d,
                                   double* X_d, uint64_t ld, prism_solve_stats* stats);
int32_t prism_solve_batched(prism_handle h, const prism_solve_opts* opts, uint32_t k, const double* B, double* X,
                            uint64_t ld, prism_solve_stats* stats);

/* ---- batches of independent systems -------------------------------------
 * The handle's matrix holds nseg independent systems on its diagonal: rows
 * [seg_ptr[s], seg_ptr[s+1]) couple only among themselves (PRISM_ERR_ARG
 * otherwise; seg_ptr is a host array of nseg + 1 offsets from 0 to n).  Any
 * IC / ILDLT / ILUT preconditioner set on the handle is then block diagonal
 * too, and one SpMV and one pair of sweeps serve all systems.  Each system is
 * solved with the recurrence of CG<double>::solve (source/Solver/CG.cpp:34-83)
 * on its own scalars and stops changing once it has converged; stats[s]
 * (nseg entries) reports its own iterations, error and true residual.  A
 * system whose right-hand side is zero is left at x = 0, converged.  FCG / CG
 * only.  The reference solves one system per call. */
int32_t prism_solve_segments_device(prism_handle h, const prism_solve_opts* opts, uint32_t nseg,
                                    const uint32_t* seg_ptr, const double* b_d, double* x_d,
                                    prism_solve_stats* stats);
int32_t prism_solve_segments(prism_handle h, const prism_solve_opts* opts, uint32_t nseg, const uint32_t* seg_ptr,
                             const double* b, double* x, prism_solve_stats* stats);

#ifdef __cplusplus
}
#endif
#endif /* PRISM_SOLVE_H */
