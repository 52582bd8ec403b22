/*
 * CPU oracle of the PrisPack solve phase -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's solve-phase algorithms, used by
 * tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py as the
 * checker.  The product library never links, loads or calls it.
 *
 * Pinning: the restatement is checked against the reference's own compiled
 * sources (oracle/_ref, built by oracle/Makefile) and against golden vectors
 * generated from them (tests/golden/, tests/golden/make_golden.py).
 */
#ifndef PRISM_ORACLE_H
#define PRISM_ORACLE_H
#include <stdint.h>

/* A triangular sweep in the streamed kernel's summation order (arguments of
 * orc_sweep_ordered); used by orc_amsed_apply for the single-precision apply. */
typedef struct orc_sweep_order {
    uint32_t n;
    int op, lower;
    const uint32_t* eptr;
    const uint32_t* edep;
    const double* ecoef;
    const uint32_t* kptr;
    const uint32_t* kdep;
    const double* kcoef;
    const double* diag;
    const uint32_t* mptr;   /* paired sweep: right-hand side map (orc_pair_rhs), else NULL */
    const uint32_t* mdep;
    const double* mcoef;
} orc_sweep_order;

/* One level of an AMSED/MSLR hierarchy (LevelStructure,
 * include/Preconditioner/AMSEDPrecondition.h:75-85) in permuted numbering. */
typedef struct orc_amsed_level {
    uint32_t ncomps;
    const uint32_t* dom_ptr;          /* ncomps + 1 global offsets */
    const uint32_t* const* blk_rp;    /* per block: ILDLT unit L^T (last level: block 0 IC L^T) */
    const uint32_t* const* blk_ci;
    const double* const* blk_val;
    const double* const* blk_diag;    /* per block: ILDLT pivots (unused on the last level) */
    const uint32_t* e_rp;             /* E: this level's B rows x its C columns (non-last levels) */
    const uint32_t* e_ci;
    const double* e_val;
    uint32_t rank;
    const double* W;                  /* nrem x rank, column-major */
    const double* H;
    /* GMSLR: ILUT blocks (blk_* = L) and F = A(C rows, B cols) */
    const uint32_t* const* blk_rp1;   /* per block: U */
    const uint32_t* const* blk_ci1;
    const double* const* blk_val1;
    const uint32_t* f_rp;
    const uint32_t* f_ci;
    const double* f_val;
    /* when set, the level's block solve is these two kernel-order sweeps over its
     * first sweep_lo->n rows (orc_amsed.single selects float arithmetic) */
    const orc_sweep_order* sweep_lo;
    const orc_sweep_order* sweep_up;
} orc_amsed_level;

typedef struct orc_amsed {
    uint32_t n, nlev;
    int gmslr;                        /* 0: AMSED, 1: GMSLR */
    int single;                       /* kernel-order sweeps (levels' sweep_lo/up) in float */
    const uint32_t* pperm;            /* new -> original */
    const uint32_t* lev_ptr;          /* nlev + 1 */
    const orc_amsed_level* levels;
} orc_amsed;

/* AMSEDPrecondition::MInvSolve(vec) (AMSEDPrecondition.cpp:2063-2087), in place */
void orc_amsed_apply(const orc_amsed* S, double* vec);

/* preconditioner described by its stored factor arrays (values widened to double) */
typedef struct orc_precond {
    int kind;                 /* 0 none, 1 IC, 2 ILUT, 3 ILDLT, 5 AMSED (amsed != NULL) */
    uint32_t n;
    const uint32_t* rp0;      /* IC/ILDLT: L^T rows; ILUT: L rows */
    const uint32_t* ci0;
    const double* v0;
    const uint32_t* rp1;      /* ILUT: U rows */
    const uint32_t* ci1;
    const double* v1;
    const double* diag;       /* ILDLT: D; ILUT: Dinv */
    const orc_amsed* amsed;
} orc_precond;

void orc_laplacian(int nx, int ny, int nz, double ax, double ay, double az, double shift,
                   uint32_t* rowptr, uint32_t* col, double* val);
void orc_spmv(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
              const double* x, double* y);
/* a gather-form triangular sweep in single precision, reference order (see oracle.c) */
void orc_sweep_f32(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
                   const double* diag, int op, int lower, const double* in, double* out);
/* a gather-form triangular sweep in the streamed kernel's summation order (see oracle.c) */
void orc_pair_rhs(uint32_t n, const uint32_t* mptr, const uint32_t* mdep, const double* mcoef, const double* in,
                  double* out);
void orc_sweep_ordered(uint32_t n, int single, int op, int lower, const uint32_t* eptr, const uint32_t* edep,
                       const double* ecoef, const uint32_t* kptr, const uint32_t* kdep, const double* kcoef,
                       const double* diag, const double* in, double* out);
/* IC (kind 1) / ILDLT (kind 3) factor values recomputed on a given pattern (see oracle.c) */
int orc_refactor(uint32_t n, int kind, const uint32_t* a_rowptr, const uint32_t* a_col, const double* a_val,
                 const uint32_t* lt_rowptr, const uint32_t* lt_col, int single, double* lt_val, double* D);
void orc_precond_apply(const orc_precond* P, double* vec);
void orc_cg(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
            const orc_precond* P, int flexible, double tol, uint32_t max_iter,
            const double* b, double* x, int32_t* num_iter, double* final_error, int32_t* converged);
void orc_gmres(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
               const orc_precond* P, int flexible, uint32_t restart, double tol,
               const double* b, double* x, int32_t* num_iter, double* final_error, int32_t* converged);
#endif
