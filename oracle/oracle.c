/*
 * CPU oracle of the PrisPack solve phase -- TEST INFRASTRUCTURE ONLY.
 * Parity is pinned against the reference's compiled sources (oracle/_ref) and
 * the golden vectors in tests/golden/.  Never linked into the product.
 *
 * Every routine restates one reference routine, in the same operation order,
 * serially (the reference's OpenMP reductions are order-nondeterministic; the
 * serial order is its single-thread behaviour).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* generateLaplacianCOO (source/MatrixClass/ModelProblem.cpp:68-133) followed by
 * transCOO2CSR's per-row insertion sort (include/MatrixClass/MatrixTools.h:16-62). */
void orc_laplacian(int nx, int ny, int nz, double ax, double ay, double az, double shift,
                   uint32_t* rowptr, uint32_t* col, double* val) {
    int numones = (nx == 1) + (ny == 1) + (nz == 1);
    double v = -1.0;
    double vxp = v - ax, vxn = v + ax, vyp = v - ay, vyn = v + ay, vzp = v - az, vzn = v + az;
    double vd = numones > 0 ? 4.0 : 6.0;
    vd -= shift;
    long n = (long)nx * ny * nz, pos = 0;
    rowptr[0] = 0;
    for (long ii = 0; ii < n; ii++) {
        long k = ii / ((long)nx * ny);
        long i = (ii - k * nx * ny) / nx;
        long j = ii - k * nx * ny - i * nx;
        long c[7];
        double w[7];
        int m = 0;
        if (k > 0) { c[m] = ii - (long)nx * ny; w[m++] = vzn; }
        if (k < nz - 1) { c[m] = ii + (long)nx * ny; w[m++] = vzp; }
        if (i > 0) { c[m] = ii - nx; w[m++] = vyn; }
        if (i < ny - 1) { c[m] = ii + nx; w[m++] = vyp; }
        if (j > 0) { c[m] = ii - 1; w[m++] = vxn; }
        if (j < nx - 1) { c[m] = ii + 1; w[m++] = vxp; }
        c[m] = ii; w[m++] = vd;
        /* sortVectorPair: insertion sort by column (include/VectorClass/VectorTools.h:39-57) */
        for (int a = 1; a < m; a++) {
            long key = c[a]; double kv = w[a]; int b = a - 1;
            while (b >= 0 && c[b] > key) { c[b + 1] = c[b]; w[b + 1] = w[b]; b--; }
            c[b + 1] = key; w[b + 1] = kv;
        }
        for (int a = 0; a < m; a++) { col[pos] = (uint32_t)c[a]; val[pos] = w[a]; pos++; }
        rowptr[ii + 1] = (uint32_t)pos;
    }
}

/* CSRMatrix::MatPVecWithRawPtr (include/MatrixClass/CSRMatrix.h:360-377) */
void orc_spmv(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
              const double* x, double* y) {
    for (uint32_t i = 0; i < n; i++) {
        double s = 0;
        for (uint32_t j = rowptr[i]; j < rowptr[i + 1]; j++) s += x[col[j]] * val[j];
        y[i] = s;
    }
}

/* One triangular sweep in gather form, in single precision, in the reference's
 * order: row r (in dependency order: increasing for a lower sweep, decreasing
 * for an upper one) sums its entries in stored order, as IncompleteLDLT.cpp:
 * 188-233 and IncompleteCholesky.cpp:249-295 do, s += val[k] * out[col[k]],
 * each value, product and sum rounded to float, and
 *   op 0: (in - s) / diag   op 1: (in - s) * diag   op 2: in - s   op 3: in / diag - s
 * with in and diag rounded to float first; out holds the float results
 * widened to double.  This is a tolerance reference for the library's
 * single-precision apply, whose kernel sums in another order (see
 * orc_sweep_ordered for that order). */
void orc_sweep_f32(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
                   const double* diag, int op, int lower, const double* in, double* out) {
    float* x = (float*)malloc(sizeof(float) * (n ? n : 1));
    for (uint32_t t = 0; t < n; t++) {
        const uint32_t r = lower ? t : n - 1 - t;
        float s = 0.0f;
        for (uint32_t k = rowptr[r]; k < rowptr[r + 1]; k++) s += (float)val[k] * x[col[k]];
        const float b = (float)in[r], d = diag ? (float)diag[r] : 1.0f;
        float res;
        if (op == 0) res = (b - s) / d;
        else if (op == 1) res = (b - s) * d;
        else if (op == 2) res = b - s;
        else res = b / d - s;
        x[r] = res;
        out[r] = (double)res;
    }
    free(x);
}

/* The right-hand side of a paired sweep (the library's wavefront pairing, no
 * reference counterpart): out[r] = in[r] - sum m in[dep] over [mptr[r],
 * mptr[r+1]), in stored order, each step one fused multiply-add in double. */
void orc_pair_rhs(uint32_t n, const uint32_t* mptr, const uint32_t* mdep, const double* mcoef, const double* in,
                  double* out) {
    for (uint32_t r = 0; r < n; r++) {
        double v = in[r];
        for (uint32_t q = mptr[r]; q < mptr[r + 1]; q++) v = fma(-mcoef[q], in[mdep[q]], v);
        out[r] = v;
    }
}

/* One triangular sweep in gather form in the summation order of the library's
 * streamed sweep kernel (no reference counterpart: the reference sums each row
 * in stored order).  For row r, [eptr[r], eptr[r+1]) of edep/ecoef are its
 * "early" positions and [kptr[r], kptr[r+1]) of kdep/kcoef its "late" ones; a
 * dependency of 0xFFFFFFFF is padding (value 0).  In the working precision
 * (float when single != 0, else double), every product-sum one fused
 * multiply-add:
 *   c_i = fma(coef, x, c_i) over early positions p with p mod 4 == i, from 0,
 *   s = (c0 + c1) + (c2 + c3),  then s = fma(coef, x, s) over the late positions,
 *   op 0, 1: (in - s) * d    op 2: in - s    op 3: in * d - s,
 * with in rounded to the working precision and d = 1 / diag (ops 0, 3, the
 * division in double) or diag (op 1), then rounded.  Rows run in dependency
 * order (increasing for a lower sweep, decreasing for an upper one); out holds
 * the results widened to double. */
void orc_sweep_ordered(uint32_t n, int single, int op, int lower, const uint32_t* eptr, const uint32_t* edep,
                       const double* ecoef, const uint32_t* kptr, const uint32_t* kdep, const double* kcoef,
                       const double* diag, const double* in, double* out) {
    float* xf = single ? (float*)malloc(sizeof(float) * (n ? n : 1)) : NULL;
    double* xd = single ? NULL : (double*)malloc(sizeof(double) * (n ? n : 1));
    for (uint32_t t = 0; t < n; t++) {
        const uint32_t r = lower ? t : n - 1 - t;
        const double dd = op == 0 || op == 3 ? 1.0 / diag[r] : (op == 1 ? diag[r] : 1.0);
        if (single) {
            float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            for (uint32_t p = eptr[r]; p < eptr[r + 1]; p++) {
                const float x = edep[p] == 0xFFFFFFFFu ? 0.0f : xf[edep[p]];
                c[(p - eptr[r]) & 3] = fmaf((float)ecoef[p], x, c[(p - eptr[r]) & 3]);
            }
            float s = (c[0] + c[1]) + (c[2] + c[3]);
            for (uint32_t p = kptr[r]; p < kptr[r + 1]; p++) {
                const float x = kdep[p] == 0xFFFFFFFFu ? 0.0f : xf[kdep[p]];
                s = fmaf((float)kcoef[p], x, s);
            }
            const float b = (float)in[r], d = (float)dd;
            float res;
            if (op == 0 || op == 1) res = (b - s) * d;
            else if (op == 2) res = b - s;
            else res = b * d - s;
            xf[r] = res;
            out[r] = (double)res;
        } else {
            double c[4] = {0.0, 0.0, 0.0, 0.0};
            for (uint32_t p = eptr[r]; p < eptr[r + 1]; p++) {
                const double x = edep[p] == 0xFFFFFFFFu ? 0.0 : xd[edep[p]];
                c[(p - eptr[r]) & 3] = fma(ecoef[p], x, c[(p - eptr[r]) & 3]);
            }
            double s = (c[0] + c[1]) + (c[2] + c[3]);
            for (uint32_t p = kptr[r]; p < kptr[r + 1]; p++) {
                const double x = kdep[p] == 0xFFFFFFFFu ? 0.0 : xd[kdep[p]];
                s = fma(kcoef[p], x, s);
            }
            const double b = in[r];
            double res;
            if (op == 0 || op == 1) res = (b - s) * dd;
            else if (op == 2) res = b - s;
            else res = b * dd - s;
            xd[r] = res;
            out[r] = res;
        }
    }
    free(xf);
    free(xd);
}

/* Numeric refactorisation of an IC (kind 1) or ILDLT (kind 3) factor on a given
 * pattern: IncompleteCholesky::setup (IncompleteCholesky.cpp:96-246) and
 * IncompleteLDLT::setup (IncompleteLDLT.cpp:39-186) with their drop test
 * (|L_ij| >= threshold * sum of |A_ij|) replaced by "L_ij is kept when (i, j) is in
 * the pattern".  Column j accumulates the entries of row j of A at or below the
 * diagonal, then subtracts L_ik * L_jk (* d_k) for each finished column k of its row
 * list (the reference's vNonZeroRow / vNextIdxRow linked lists), divides the kept
 * entries by the pivot (sqrt of it for IC) and stores them rounded to float when
 * single != 0.  lt_rowptr / lt_col: the pattern of L^T by rows (IC: the diagonal
 * first, ILDLT: no diagonal), rows in increasing order; lt_val receives the values,
 * D (ILDLT) the pivots.  Returns 0, 4 (IC: non-positive pivot) or 3 (ILDLT: zero
 * pivot). */
int orc_refactor(uint32_t n, int kind, const uint32_t* a_rowptr, const uint32_t* a_col, const double* a_val,
                 const uint32_t* lt_rowptr, const uint32_t* lt_col, int single, double* lt_val, double* D) {
    const int ldlt = kind == 3;
    uint8_t* used = (uint8_t*)calloc(n ? n : 1, 1);
    double* colv = (double*)calloc(n ? n : 1, sizeof(double));
    uint32_t* nz_row = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t* next_idx = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t* touched = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    int rc = 0;
    for (uint32_t i = 0; i < n; i++) nz_row[i] = UINT32_MAX;
#define STORE(x) (single ? (double)(float)(x) : (x))
    for (uint32_t j = 0; j < n && !rc; j++) {
        uint32_t cnt = 0;
        for (uint32_t p = a_rowptr[j]; p < a_rowptr[j + 1]; p++) {
            const uint32_t i = a_col[p];
            if (i >= j) {
                if (!used[i]) {
                    colv[i] = 0.0;
                    used[i] = 1;
                    touched[cnt++] = i;
                }
                colv[i] += a_val[p];
            }
        }
        uint32_t k = nz_row[j];
        while (k != UINT32_MAX) {
            uint32_t start = next_idx[k];
            const double Ljk = lt_val[start];
            const double dk = ldlt ? D[k] : 0.0;
            for (uint32_t p = start; p < lt_rowptr[k + 1]; p++) {
                const uint32_t i = lt_col[p];
                if (!used[i]) {
                    used[i] = 1;
                    colv[i] = 0.0;
                    touched[cnt++] = i;
                }
                if (ldlt) colv[i] -= lt_val[p] * Ljk * dk;
                else colv[i] -= lt_val[p] * Ljk;
            }
            start += 1;
            const uint32_t knext = nz_row[k];
            if (start < lt_rowptr[k + 1]) {
                next_idx[k] = start;
                const uint32_t i = lt_col[start];
                nz_row[k] = nz_row[i];
                nz_row[i] = k;
            }
            k = knext;
        }
        double piv = colv[j];
        uint32_t w = lt_rowptr[j];
        if (ldlt) {
            if (fabs(piv) < 1e-15) rc = 3;
            D[j] = piv;
            next_idx[j] = w;
        } else {
            if (piv <= 0.0) rc = 4;
            piv = sqrt(piv);
            lt_val[w++] = STORE(piv);
            next_idx[j] = w;
        }
        /* the kept entries in increasing row order (the pattern's own order) */
        int first = 1;
        for (uint32_t q = w; q < lt_rowptr[j + 1]; q++) {
            const uint32_t i = lt_col[q];
            if (first) {
                first = 0;
                nz_row[j] = nz_row[i];
                nz_row[i] = j;
            }
            lt_val[q] = STORE(colv[i] / piv);
        }
        for (uint32_t t = 0; t < cnt; t++) used[touched[t]] = 0;
    }
#undef STORE
    free(used);
    free(colv);
    free(nz_row);
    free(next_idx);
    free(touched);
    return rc;
}

/* ---- AMSED ----------------------------------------------------------------- */
static void ildlt_inplace(uint32_t n, const uint32_t* rp, const uint32_t* ci, const double* v, const double* D,
                          double* vec) {
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t k = rp[i]; k < rp[i + 1]; k++) vec[ci[k]] -= v[k] * vec[i];
    for (uint32_t i = 0; i < n; i++) vec[i] /= D[i];
    for (uint32_t i = n; i-- > 0;)
        for (uint32_t k = rp[i]; k < rp[i + 1]; k++) vec[i] -= v[k] * vec[ci[k]];
}

static void ic_inplace(uint32_t n, const uint32_t* rp, const uint32_t* ci, const double* v, double* vec) {
    for (uint32_t i = 0; i < n; i++) {
        double t = vec[i] / v[rp[i]];
        vec[i] = t;
        for (uint32_t k = rp[i] + 1; k < rp[i + 1]; k++) vec[ci[k]] -= v[k] * t;
    }
    for (uint32_t i = n; i-- > 0;) {
        double t = vec[i];
        for (uint32_t k = rp[i] + 1; k < rp[i + 1]; k++) t -= v[k] * vec[ci[k]];
        vec[i] = t / v[rp[i]];
    }
}

/* IncompleteLU::MSolveLower/UpperUsePtr (IncompleteLU.cpp:268-297), in place */
static void ilut_inplace(uint32_t n, const uint32_t* lrp, const uint32_t* lci, const double* lv, const uint32_t* urp,
                         const uint32_t* uci, const double* uv, const double* dinv, double* vec) {
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t k = lrp[i]; k < lrp[i + 1]; k++) vec[i] -= lv[k] * vec[lci[k]];
    for (uint32_t i = n; i > 0; i--) {
        for (uint32_t k = urp[i - 1]; k < urp[i]; k++) vec[i - 1] -= uv[k] * vec[uci[k]];
        vec[i - 1] *= dinv[i - 1];
    }
}

/* levelBlockInvSolve (AMSEDPrecondition.cpp:1690-1754, GMSLRDPrecondition.cpp:1170-1229):
 * x starts at the level's first row */
/* the level's block solve as the two kernel-order sweeps (single-precision apply) */
static void amsed_ordered_block_solve(const orc_amsed* S, const orc_amsed_level* L, double* x) {
    const orc_sweep_order* lo = L->sweep_lo;
    const orc_sweep_order* up = L->sweep_up;
    const uint32_t nb = lo->n > up->n ? lo->n : up->n;
    double* t = malloc((size_t)(nb ? nb : 1) * sizeof(double));
    double* b = malloc((size_t)(nb ? nb : 1) * sizeof(double));
    /* a paired sweep's right-hand side first (mptr NULL: not paired) */
    const double* in = x;
    if (lo->mptr) {
        orc_pair_rhs(lo->n, lo->mptr, lo->mdep, lo->mcoef, x, b);
        in = b;
    }
    orc_sweep_ordered(lo->n, S->single, lo->op, lo->lower, lo->eptr, lo->edep, lo->ecoef, lo->kptr, lo->kdep,
                      lo->kcoef, lo->diag, in, t);
    in = t;
    if (up->mptr) {
        orc_pair_rhs(up->n, up->mptr, up->mdep, up->mcoef, t, b);
        in = b;
    }
    orc_sweep_ordered(up->n, S->single, up->op, up->lower, up->eptr, up->edep, up->ecoef, up->kptr, up->kdep,
                      up->kcoef, up->diag, in, x);
    free(b);
    free(t);
}

static void amsed_block_solve(const orc_amsed* S, uint32_t level, double* x) {
    const orc_amsed_level* L = &S->levels[level];
    const int last = level == S->nlev - 1;
    if (L->sweep_lo) {
        amsed_ordered_block_solve(S, L, x);
        return;
    }
    for (uint32_t b = 0; b < L->ncomps; b++) {
        double* seg = x + (L->dom_ptr[b] - L->dom_ptr[0]);
        uint32_t nb = L->dom_ptr[b + 1] - L->dom_ptr[b];
        if (S->gmslr) {
            if (!last || b == 0)
                ilut_inplace(nb, L->blk_rp[b], L->blk_ci[b], L->blk_val[b], L->blk_rp1[b], L->blk_ci1[b],
                             L->blk_val1[b], L->blk_diag[b], seg);
        } else if (last) {
            if (b == 0) ic_inplace(nb, L->blk_rp[0], L->blk_ci[0], L->blk_val[0], seg);
        } else {
            ildlt_inplace(nb, L->blk_rp[b], L->blk_ci[b], L->blk_val[b], L->blk_diag[b], seg);
        }
    }
}

/* levelCInvRecursiveSolve(level, x, .) (AMSEDPrecondition.cpp:1494-1587); x = C block of `level` */
static void amsed_c_solve(const orc_amsed* S, int level, double* x) {
    const int next = level + 1;
    if (level == (int)S->nlev - 2) {
        const orc_amsed_level* LL = &S->levels[S->nlev - 1];
        if (LL->sweep_lo)
            amsed_ordered_block_solve(S, LL, x);
        else if (S->gmslr)
            ilut_inplace(LL->dom_ptr[1] - LL->dom_ptr[0], LL->blk_rp[0], LL->blk_ci[0], LL->blk_val[0], LL->blk_rp1[0],
                         LL->blk_ci1[0], LL->blk_val1[0], LL->blk_diag[0], x);
        else
            ic_inplace(LL->dom_ptr[1] - LL->dom_ptr[0], LL->blk_rp[0], LL->blk_ci[0], LL->blk_val[0], x);
        return;
    }
    const orc_amsed_level* L = &S->levels[next];
    const uint32_t nb = S->lev_ptr[next + 1] - S->lev_ptr[next];
    const uint32_t nrem = S->n - S->lev_ptr[next + 1];
    amsed_block_solve(S, (uint32_t)next, x);
    double* xc = calloc(nrem ? nrem : 1, sizeof(double));
    if (S->gmslr) { /* x_copy = F x1 (GMSLRDPrecondition.cpp:1080) */
        for (uint32_t i = 0; i < nrem; i++) {
            double s = 0;
            for (uint32_t k = L->f_rp[i]; k < L->f_rp[i + 1]; k++) s += x[L->f_ci[k]] * L->f_val[k];
            xc[i] = s;
        }
    } else { /* transMatPVec: scatter in row order */
        for (uint32_t i = 0; i < nb; i++)
            for (uint32_t k = L->e_rp[i]; k < L->e_rp[i + 1]; k++) xc[L->e_ci[k]] += L->e_val[k] * x[i];
    }
    for (uint32_t i = 0; i < nrem; i++) x[nb + i] -= xc[i];
    memcpy(xc, x + nb, nrem * sizeof(double));
    amsed_c_solve(S, next, x + nb);
    if (L->rank > 0) {
        double* t = calloc(L->rank, sizeof(double));
        double* t2 = calloc(nrem ? nrem : 1, sizeof(double));
        for (uint32_t i = 0; i < L->rank; i++) /* DenseMatrix::transposeVec */
            for (uint32_t j = 0; j < nrem; j++) t[i] += L->W[(size_t)i * nrem + j] * xc[j];
        for (uint32_t i = 0; i < L->rank; i++) t[i] *= L->H[i];
        for (uint32_t i = 0; i < L->rank; i++) /* DenseMatrix::MatVec */
            for (uint32_t j = 0; j < nrem; j++) t2[j] += L->W[(size_t)i * nrem + j] * t[i];
        for (uint32_t j = 0; j < nrem; j++) x[nb + j] += t2[j];
        free(t);
        free(t2);
    }
    double* tmp = calloc(nb ? nb : 1, sizeof(double));
    for (uint32_t i = 0; i < nb; i++) { /* MatPVecWithRawPtr */
        double s = 0;
        for (uint32_t k = L->e_rp[i]; k < L->e_rp[i + 1]; k++) s += x[nb + L->e_ci[k]] * L->e_val[k];
        tmp[i] = s;
    }
    amsed_block_solve(S, (uint32_t)next, tmp);
    for (uint32_t i = 0; i < nb; i++) x[i] -= tmp[i];
    free(tmp);
    free(xc);
}

void orc_amsed_apply(const orc_amsed* S, double* vec) {
    double* p = malloc((size_t)S->n * sizeof(double));
    for (uint32_t i = 0; i < S->n; i++) p[i] = vec[S->pperm[i]]; /* prepareRightHand */
    amsed_c_solve(S, -1, p);
    for (uint32_t i = 0; i < S->n; i++) vec[S->pperm[i]] = p[i]; /* recoverRightHand */
    free(p);
}

/* TriangularPrecondition::MInvSolve (include/Preconditioner/BasePreconditon.h:307-315):
 * lower, (ILDLT: diagonal), upper -- in place. */
void orc_precond_apply(const orc_precond* P, double* vec) {
    const uint32_t n = P->n;
    if (P->kind == 5) {
        orc_amsed_apply(P->amsed, vec);
    } else if (P->kind == 1) {
        /* IncompleteCholesky::MSolveLowerUsePtr (IncompleteCholesky.cpp:249-271): column scatter */
        for (uint32_t i = 0; i < n; i++) {
            uint32_t k = P->rp0[i];
            double t = vec[i] / P->v0[k];
            vec[i] = t;
            for (k = P->rp0[i] + 1; k < P->rp0[i + 1]; k++) vec[P->ci0[k]] -= P->v0[k] * t;
        }
        /* MSolveUpperUsePtr (IncompleteCholesky.cpp:274-295): row gather */
        for (uint32_t i = n; i-- > 0;) {
            double t = vec[i];
            for (uint32_t k = P->rp0[i] + 1; k < P->rp0[i + 1]; k++) t -= P->v0[k] * vec[P->ci0[k]];
            vec[i] = t / P->v0[P->rp0[i]];
        }
    } else if (P->kind == 3) {
        /* IncompleteLDLT lower (IncompleteLDLT.cpp:216-233), diagonal (:206-214), upper (:188-204) */
        for (uint32_t i = 0; i < n; i++)
            for (uint32_t k = P->rp0[i]; k < P->rp0[i + 1]; k++) vec[P->ci0[k]] -= P->v0[k] * vec[i];
        for (uint32_t i = 0; i < n; i++) vec[i] /= P->diag[i];
        for (uint32_t i = n; i-- > 0;)
            for (uint32_t k = P->rp0[i]; k < P->rp0[i + 1]; k++) vec[i] -= P->v0[k] * vec[P->ci0[k]];
    } else if (P->kind == 2) {
        /* IncompleteLU lower (IncompleteLU.cpp:284-297), upper (:268-282) */
        for (uint32_t i = 0; i < n; i++)
            for (uint32_t k = P->rp0[i]; k < P->rp0[i + 1]; k++) vec[i] -= P->v0[k] * vec[P->ci0[k]];
        for (uint32_t i = n; i > 0; i--) {
            for (uint32_t k = P->rp1[i - 1]; k < P->rp1[i]; k++) vec[i - 1] -= P->v1[k] * vec[P->ci1[k]];
            vec[i - 1] *= P->diag[i - 1];
        }
    }
}

static double dot(uint32_t n, const double* a, const double* b) {
    double s = 0.0; /* BaseVector::innerProduct serial branch (BaseVector.h:429-448) */
    for (uint32_t i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

/* CG<double>::solve (source/Solver/CG.cpp:34-83), including the second
 * v = A d at the top of every iteration. */
void orc_cg(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
            const orc_precond* P, int flexible, double tol, uint32_t max_iter,
            const double* b, double* x, int32_t* num_iter, double* final_error, int32_t* converged) {
    double* r = calloc(n, sizeof(double));
    double* v = calloc(n, sizeof(double));
    double* w = calloc(n, sizeof(double));
    double* d = calloc(n, sizeof(double));
    int has_p = P && P->kind != 0;
    *converged = 0;
    uint32_t m = max_iter;
    double norm_b = sqrt(dot(n, b, b)), norm = -1.0, v1, v2;
    orc_spmv(n, rowptr, col, val, x, r);
    for (uint32_t i = 0; i < n; i++) w[i] = 1 * b[i] + -1 * r[i];
    memcpy(r, w, n * sizeof(double));
    if (has_p) orc_precond_apply(P, w);
    memcpy(d, w, n * sizeof(double));
    orc_spmv(n, rowptr, col, val, d, v);
    v1 = dot(n, d, r);
    v2 = dot(n, d, v);
    v1 /= v2;
    for (uint32_t i = 0; i < n; i++) x[i] = 1 * x[i] + v1 * d[i];
    for (uint32_t i = 0; i < n; i++) r[i] = 1 * r[i] + -v1 * v[i];
    for (uint32_t it = 1; it < max_iter; it++) {
        norm = sqrt(dot(n, r, r)) / norm_b;
        if (norm < tol) { *converged = 1; m = it; break; }
        memcpy(w, r, n * sizeof(double));
        if (flexible && has_p) orc_precond_apply(P, w);
        orc_spmv(n, rowptr, col, val, d, v);
        v1 = dot(n, w, v);
        v2 = dot(n, d, v);
        v1 = v1 / v2;
        for (uint32_t i = 0; i < n; i++) d[i] = 1 * w[i] + -v1 * d[i];
        v1 = dot(n, d, r);
        orc_spmv(n, rowptr, col, val, d, v);
        v2 = dot(n, d, v);
        v1 = v1 / v2;
        for (uint32_t i = 0; i < n; i++) x[i] = 1 * x[i] + v1 * d[i];
        for (uint32_t i = 0; i < n; i++) r[i] = 1 * r[i] + -v1 * v[i];
    }
    *num_iter = (int32_t)(m + 1);
    *final_error = norm;
    free(r); free(v); free(w); free(d);
}

/* Kahan-compensated Σ x² as BaseVector::sumKahan(start, len, func) (BaseVector.h:635-648) */
static double sum_sq_kahan(uint32_t n, const double* x) {
    double s = 0.0, c = 0.0, t, ns;
    for (uint32_t i = 0; i < n; i++) {
        t = x[i] * x[i] + c;
        ns = s + t;
        c = t - (ns - s);
        s = ns;
    }
    return s + c;
}

/* GMRES<double>::givensTransform (source/Solver/GMRES.cpp:73-101); H column-major (m+1) x m */
static void givens(double* H, uint32_t ld, double* c, double* s, double* ksi, uint32_t j) {
    double val0, val1, val2, tao;
    for (uint32_t i = 0; i < j; i++) {
        val1 = H[i + j * ld];
        val2 = H[i + 1 + j * ld];
        val0 = c[i] * val2 - s[i] * val1;
        H[i + 1 + j * ld] = val0;
        val0 = c[i] * val1 + s[i] * val2;
        H[i + j * ld] = val0;
    }
    val1 = H[j + j * ld];
    val2 = H[j + 1 + j * ld];
    if (fabs(val1) > fabs(val2)) {
        tao = val2 / val1;
        c[j] = 1 / sqrt(fabs(1.0 + tao * tao));
        s[j] = c[j] * tao;
    } else {
        tao = val1 / val2;
        s[j] = 1 / sqrt(fabs(1.0 + tao * tao));
        c[j] = s[j] * tao;
    }
    H[j + j * ld] = c[j] * val1 + s[j] * val2;
    H[j + 1 + j * ld] = 0.0;
    ksi[j + 1] = -s[j] * ksi[j];
    ksi[j] = c[j] * ksi[j];
}

/* GMRES<double>::solve (source/Solver/GMRES.cpp:122-221) with setRestart
 * (GMRES.cpp:60-70) when restart > 0; MAX_ITER_NUM_SOLVER = 500 (config/config.h:25). */
void orc_gmres(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
               const orc_precond* P, int flexible, uint32_t restart, double tol,
               const double* b, double* x, int32_t* num_iter, double* final_error, int32_t* converged) {
    int32_t max_iter = 500;
    uint32_t mm = n;
    if (restart > 0) {
        mm = restart;
        max_iter = max_iter / (int32_t)restart;
        if (restart >= n) mm = n - 1;
    } else {
        mm = n - 1;
    }
    uint32_t m = mm;
    double beta, val0, rnorm = 0.0, rel = 0.0;
    double bnorm = sqrt(sum_sq_kahan(n, b));
    double* vj = calloc(n, sizeof(double));
    double* wj = calloc(n, sizeof(double));
    double* r = calloc(n, sizeof(double));
    double* ksi = calloc(mm + 1, sizeof(double));
    double* s = calloc(mm + 1, sizeof(double));
    double* c = calloc(mm + 1, sizeof(double));
    double* V = calloc((size_t)n * (mm + 1), sizeof(double));
    double* H = calloc((size_t)(mm + 1) * mm, sizeof(double));
    double* Z = flexible ? calloc((size_t)n * (mm + 1), sizeof(double)) : NULL;
    const uint32_t ld = mm + 1;
    *converged = 0;
    orc_spmv(n, rowptr, col, val, x, r);
    for (uint32_t i = 0; i < n; i++) vj[i] = 1 * b[i] + -1 * r[i];
    beta = sqrt(sum_sq_kahan(n, vj));
    int32_t k = -1;
    while (!*converged && k < max_iter) {
        ++k;
        for (uint32_t i = 0; i < n; i++) vj[i] *= 1 / beta;
        memcpy(V, vj, n * sizeof(double));
        for (uint32_t i = 0; i < mm; i++) ksi[i] = 0;
        ksi[0] = beta;
        for (uint32_t j = 0; j < m; j++) {
            if (flexible) {
                if (P && P->kind) orc_precond_apply(P, vj);
                memcpy(Z + (size_t)j * n, vj, n * sizeof(double));
            }
            orc_spmv(n, rowptr, col, val, vj, wj);
            for (uint32_t i = 0; i < j + 1; i++) {
                memcpy(vj, V + (size_t)i * n, n * sizeof(double));
                val0 = dot(n, wj, vj);
                H[i + j * ld] = val0;
                for (uint32_t q = 0; q < n; q++) vj[q] *= val0;
                for (uint32_t q = 0; q < n; q++) wj[q] = wj[q] + -1 * vj[q];
            }
            val0 = sqrt(sum_sq_kahan(n, wj));
            H[j + 1 + j * ld] = val0;
            if (fabs(val0) == 0) { m = j; break; }
            memcpy(vj, wj, n * sizeof(double));
            for (uint32_t q = 0; q < n; q++) vj[q] *= 1 / val0;
            memcpy(V + (size_t)(j + 1) * n, vj, n * sizeof(double));
            givens(H, ld, c, s, ksi, j);
            rnorm = fabs(ksi[j + 1]);
            rel = rnorm / bnorm;
            if (rel < tol) { m = j; break; }
        }
        /* retrospectiveSolver (GMRES.cpp:103-119) */
        for (int i = (int)m - 1; i >= 0; --i) {
            for (int jj = i + 1; jj < (int)m; ++jj) ksi[i] = ksi[i] - H[i + jj * ld] * ksi[jj];
            ksi[i] = ksi[i] / H[i + i * ld];
        }
        ksi[m] = 0;
        ksi[m] = 0;
        /* x += Z ksi (flexible) or V ksi: DenseMatrix::MatVec over m+1 columns (DenseMatrix.cpp:208-243) */
        const double* B = flexible ? Z : V;
        for (uint32_t q = 0; q < n; q++) wj[q] = 0;
        for (uint32_t jj = 0; jj < mm + 1; jj++) {
            double kj = ksi[jj];
            for (uint32_t q = 0; q < n; q++) wj[q] += B[(size_t)jj * n + q] * kj;
        }
        for (uint32_t q = 0; q < n; q++) x[q] = x[q] + 1 * wj[q];
        *converged = rel < tol;
        orc_spmv(n, rowptr, col, val, x, r);
        for (uint32_t i = 0; i < n; i++) vj[i] = 1 * b[i] + -1 * r[i];
        beta = rnorm;
    }
    *final_error = rel;
    *num_iter = k * (int32_t)mm + (int32_t)m;
    free(vj); free(wj); free(r); free(ksi); free(s); free(c); free(V); free(H);
    if (Z) free(Z);
}
