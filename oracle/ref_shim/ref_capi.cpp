// Test-only C entry points around the reference's own CPU classes.
//
// This file is compiled together with the reference's unmodified sources
// (include/, source/ of PrisPack) by oracle/Makefile into oracle/_ref/.
// It is the checker's view of the reference: it lets the Python tests and the
// CPU-baseline arm of bench.py drive HOST::CSRMatrix, HOST::IncompleteCholesky,
// HOST::IncompleteLDLT, HOST::IncompleteLU, HOST::CG and HOST::GMRES through
// plain pointers.  Nothing in the product library links against it.
//
// The reference keeps factor arrays in private members without getters for
// ILDLT, so private/protected are opened up for this translation unit only,
// after every standard header has been included.
#include "config/headers.h"
#include <omp.h>
#include <functional>
#include <numeric>
// everything that carries OpenMP pragmas (private(...) clauses) first
#include "MatrixClass/CSRMatrix.h"
#include "MatrixClass/DenseMatrix.h"
#include "MatrixClass/ModelProblem.h"
#include "VectorClass/VectorTools.h"
#include "utils/MemoryTools/SharedPtrTools.h"
#include "utils/TimerTools/CPUtimer.hpp"
#include "Preconditioner/BasePreconditon.h"
#include "utils/ExternalTools/MatrixReorderTools.h"
#include "utils/ExternalTools/MetisTools.h"
#include "utils/TestTools/WriteMtxTools.h"
#include "utils/TestTools/ReadMtxTools.h"
#include "utils/TestTools/checkTools.hpp"
#define private public
#define protected public
#include "Preconditioner/IncompleteCholesky.h"
#include "Preconditioner/IncompleteLDLT.h"
#include "Preconditioner/IncompleteLU.h"
#include "Solver/CG.h"
#include "Solver/GMRES.h"
#include "Preconditioner/AMSEDPrecondition.h"
#include "Preconditioner/GMSLRPrecondition.h"
#undef private
#undef protected

using namespace HOST;

namespace {
using CSRd = CSRMatrix<FLOAT64>;

unsigned g_seed_base = 20241116u, g_seed_calls = 0u;

struct RefPrecond {
    int kind;        // 1 = IC, 2 = ILUT, 3 = ILDLT, 5 = AMSED
    int lowPrecision;  // 1 = factor values stored in FP32
    std::shared_ptr<BasePrecondition<FLOAT64>> p;
};

template <typename V>
void copyVec(const HostVector<V>& src, V* dst, UINT32 n) {
    for (UINT32 i = 0; i < n; ++i) dst[i] = src[i];
}
// Factor export.  which: 0 = first stored triangle (IC/ILDLT: L^T rows; ILUT: L),
// 1 = second (ILUT: U).  Values are widened to double.
template <typename Low>
const CSRMatrix<Low>* factorMat(RefPrecond* r, int which) {
    if (r->kind == 1) return &*static_cast<IncompleteCholesky<Low, FLOAT64>*>(r->p.get())->m_matTransL;
    if (r->kind == 3) return &*static_cast<IncompleteLDLT<Low, FLOAT64>*>(r->p.get())->m_matTransL;
    auto* lu = static_cast<IncompleteLU<Low, FLOAT64>*>(r->p.get());
    return which == 0 ? &*lu->m_L : &*lu->m_U;
}

template <typename Low>
void factorDims(RefPrecond* r, int which, unsigned* n, unsigned* nnz) {
    const CSRMatrix<Low>* M = factorMat<Low>(r, which);
    *n = M->getRowNum();
    *nnz = M->getRowOffsetPtr(0)[M->getRowNum()];
}

template <typename Low>
void factorCopy(RefPrecond* r, int which, unsigned* rowptr, unsigned* col, double* val, double* diag) {
    const CSRMatrix<Low>* M = factorMat<Low>(r, which);
    UINT32 n = M->getRowNum();
    const UINT32* rp = M->getRowOffsetPtr(0);
    for (UINT32 i = 0; i <= n; ++i) rowptr[i] = rp[i];
    for (UINT32 k = 0; k < rp[n]; ++k) { col[k] = M->getColIndicesPtr(0)[k]; val[k] = (double)M->getCSRValuesPtr(0)[k]; }
    if (diag) {
        if (r->kind == 3) {
            auto* p = static_cast<IncompleteLDLT<Low, FLOAT64>*>(r->p.get());
            for (UINT32 i = 0; i < n; ++i) diag[i] = (*p->m_diagVals)[i];
        } else if (r->kind == 2) {
            auto* p = static_cast<IncompleteLU<Low, FLOAT64>*>(r->p.get());
            for (UINT32 i = 0; i < n; ++i) diag[i] = (double)(*p->m_diagVals)[i];
        }
    }
}

}  // namespace

extern "C" {

// ---- CSR -----------------------------------------------------------------
void* ref_csr_laplacian(int nx, int ny, int nz, double ax, double ay, double az, double shift) {
    auto* A = new CSRd();
    generateLaplacianCSR<FLOAT64>(*A, nx, ny, nz, ax, ay, az, shift);
    return A;
}

void* ref_csr_poisson(unsigned blk) {
    auto* A = new CSRd();
    generatePoissonCSR<FLOAT64>(*A, blk);
    return A;
}

void* ref_csr_from_arrays(unsigned n, const unsigned* rowptr, const unsigned* col, const double* val) {
    UINT32 nnz = rowptr[n];
    auto* A = new CSRd(n, n, nnz, memoryBase);
    UINT32* rp = A->getRowOffsetPtr(0);
    UINT32* ci = A->getColIndicesPtr(0);
    FLOAT64* v = A->getCSRValuesPtr(0);
    for (UINT32 i = 0; i <= n; ++i) rp[i] = rowptr[i];
    for (UINT32 k = 0; k < nnz; ++k) { ci[k] = col[k]; v[k] = val[k]; }
    return A;
}

void ref_csr_dims(void* h, unsigned* n, unsigned* nnz) {
    auto* A = static_cast<CSRd*>(h);
    *n = A->getRowNum();
    *nnz = A->getRowOffsetPtr(0)[A->getRowNum()];
}

void ref_csr_copy(void* h, unsigned* rowptr, unsigned* col, double* val) {
    auto* A = static_cast<CSRd*>(h);
    UINT32 n = A->getRowNum();
    const UINT32* rp = A->getRowOffsetPtr(0);
    for (UINT32 i = 0; i <= n; ++i) rowptr[i] = rp[i];
    for (UINT32 k = 0; k < rp[n]; ++k) { col[k] = A->getColIndicesPtr(0)[k]; val[k] = A->getCSRValuesPtr(0)[k]; }
}

void ref_csr_free(void* h) { delete static_cast<CSRd*>(h); }

// HOST::ReadMtxTools<double>::loadMatrix of a Matrix Market file (1-based), part 0: the real
// matrix (or a complex file's real part), 1: a complex file's imaginary part.  The reader
// changes the working directory to dirname(binaryPath): "./" keeps it.
void* ref_read_mtx(const char* path, int part) {
    char here[] = "./reader";
    ReadMtxTools<FLOAT64> rd(here, path, 1);
    auto* A = new CSRd();
    if (part == 0) {
        rd.loadMatrix(*A);
    } else {
        CSRd re;
        rd.loadMatrix(re, *A);
    }
    return A;
}

void ref_spmv(void* h, const double* x, double* y) {
    auto* A = static_cast<CSRd*>(h);
    A->MatPVecWithRawPtr(x, y);
}

// ---- preconditioners -------------------------------------------------------
// kind: 1 IC (threshold), 2 ILUT (lfill, tol), 3 ILDLT (tol)
void* ref_precond_create(void* hA, int kind, int lowPrecision, double tol, int lfill) {
    auto* A = static_cast<CSRd*>(hA);
    // the preconditioner keeps a shared_ptr alias; the matrix stays owned by the caller
    std::shared_ptr<CSRd> sp(A, [](CSRd*) {});
    auto* r = new RefPrecond{kind, lowPrecision, nullptr};
    if (kind == 1) {
        if (lowPrecision) r->p = std::make_shared<IncompleteCholesky<FLOAT32, FLOAT64>>(sp, tol);
        else r->p = std::make_shared<IncompleteCholesky<FLOAT64, FLOAT64>>(sp, tol);
    } else if (kind == 2) {
        if (lowPrecision) r->p = std::make_shared<IncompleteLU<FLOAT32, FLOAT64>>(sp, (UINT32)lfill, tol);
        else r->p = std::make_shared<IncompleteLU<FLOAT64, FLOAT64>>(sp, (UINT32)lfill, tol);
    } else if (kind == 3) {
        if (lowPrecision) r->p = std::make_shared<IncompleteLDLT<FLOAT32, FLOAT64>>(sp, tol);
        else r->p = std::make_shared<IncompleteLDLT<FLOAT64, FLOAT64>>(sp, tol);
    } else {
        delete r;
        return nullptr;
    }
    return r;
}

int ref_precond_setup(void* h) {
    auto* r = static_cast<RefPrecond*>(h);
    if (r->kind == 5) g_seed_calls = 0;
    try {
        r->p->setup();
    } catch (...) {
        return -1;
    }
    return r->p->isReady() ? 0 : -2;
}

void ref_precond_free(void* h) { delete static_cast<RefPrecond*>(h); }

unsigned ref_precond_mnnz(void* h) { return static_cast<RefPrecond*>(h)->p->getPreconditionNonZeroCount(); }

void ref_precond_factor_dims(void* h, int which, unsigned* n, unsigned* nnz) {
    auto* r = static_cast<RefPrecond*>(h);
    if (r->lowPrecision) factorDims<FLOAT32>(r, which, n, nnz);
    else factorDims<FLOAT64>(r, which, n, nnz);
}

void ref_precond_factor_copy(void* h, int which, unsigned* rowptr, unsigned* col, double* val, double* diag) {
    auto* r = static_cast<RefPrecond*>(h);
    if (r->lowPrecision) factorCopy<FLOAT32>(r, which, rowptr, col, val, diag);
    else factorCopy<FLOAT64>(r, which, rowptr, col, val, diag);
}

// vec <- M^{-1} vec (TriangularPrecondition::MInvSolve, in place)
void ref_precond_apply(void* h, unsigned n, double* vec) {
    auto* r = static_cast<RefPrecond*>(h);
    DenseVector<FLOAT64> v(n);
    for (UINT32 i = 0; i < n; ++i) v[i] = vec[i];
    r->p->MInvSolve(v);
    for (UINT32 i = 0; i < n; ++i) vec[i] = v[i];
}

// ---- solvers ---------------------------------------------------------------
// cgType: 0 NormalCG, 1 FlexibleCG.  hP may be null.  x is the in/out guess.
int ref_cg_solve(void* hA, void* hP, int cgType, double tol, unsigned maxIter, const double* b, double* x,
                 int* numIter, double* finalError, int* converged) {
    auto* A = static_cast<CSRd*>(hA);
    UINT32 n = A->getRowNum();
    DenseVector<FLOAT64> vb(n), vx(n);
    for (UINT32 i = 0; i < n; ++i) { vb[i] = b[i]; vx[i] = x[i]; }
    if (hP) {
        auto* r = static_cast<RefPrecond*>(hP);
        CG<FLOAT64> s(n, r->p, cgType ? FlexibleCG : NormalCG, tol, maxIter);
        s.solve(*A, vb, vx);
        *numIter = s.getNumIter();
        *finalError = s.getError();
        *converged = s.getConvergence();
    } else {
        CG<FLOAT64> s(n, tol, maxIter);
        s.solve(*A, vb, vx);
        *numIter = s.getNumIter();
        *finalError = s.getError();
        *converged = s.getConvergence();
    }
    for (UINT32 i = 0; i < n; ++i) x[i] = vx[i];
    return 0;
}

// gmresType: 0 NormalGMRES, 1 FlexibleGMRES; restart > 0 enables setRestart(true, restart)
int ref_gmres_solve(void* hA, void* hP, int gmresType, unsigned restart, double tol, const double* b, double* x,
                    int* numIter, double* finalError, int* converged) {
    auto* A = static_cast<CSRd*>(hA);
    UINT32 n = A->getRowNum();
    DenseVector<FLOAT64> vb(n), vx(n);
    for (UINT32 i = 0; i < n; ++i) { vb[i] = b[i]; vx[i] = x[i]; }
    std::shared_ptr<BasePrecondition<FLOAT64>> p;
    if (hP) p = static_cast<RefPrecond*>(hP)->p;
    GMRES<FLOAT64> s(n, p, tol, gmresType ? FlexibleGMRES : NormalGMRES);
    if (restart > 0) s.setRestart(true, restart);
    s.solve(*A, vb, vx);
    *numIter = s.getNumIter();
    *finalError = s.getError();
    *converged = s.getConvergence();
    for (UINT32 i = 0; i < n; ++i) x[i] = vx[i];
    return 0;
}

int ref_omp_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"

// ---- AMSED -------------------------------------------------------------------
extern "C" unsigned prism_ref_next_seed(void) { return g_seed_base + g_seed_calls++; }

extern "C" void ref_set_seed(unsigned seed) {
    g_seed_base = seed;
    g_seed_calls = 0;
}

extern "C" void* ref_amsed_create(void* hA, int levels, int lanczos_steps, int low_rank, double eig_bound, int reorder,
                       int lowrank_type, int lanczos_type, int low_precision) {
    auto* A = static_cast<CSRd*>(hA);
    std::shared_ptr<CSRd> sp(A, [](CSRd*) {});
    auto* r = new RefPrecond{5, low_precision, nullptr};
    auto ro = (MatrixReorderOption_t)reorder;
    auto lt = (LowRankCorrectType_t)lowrank_type;
    auto lz = (LanczosType_t)lanczos_type;
    if (low_precision)
        r->p = std::make_shared<AMSEDPrecondition<FLOAT32, FLOAT64>>(sp, levels, lanczos_steps, low_rank, eig_bound, ro, lt, lz);
    else
        r->p = std::make_shared<AMSEDPrecondition<FLOAT64, FLOAT64>>(sp, levels, lanczos_steps, low_rank, eig_bound, ro, lt, lz);
    return r;
}

template <typename Low>
static AMSEDPrecondition<Low, FLOAT64>* amsed(void* h) {
    return static_cast<AMSEDPrecondition<Low, FLOAT64>*>(static_cast<RefPrecond*>(h)->p.get());
}

template <typename Low>
static void amsed_info_t(void* h, unsigned* nlev, unsigned* lev_ptr, unsigned* ncomps, unsigned* ranks,
                         unsigned* mnnz) {
    auto* a = amsed<Low>(h);
    *nlev = a->m_nlev_used;
    if (mnnz) *mnnz = a->getPreconditionNonZeroCount();
    for (UINT32 l = 0; l < a->m_nlev_used; ++l) {
        if (ncomps) ncomps[l] = a->m_levs_all[l]->ncomps;
        if (ranks) ranks[l] = a->m_levs_all[l]->rank;
    }
    if (lev_ptr)
        for (UINT32 l = 0; l <= a->m_nlev_used; ++l) lev_ptr[l] = a->m_lev_ptr_v[l];
}

extern "C" void ref_amsed_info(void* h, unsigned* nlev, unsigned* lev_ptr, unsigned* ncomps, unsigned* ranks, unsigned* mnnz) {
    if (static_cast<RefPrecond*>(h)->lowPrecision) amsed_info_t<FLOAT32>(h, nlev, lev_ptr, ncomps, ranks, mnnz);
    else amsed_info_t<FLOAT64>(h, nlev, lev_ptr, ncomps, ranks, mnnz);
}

template <typename Low>
static void amsed_perm_t(void* h, unsigned* perm) {
    auto* a = amsed<Low>(h);
    for (UINT32 i = 0; i < a->m_pperm.getLength(); ++i) perm[i] = a->m_pperm[i];
}

extern "C" void ref_amsed_perm(void* h, unsigned* perm) {
    if (static_cast<RefPrecond*>(h)->lowPrecision) amsed_perm_t<FLOAT32>(h, perm);
    else amsed_perm_t<FLOAT64>(h, perm);
}

template <typename Low>
static void amsed_dom_t(void* h, int level, unsigned* dom) {
    auto* a = amsed<Low>(h);
    auto& d = *a->m_dom_ptr_v2[level];
    for (UINT32 i = 0; i < d.getLength(); ++i) dom[i] = d[i];
}

extern "C" void ref_amsed_dom_ptr(void* h, int level, unsigned* dom) {
    if (static_cast<RefPrecond*>(h)->lowPrecision) amsed_dom_t<FLOAT32>(h, level, dom);
    else amsed_dom_t<FLOAT64>(h, level, dom);
}

// block factor: last level -> IncompleteCholesky L^T; other levels -> IncompleteLDLT L^T + D
template <typename Low>
static void amsed_block_t(void* h, int level, int block, unsigned* n, unsigned* nnz, unsigned* rowptr, unsigned* col,
                          double* val, double* diag) {
    auto* a = amsed<Low>(h);
    auto& L = *a->m_levs_all[level];
    const CSRMatrix<Low>* M;
    const bool last = (UINT32)level == a->m_nlev_used - 1;
    if (last) M = &*static_cast<IncompleteCholesky<Low, FLOAT64>*>(L.B_precond[block].get())->m_matTransL;
    else M = &*static_cast<IncompleteLDLT<Low, FLOAT64>*>(L.B_precond[block].get())->m_matTransL;
    *n = M->getRowNum();
    *nnz = M->getRowOffsetPtr(0)[M->getRowNum()];
    if (rowptr) {
        for (UINT32 i = 0; i <= *n; ++i) rowptr[i] = M->getRowOffsetPtr(0)[i];
        for (UINT32 k = 0; k < *nnz; ++k) { col[k] = M->getColIndicesPtr(0)[k]; val[k] = (double)M->getCSRValuesPtr(0)[k]; }
        if (!last && diag) {
            auto* p = static_cast<IncompleteLDLT<Low, FLOAT64>*>(L.B_precond[block].get());
            for (UINT32 i = 0; i < *n; ++i) diag[i] = (*p->m_diagVals)[i];
        }
    }
}

extern "C" void ref_amsed_block(void* h, int level, int block, unsigned* n, unsigned* nnz, unsigned* rowptr, unsigned* col,
                     double* val, double* diag) {
    if (static_cast<RefPrecond*>(h)->lowPrecision) amsed_block_t<FLOAT32>(h, level, block, n, nnz, rowptr, col, val, diag);
    else amsed_block_t<FLOAT64>(h, level, block, n, nnz, rowptr, col, val, diag);
}

template <typename Low>
static void amsed_lowrank_t(void* h, int level, unsigned* rank, unsigned* nrem, double* W, double* H) {
    auto* a = amsed<Low>(h);
    auto& L = *a->m_levs_all[level];
    *rank = L.rank;
    *nrem = a->m_lev_ptr_v[a->m_nlev_used] - a->m_lev_ptr_v[level + 1];
    if (W && L.rank) {
        const double* w = L.W_mat.getMatValPtr();
        for (size_t k = 0; k < (size_t)L.rank * *nrem; ++k) W[k] = w[k];
        for (UINT32 i = 0; i < L.rank; ++i) H[i] = L.H_vec[i];
    }
}

extern "C" void ref_amsed_lowrank(void* h, int level, unsigned* rank, unsigned* nrem, double* W, double* H) {
    if (static_cast<RefPrecond*>(h)->lowPrecision) amsed_lowrank_t<FLOAT32>(h, level, rank, nrem, W, H);
    else amsed_lowrank_t<FLOAT64>(h, level, rank, nrem, W, H);
}


// rcmReorderCSR (include/utils/ExternalTools/MatrixReorderTools.h:51-85) on a caller CSR
extern "C" void ref_rcm(unsigned n, const unsigned* rowptr, const unsigned* col, unsigned* perm) {
    CSRd A(n, n, rowptr[n], memoryBase);
    for (UINT32 i = 0; i <= n; ++i) A.getRowOffsetPtr(0)[i] = rowptr[i];
    for (UINT32 k = 0; k < rowptr[n]; ++k) { A.getColIndicesPtr(0)[k] = col[k]; A.getCSRValuesPtr(0)[k] = 1.0; }
    DenseVector<UINT32> p(n);
    rcmReorderCSR(A, p);
    for (UINT32 i = 0; i < n; ++i) perm[i] = p[i];
}

// ---- GMSLR -------------------------------------------------------------------
extern "C" void* ref_gmslr_create(void* hA, int levels, int lanczos_steps, int low_rank, int reorder,
                                  int low_precision) {
    auto* A = static_cast<CSRd*>(hA);
    std::shared_ptr<CSRd> sp(A, [](CSRd*) {});
    auto* r = new RefPrecond{4, low_precision, nullptr};
    auto ro = (MatrixReorderOption_t)reorder;
    if (low_precision)
        r->p = std::make_shared<GMSLRPrecondition<FLOAT32, FLOAT64>>(sp, levels, lanczos_steps, low_rank, ro);
    else
        r->p = std::make_shared<GMSLRPrecondition<FLOAT64, FLOAT64>>(sp, levels, lanczos_steps, low_rank, ro);
    return r;
}

template <typename Low>
static GMSLRPrecondition<Low, FLOAT64>* gmslr(void* h) {
    return static_cast<GMSLRPrecondition<Low, FLOAT64>*>(static_cast<RefPrecond*>(h)->p.get());
}

template <typename Low>
static void gmslr_info_t(void* h, unsigned* nlev, unsigned* lev_ptr, unsigned* ncomps, unsigned* ranks, unsigned* mnnz,
                         double* wmax) {
    auto* a = gmslr<Low>(h);
    *nlev = a->m_nlev_used;
    if (mnnz) *mnnz = a->getPreconditionNonZeroCount();
    double m = 0.0;
    for (UINT32 l = 0; l < a->m_nlev_used; ++l) {
        auto& L = *a->m_levs_all[l];
        if (ncomps) ncomps[l] = L.ncomps;
        if (ranks) ranks[l] = L.rank;
        if (l + 1 < a->m_nlev_used && L.rank)
            for (size_t k = 0; k < (size_t)L.rank * L.W_mat.getRowNum(); ++k)
                m = std::max(m, std::fabs(L.W_mat.getMatValPtr()[k]));
    }
    if (wmax) *wmax = m;
    if (lev_ptr)
        for (UINT32 l = 0; l <= a->m_nlev_used; ++l) lev_ptr[l] = a->m_lev_ptr_v[l];
}

extern "C" void ref_gmslr_info(void* h, unsigned* nlev, unsigned* lev_ptr, unsigned* ncomps, unsigned* ranks,
                               unsigned* mnnz, double* wmax) {
    if (static_cast<RefPrecond*>(h)->lowPrecision) gmslr_info_t<FLOAT32>(h, nlev, lev_ptr, ncomps, ranks, mnnz, wmax);
    else gmslr_info_t<FLOAT64>(h, nlev, lev_ptr, ncomps, ranks, mnnz, wmax);
}

template <typename Low>
static void gmslr_perm_t(void* h, unsigned* perm) {
    auto* a = gmslr<Low>(h);
    for (UINT32 i = 0; i < a->m_pperm.getLength(); ++i) perm[i] = a->m_pperm[i];
}

extern "C" void ref_gmslr_perm(void* h, unsigned* perm) {
    if (static_cast<RefPrecond*>(h)->lowPrecision) gmslr_perm_t<FLOAT32>(h, perm);
    else gmslr_perm_t<FLOAT64>(h, perm);
}

// ILUT block factor (which 0: L, 1: U; diag: Dinv)
template <typename Low>
static void gmslr_block_t(void* h, int level, int block, int which, unsigned* n, unsigned* nnz, unsigned* rowptr,
                          unsigned* col, double* val, double* diag) {
    auto* a = gmslr<Low>(h);
    auto& L = *a->m_levs_all[level];
    auto* lu = static_cast<IncompleteLU<Low, FLOAT64>*>(L.B_precond[block].get());
    const CSRMatrix<Low>* M = which == 0 ? &*lu->m_L : &*lu->m_U;
    *n = M->getRowNum();
    *nnz = M->getRowOffsetPtr(0)[M->getRowNum()];
    if (rowptr) {
        for (UINT32 i = 0; i <= *n; ++i) rowptr[i] = M->getRowOffsetPtr(0)[i];
        for (UINT32 k = 0; k < *nnz; ++k) { col[k] = M->getColIndicesPtr(0)[k]; val[k] = (double)M->getCSRValuesPtr(0)[k]; }
        if (diag) for (UINT32 i = 0; i < *n; ++i) diag[i] = (double)(*lu->m_diagVals)[i];
    }
}

extern "C" void ref_gmslr_block(void* h, int level, int block, int which, unsigned* n, unsigned* nnz,
                                unsigned* rowptr, unsigned* col, double* val, double* diag) {
    if (static_cast<RefPrecond*>(h)->lowPrecision) gmslr_block_t<FLOAT32>(h, level, block, which, n, nnz, rowptr, col, val, diag);
    else gmslr_block_t<FLOAT64>(h, level, block, which, n, nnz, rowptr, col, val, diag);
}
