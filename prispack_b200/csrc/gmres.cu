// Restarted (flexible) GMRES on the device: GMRES<double>::solve
// (source/Solver/GMRES.cpp:122-221) with setRestart (GMRES.cpp:60-70).
//
// Same recurrence as the reference: modified Gram-Schmidt Arnoldi (one fused
// kernel per link: the axpy of link i with the dot of link i+1), Givens QR of
// the Hessenberg column and back substitution (O(m) scalars, on the host, in
// the reference's operation order), the same convergence estimate, the same
// restart from the Givens estimate (GMRES.cpp:214) and the same iteration
// count convention numIter = k*m + m_final (GMRES.cpp:218).  Reductions sum
// in a fixed tree order rather than serially (and without the Kahan
// compensation of BaseVector::sumKahan), so scalars agree to rounding level.
#include <cmath>
#include <vector>

#include "kernels.cuh"
#include "solve.cuh"

namespace prism {

namespace {
int vgrid(const Handle& h, uint32_t n) {
    long want = ((long)n + kBlock - 1) / kBlock;
    long cap = (long)h.info.sms * 4;
    if (want < 1) want = 1;
    return (int)(want < cap ? want : cap);
}

// GMRES<ValType>::givensTransform (GMRES.cpp:73-101); H column-major (ld x m)
void givens(std::vector<double>& H, uint32_t ld, std::vector<double>& c, std::vector<double>& s,
            std::vector<double>& ksi, uint32_t j) {
    double val0, val1, val2, tao;
    for (uint32_t i = 0; i < j; ++i) {
        val1 = H[i + j * ld];
        val2 = H[i + 1 + j * ld];
        val0 = c[i] * val2 - s[i] * val1;
        H[i + 1 + j * ld] = val0;
        val0 = c[i] * val1 + s[i] * val2;
        H[i + j * ld] = val0;
    }
    val1 = H[j + j * ld];
    val2 = H[j + 1 + j * ld];
    if (std::fabs(val1) > std::fabs(val2)) {
        tao = val2 / val1;
        c[j] = 1 / std::sqrt(std::fabs(1.0 + tao * tao));
        s[j] = c[j] * tao;
    } else {
        tao = val1 / val2;
        s[j] = 1 / std::sqrt(std::fabs(1.0 + tao * tao));
        c[j] = s[j] * tao;
    }
    H[j + j * ld] = c[j] * val1 + s[j] * val2;
    H[j + 1 + j * ld] = 0.0;
    ksi[j + 1] = -s[j] * ksi[j];
    ksi[j] = c[j] * ksi[j];
}

// GMRES<ValType>::retrospectiveSolver (GMRES.cpp:103-119)
void back_substitute(const std::vector<double>& H, uint32_t ld, std::vector<double>& ksi, uint32_t dim) {
    for (int i = (int)dim - 1; i >= 0; --i) {
        for (int j = i + 1; j < (int)dim; ++j) ksi[i] = ksi[i] - H[i + j * ld] * ksi[j];
        ksi[i] = ksi[i] / H[i + i * ld];
    }
    ksi[dim] = 0;
}
}  // namespace

void gmres_solve(Handle& h, const prism_solve_opts& o, const double* b, double* x, prism_solve_stats* st) {
    const uint32_t n = h.A.n;
    cudaStream_t s = h.stream;
    const bool flexible = o.solver == PRISM_SOLVER_FGMRES;
    Precond* P = h.P.get();
    if (flexible && !P) throw Error(PRISM_ERR_NOT_READY, "FlexibleGMRES must use a preconditioner (GMRES.cpp:165-168)");
    h.ensure_workspace();
    // setRestart(true, m) / no restart (GMRES.cpp:60-70); maxIter = MAX_ITER_NUM_SOLVER = 500
    int32_t max_cycles = 500;
    uint32_t mm;
    if (o.restart > 0) {
        mm = o.restart;
        max_cycles = max_cycles / (int32_t)o.restart;
        if (o.restart >= n) mm = n - 1;
    } else {
        mm = n - 1;
    }
    if (mm == 0) throw Error(PRISM_ERR_ARG, "GMRES needs n >= 2");
    if (mm + 2 > Handle::kMaxKrylov) throw Error(PRISM_ERR_ARG, "restart length too large for the Krylov workspace");
    const size_t cols = (size_t)mm + 1;
    if (h.V.size() < cols * n) h.V.alloc(cols * n);
    if (flexible && h.Z.size() < cols * n) h.Z.alloc(cols * n);
    if (h.ksi.size() < cols) h.ksi.alloc(cols);
    // the reference's Z is zero-initialised (calloc) and columns beyond the
    // current step are read with stale coefficients (see x update below)
    PRISM_CUDA(cudaMemsetAsync(h.V.get(), 0, cols * n * sizeof(double), s));
    if (flexible) PRISM_CUDA(cudaMemsetAsync(h.Z.get(), 0, cols * n * sizeof(double), s));
    double* V = h.V.get();
    double* Z = flexible ? h.Z.get() : nullptr;
    double* w = h.w.get();
    double* y = h.y.get();
    double* vj = h.r.get();
    double* sc = h.red.scalars.get();
    double* hcol = sc + SC_H0;
    const int vg = vgrid(h, n);
    uint32_t applies = 0, spmvs = 0;
    std::vector<double> H(cols * mm, 0.0), cs(cols, 0.0), sn(cols, 0.0), ksi(cols, 0.0);

    PRISM_CUDA(cudaEventRecord(h.ev0, s));
    // r = A x; vj = b - r; Σ b², Σ vj²
    h.spmv(x, y);
    ++spmvs;
    k_residual<<<vg, kBlock, 0, s>>>(n, b, y, vj, h.red.slot(SC_BB));
    PRISM_LAUNCHED();
    PRISM_CUDA(cudaMemcpyAsync(h.pinned, sc, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    h.check_status();
    const double bnorm = std::sqrt(h.pinned[SC_BB]);
    double beta = std::sqrt(h.pinned[SC_RES]);
    double rnorm = 0.0, rel = 0.0;
    bool converged = false;
    uint32_t m = mm;
    int32_t k = -1;
    while (!converged && k < max_cycles) {
        ++k;
        // V_0 = vj * (1/beta)
        k_scale<<<vg, kBlock, 0, s>>>(n, vj, 1.0 / beta, V);
        PRISM_LAUNCHED();
        std::fill(ksi.begin(), ksi.begin() + mm, 0.0);
        ksi[0] = beta;
        for (uint32_t j = 0; j < m; ++j) {
            const double* vjcol = V + (size_t)j * n;
            const double* opnd = vjcol;
            if (flexible) {
                double* zj = Z + (size_t)j * n;
                P->apply(s, vjcol, zj);
                ++applies;
                opnd = zj;
            }
            // w = A opnd ; Σ w·V_0
            h.spmv(opnd, w, 0);
            ++spmvs;
            // MGS: link i subtracts h_{i-1} V_{i-1} and forms h_i = w·V_i; the last link forms ||w||²
            for (uint32_t i = 0; i <= j + 1; ++i) {
                const double* vprev = i > 0 ? V + (size_t)(i - 1) * n : nullptr;
                const double* vnext = i <= j ? V + (size_t)i * n : nullptr;
                k_mgs<<<vg, kBlock, 0, s>>>(n, w, vprev, hcol + (i > 0 ? i - 1 : 0), vnext, h.red.slot(SC_H0 + i));
                PRISM_LAUNCHED();
            }
            PRISM_CUDA(cudaMemcpyAsync(h.pinned, hcol, (j + 2) * sizeof(double), cudaMemcpyDeviceToHost, s));
            h.check_status();
            for (uint32_t i = 0; i <= j; ++i) H[i + j * cols] = h.pinned[i];
            const double hnext = std::sqrt(h.pinned[j + 1]);
            if (!std::isfinite(hnext)) throw Error(PRISM_ERR_NONFINITE, "non-finite Arnoldi norm");
            H[j + 1 + j * cols] = hnext;
            if (std::fabs(hnext) == 0) {  // lucky breakdown (GMRES.cpp:183-186)
                m = j;
                break;
            }
            // V_{j+1} = w * (1/h)
            k_scale<<<vg, kBlock, 0, s>>>(n, w, 1.0 / hnext, V + (size_t)(j + 1) * n);
            PRISM_LAUNCHED();
            givens(H, (uint32_t)cols, cs, sn, ksi, j);
            rnorm = std::fabs(ksi[j + 1]);
            rel = rnorm / bnorm;
            if (rel < o.tol) {
                m = j;
                break;
            }
        }
        // least squares R y = g, then x += Z ksi (flexible) or V ksi over all m+1 columns
        back_substitute(H, (uint32_t)cols, ksi, m);
        ksi[m] = 0;
        PRISM_CUDA(cudaMemcpyAsync(h.ksi.get(), ksi.data(), cols * sizeof(double), cudaMemcpyHostToDevice, s));
        k_gemv_add<<<vg, kBlock, 0, s>>>(n, flexible ? Z : V, (uint32_t)cols, h.ksi.get(), x);
        PRISM_LAUNCHED();
        converged = rel < o.tol;
        // vj = b - A x ; the next cycle restarts from the Givens estimate (GMRES.cpp:212-214)
        h.spmv(x, y);
        ++spmvs;
        k_residual<<<vg, kBlock, 0, s>>>(n, b, y, vj, h.red.slot(SC_BB));
        PRISM_LAUNCHED();
        beta = rnorm;
        PRISM_CUDA(cudaStreamSynchronize(s));  // ksi host buffer is reused next cycle
    }
    PRISM_CUDA(cudaEventRecord(h.ev1, s));
    PRISM_CUDA(cudaMemcpyAsync(h.pinned, sc, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    h.check_status();
    float ms = 0.f;
    PRISM_CUDA(cudaEventElapsedTime(&ms, h.ev0, h.ev1));
    if (st) {
        st->num_iter = k * (int32_t)mm + (int32_t)m;
        st->converged = converged;
        st->final_error = rel;
        st->true_rel_residual = std::sqrt(h.pinned[SC_RES]) / std::sqrt(h.pinned[SC_BB]);
        st->precond_applies = applies;
        st->spmv_count = spmvs;
        st->device_ms = ms;
    }
}

}  // namespace prism
