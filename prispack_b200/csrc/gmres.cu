// Restarted (flexible) GMRES on the device: GMRES<double>::solve
// (source/Solver/GMRES.cpp:122-221) with setRestart (GMRES.cpp:60-70).
//
// Same recurrence as the reference: Arnoldi with the preconditioner applied
// to each basis vector (FlexibleGMRES), Givens QR of the Hessenberg column
// (givensTransform, GMRES.cpp:73-101, in the reference's operation order),
// the same convergence estimate |ksi_{j+1}| / ||b|| (GMRES.cpp:192-194), back
// substitution (retrospectiveSolver, GMRES.cpp:103-119), the restart from the
// Givens estimate (GMRES.cpp:214), the cycle length that keeps a reduced m
// from one cycle to the next (GMRES.cpp:126, 184, 196), and the iteration
// count numIter = k*m + m_final (GMRES.cpp:218).
//
// What differs.  The orthogonalisation is classical Gram-Schmidt applied
// twice (CGS2) instead of the reference's modified Gram-Schmidt: the same
// basis in exact arithmetic, at least as well orthogonalised in floating
// point, and three passes over the basis per step whatever the step index,
// fused with their reductions:
//   k_gm_dots     h1 = V^T w (and, flexible, z_j into column j of Z)
//   k_gm_update   w -= V h1, then h2 = V^T w
//   k_gm_update   w -= V h2, ||w||^2, and in the last block to finish: the
//                 Hessenberg column h1 + h2, its Givens rotation, the
//                 residual estimate and the decision to go on
//   k_gm_next     v_{j+1} = w / ||w||
// Every scalar of the cycle (Hessenberg matrix, rotations, ksi, step index,
// state) lives in device memory.  A restart cycle is one CUDA graph: a WHILE
// conditional node whose body is one Arnoldi step (preconditioner apply,
// SpMV and the four kernels above); the Givens kernel ends the loop on the
// device (cudaGraphSetConditional), so the host reads the solver state once
// per cycle.  Where the graph cannot be built (or the caller asks for
// PRISM_LAUNCH_STREAM) the same kernels run as plain launches and the host
// reads the state after every step.  Reductions sum in a fixed order
// (bitwise repeatable for a given grid), not serially with Kahan
// compensation (BaseVector::sumKahan), so scalars agree with the reference's
// to rounding level.
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "kernels.cuh"
#include "solve.cuh"

namespace prism {

namespace {
constexpr int kGmCols = 8;  // basis columns one reduction pass handles at once

int vgrid(const Handle& h, uint32_t n) {
    long want = ((long)n + kBlock - 1) / kBlock;
    long cap = (long)h.info.sms * 4;
    if (want < 1) want = 1;
    return (int)(want < cap ? want : cap);
}

// Where a GMRES solve's scalars live (device memory).
enum : uint32_t { GM_RUN = 0, GM_CONVERGED = 1, GM_BREAKDOWN = 2, GM_NONFINITE = 3, GM_CYCLE_END = 4 };
struct GmState {
    double bnorm, tol, beta, rnorm, rel, hnext;
    uint32_t j;        // Arnoldi step of this cycle
    uint32_t m;        // cycle length: the restart length, reduced after a breakdown or convergence
    uint32_t ld;       // leading dimension of H (restart length + 1)
    uint32_t state;    // GM_*
    uint32_t m_final;  // the step the cycle ended at (the reference's m after its inner loop)
    uint32_t steps;    // Arnoldi steps run in this cycle
};
struct GmPtrs {
    GmState* st;
    double* H;      // ld x restart, column-major
    double* cs;     // [ld]
    double* sn;     // [ld]
    double* ksi;    // [ld]
    double* h1;     // [ld]
    double* h2;     // [ld]
    double* part;   // [grid x ld] block partial sums
    unsigned* ticket;
};

// last-block election after every block's partials are written
__device__ __forceinline__ bool gm_last_block(unsigned* ticket) {
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// out[c] = sum over blocks of part[b * ld + c], c < ncols, blocks in order; re-arms the ticket.
__device__ __forceinline__ void gm_reduce_columns(const GmPtrs& g, uint32_t ncols, uint32_t ld, double* out) {
    for (uint32_t c = threadIdx.x; c < ncols; c += blockDim.x) {
        double s = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) s += __ldcg(g.part + (size_t)b * ld + c);
        out[c] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) *g.ticket = 0u;
}

// Block partial sums of V[:, c]^T x for c < ncols over this thread's rows (grid-stride),
// kGmCols columns per pass, into part[block * ld + c].
__device__ __forceinline__ void gm_block_dots(uint32_t n, const double* __restrict__ x, const double* __restrict__ V,
                                              uint32_t ncols, const GmPtrs& g, uint32_t ld) {
    __shared__ double red[kGmCols * 32];
    for (uint32_t c0 = 0; c0 < ncols; c0 += kGmCols) {
        double acc[kGmCols];
#pragma unroll
        for (int q = 0; q < kGmCols; ++q) acc[q] = 0.0;
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
            const double xi = x[i];
#pragma unroll
            for (int q = 0; q < kGmCols; ++q)
                if (c0 + q < ncols) acc[q] += V[(size_t)(c0 + q) * n + i] * xi;
        }
        block_sum<kGmCols>(acc, red);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int q = 0; q < kGmCols; ++q)
                if (c0 + q < ncols) g.part[(size_t)blockIdx.x * ld + c0 + q] = acc[q];
        }
    }
}

// V_0 = vj / beta and the cycle's scalars (GMRES.cpp:131-135): ksi[0 .. m_m) = 0, ksi[0] = beta.
__global__ void __launch_bounds__(kBlock) k_gm_start(uint32_t n, const double* __restrict__ vj, double* __restrict__ V,
                                                     double* __restrict__ vcur, GmPtrs g, uint32_t restart) {
    const double inv = 1 / g.st->beta;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double v = vj[i] * inv;
        V[i] = v;
        vcur[i] = v;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (uint32_t c = 0; c < restart; ++c) g.ksi[c] = 0.0;
        g.ksi[0] = g.st->beta;
        g.st->j = 0;
        g.st->steps = 0;
        g.st->state = GM_RUN;
        g.st->m_final = g.st->m;
    }
}

// h1 = V[:, 0..j]^T w; flexible: Z[:, j] = z (the preconditioned basis vector, GMRES.cpp:164-170).
__global__ void __launch_bounds__(kBlock) k_gm_dots(uint32_t n, const double* __restrict__ w,
                                                    const double* __restrict__ V, const double* __restrict__ z,
                                                    double* __restrict__ Z, GmPtrs g) {
    const uint32_t j = g.st->j, ld = g.st->ld;
    if (g.st->state != GM_RUN) return;
    if (Z) {
        double* zj = Z + (size_t)j * n;
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) zj[i] = z[i];
    }
    gm_block_dots(n, w, V, j + 1, g, ld);
    if (gm_last_block(g.ticket)) gm_reduce_columns(g, j + 1, ld, g.h1);
}

// GMRES<ValType>::givensTransform (GMRES.cpp:73-101) on column j of H (device copy, one thread).
__device__ void gm_givens(const GmPtrs& g, uint32_t ld, uint32_t j) {
    double* H = g.H + (size_t)j * ld;
    double val0, val1, val2, tao;
    for (uint32_t i = 0; i < j; ++i) {
        val1 = H[i];
        val2 = H[i + 1];
        val0 = g.cs[i] * val2 - g.sn[i] * val1;
        H[i + 1] = val0;
        val0 = g.cs[i] * val1 + g.sn[i] * val2;
        H[i] = val0;
    }
    val1 = H[j];
    val2 = H[j + 1];
    if (fabs(val1) > fabs(val2)) {
        tao = val2 / val1;
        g.cs[j] = 1 / sqrt(fabs(1.0 + tao * tao));
        g.sn[j] = g.cs[j] * tao;
    } else {
        tao = val1 / val2;
        g.sn[j] = 1 / sqrt(fabs(1.0 + tao * tao));
        g.cs[j] = g.sn[j] * tao;
    }
    H[j] = g.cs[j] * val1 + g.sn[j] * val2;
    H[j + 1] = 0.0;
    g.ksi[j + 1] = -g.sn[j] * g.ksi[j];
    g.ksi[j] = g.cs[j] * g.ksi[j];
}

// w -= V[:, 0..j] coef (coef = h1 or h2), then
//   FINAL = false: h2 = V^T w;
//   FINAL = true:  ||w||^2, and in the last block the end of the Arnoldi step: column j of H
//                  (h1 + h2, then ||w||), breakdown (GMRES.cpp:183-186), the Givens rotation,
//                  the residual estimate and the convergence test (GMRES.cpp:190-198); the
//                  graph's loop condition when cond != 0.
template <bool FINAL>
__global__ void __launch_bounds__(kBlock) k_gm_update(uint32_t n, double* __restrict__ w, const double* __restrict__ V,
                                                      GmPtrs g, cudaGraphConditionalHandle cond, int use_cond) {
    __shared__ double coef[Handle::kMaxKrylov + 1];
    const uint32_t j = g.st->j, ld = g.st->ld;
    if (g.st->state != GM_RUN) return;
    const double* src = FINAL ? g.h2 : g.h1;
    for (uint32_t c = threadIdx.x; c <= j; c += blockDim.x) coef[c] = src[c];
    __syncthreads();
    double nrm[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double t = w[i];
        for (uint32_t c = 0; c <= j; ++c) t -= coef[c] * V[(size_t)c * n + i];
        w[i] = t;
        if (FINAL) nrm[0] += t * t;
    }
    if (!FINAL) {
        // the rows this thread just wrote are its own: no grid-wide wait before the dots
        gm_block_dots(n, w, V, j + 1, g, ld);
        if (gm_last_block(g.ticket)) gm_reduce_columns(g, j + 1, ld, g.h2);
        return;
    }
    __shared__ double red[32];
    block_sum<1>(nrm, red);
    if (threadIdx.x == 0) g.part[blockIdx.x] = nrm[0];
    if (!gm_last_block(g.ticket)) return;
    double s = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) s += __ldcg(g.part + b);
    nrm[0] = s;
    block_sum<1>(nrm, red);
    if (threadIdx.x != 0) return;
    *g.ticket = 0u;
    GmState& st = *g.st;
    double* Hj = g.H + (size_t)j * ld;
    for (uint32_t i = 0; i <= j; ++i) Hj[i] = g.h1[i] + g.h2[i];
    const double hn = sqrt(nrm[0]);
    Hj[j + 1] = hn;
    st.hnext = hn;
    st.steps = j + 1;
    uint32_t go = 0;
    if (!isfinite(hn)) {
        st.state = GM_NONFINITE;
        st.m_final = j;
    } else if (fabs(hn) == 0) {
        st.state = GM_BREAKDOWN;
        st.m_final = j;
    } else {
        gm_givens(g, ld, j);
        st.rnorm = fabs(g.ksi[j + 1]);
        st.rel = st.rnorm / st.bnorm;
        if (st.rel < st.tol) {
            st.state = GM_CONVERGED;
            st.m_final = j;
        } else if (j + 1 >= st.m) {
            st.state = GM_CYCLE_END;
            st.m_final = st.m;
        } else {
            go = 1;
        }
    }
    if (use_cond) cudaGraphSetConditional(cond, go);
}

// v_{j+1} = w / ||w|| into column j+1 of V and the next step's operand (GMRES.cpp:187-189),
// unless the step broke down; then the step index moves on (last block).
__global__ void __launch_bounds__(kBlock) k_gm_next(uint32_t n, const double* __restrict__ w, double* __restrict__ V,
                                                    double* __restrict__ vcur, GmPtrs g) {
    const uint32_t j = g.st->j, state = g.st->state;
    if (state != GM_BREAKDOWN && state != GM_NONFINITE) {
        const double inv = 1 / g.st->hnext;
        double* vn = V + (size_t)(j + 1) * n;
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
            const double v = w[i] * inv;
            vn[i] = v;
            vcur[i] = v;
        }
    }
    if (gm_last_block(g.ticket) && threadIdx.x == 0) {
        if (state == GM_RUN) g.st->j = j + 1;
        *g.ticket = 0u;
    }
}

// GMRES<ValType>::retrospectiveSolver (GMRES.cpp:103-119) for dim = m_final, ksi[m] = 0
// (GMRES.cpp:202), and the next cycle's start from the Givens estimate (GMRES.cpp:214).
__global__ void k_gm_finish(GmPtrs g) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    GmState& st = *g.st;
    const uint32_t dim = st.m_final, ld = st.ld;
    for (int i = (int)dim - 1; i >= 0; --i) {
        for (int j = i + 1; j < (int)dim; ++j) g.ksi[i] = g.ksi[i] - g.H[i + (size_t)j * ld] * g.ksi[j];
        g.ksi[i] = g.ksi[i] / g.H[i + (size_t)i * ld];
    }
    g.ksi[dim] = 0;
    st.m = dim;
    st.beta = st.rnorm;
}

// ||b|| and beta = ||b - A x|| from the residual reduction, the solve's constants.
__global__ void k_gm_init(GmState* st, const double* sc, double tol, uint32_t restart) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    st->bnorm = sqrt(sc[SC_BB]);
    st->beta = sqrt(sc[SC_RES]);
    st->tol = tol;
    st->rnorm = 0.0;
    st->rel = 0.0;
    st->hnext = 0.0;
    st->j = 0;
    st->m = restart;
    st->ld = restart + 1;
    st->state = GM_RUN;
    st->m_final = restart;
    st->steps = 0;
}
}  // namespace

// An instantiated restart-cycle graph and what its captured Arnoldi step reads and writes.
struct CycleGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t nodes = 0;
    // the key: the preconditioner object, every buffer the step touches, the sizes
    uint64_t precond_uid = 0;
    const void* bufs[7] = {};
    uint32_t n = 0, restart = 0;
    bool flexible = false;
    ~CycleGraph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

// Workspace of the device GMRES, kept by the handle between solves.
struct GmresWork {
    std::unique_ptr<CycleGraph> graph;  // the last cycle graph built, reused while its key holds
    DevBuf<double> H, cs, sn, ksi, h1, h2, part, vcur, zcur;
    DevBuf<GmState> st;
    DevBuf<unsigned> ticket;
    uint32_t ld = 0, n = 0;
    int grid = 0;
    void ensure(uint32_t n_, uint32_t ld_, int grid_, cudaStream_t s) {
        if (n_ == n && ld_ == ld && grid_ <= grid) return;
        graph.reset();
        H.alloc((size_t)ld_ * (ld_ - 1));
        cs.alloc(ld_);
        sn.alloc(ld_);
        ksi.alloc(ld_);
        h1.alloc(ld_);
        h2.alloc(ld_);
        part.alloc((size_t)grid_ * ld_);
        vcur.alloc(n_);
        zcur.alloc(n_);
        st.alloc(1);
        ticket.alloc(1);
        PRISM_CUDA(cudaMemsetAsync(ticket.get(), 0, sizeof(unsigned), s));
        PRISM_CUDA(cudaMemsetAsync(H.get(), 0, H.size() * sizeof(double), s));
        PRISM_CUDA(cudaMemsetAsync(cs.get(), 0, ld_ * sizeof(double), s));
        PRISM_CUDA(cudaMemsetAsync(sn.get(), 0, ld_ * sizeof(double), s));
        PRISM_CUDA(cudaMemsetAsync(ksi.get(), 0, ld_ * sizeof(double), s));
        n = n_;
        ld = ld_;
        grid = grid_;
    }
    GmPtrs ptrs() {
        return GmPtrs{st.get(), H.get(), cs.get(), sn.get(), ksi.get(), h1.get(), h2.get(), part.get(), ticket.get()};
    }
};
void gmres_release(GmresWork* w) { delete w; }

namespace {
// One Arnoldi step (GMRES.cpp:162-198) on stream s: the preconditioner on the current basis
// vector, the SpMV, CGS2 and the Givens step.
void arnoldi_step(Handle& h, cudaStream_t s, GmresWork& W, bool flexible, cudaGraphConditionalHandle cond,
                  int use_cond) {
    const uint32_t n = h.A.n;
    const int vg = vgrid(h, n);
    Precond* P = h.P.get();
    double* w = h.w.get();
    double* V = h.V.get();
    const double* opnd = W.vcur.get();
    if (flexible) {
        P->apply(s, W.vcur.get(), W.zcur.get());
        opnd = W.zcur.get();
    }
    h.spmv(opnd, w, 0);
    GmPtrs g = W.ptrs();
    k_gm_dots<<<vg, kBlock, 0, s>>>(n, w, V, flexible ? W.zcur.get() : nullptr, flexible ? h.Z.get() : nullptr, g);
    PRISM_LAUNCHED();
    k_gm_update<false><<<vg, kBlock, 0, s>>>(n, w, V, g, cond, 0);
    PRISM_LAUNCHED();
    k_gm_update<true><<<vg, kBlock, 0, s>>>(n, w, V, g, cond, use_cond);
    PRISM_LAUNCHED();
    k_gm_next<<<vg, kBlock, 0, s>>>(n, w, V, W.vcur.get(), g);
    PRISM_LAUNCHED();
}

// The restart cycle as a graph: WHILE (condition set by the Givens kernel) { Arnoldi step }.
// Captured on a private stream that stands in for the handle's stream meanwhile.  Returns
// nullptr (and clears the error) where the runtime refuses any part of it.
std::unique_ptr<CycleGraph> build_cycle_graph(Handle& h, GmresWork& W, bool flexible) {
    auto G = std::make_unique<CycleGraph>();
    cudaStream_t cap = nullptr;
    auto fail = [&]() -> std::unique_ptr<CycleGraph> {
        cudaGetLastError();
        if (cap) cudaStreamDestroy(cap);
        return nullptr;
    };
    if (cudaGraphCreate(&G->graph, 0) != cudaSuccess) return fail();
    cudaGraphConditionalHandle cond;
    if (cudaGraphConditionalHandleCreate(&cond, G->graph, 1, cudaGraphCondAssignDefault) != cudaSuccess) return fail();
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = cond;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    if (cudaGraphAddNode(&node, G->graph, nullptr, 0, &p) != cudaSuccess) return fail();
    cudaGraph_t body = p.conditional.phGraph_out[0];
    if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) return fail();
    if (cudaStreamBeginCaptureToGraph(cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return fail();
    cudaStream_t keep = h.stream;
    h.stream = cap;  // everything the apply and the SpMV enqueue goes to the capture
    bool ok = true;
    try {
        arnoldi_step(h, cap, W, flexible, cond, 1);
    } catch (const Error&) {
        ok = false;
    }
    h.stream = keep;
    cudaGraph_t out = nullptr;
    const cudaError_t e = cudaStreamEndCapture(cap, &out);
    if (!ok || e != cudaSuccess) return fail();
    size_t count = 0;
    if (cudaGraphGetNodes(body, nullptr, &count) == cudaSuccess) G->nodes = (uint32_t)count;
    if (cudaGraphInstantiate(&G->exec, G->graph, 0) != cudaSuccess) return fail();
    cudaStreamDestroy(cap);
    return G;
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
    const uint32_t cols = mm + 1;
    const int vg = vgrid(h, n);
    if (h.V.size() < (size_t)cols * n) h.V.alloc((size_t)cols * n);
    if (flexible && h.Z.size() < (size_t)cols * n) h.Z.alloc((size_t)cols * n);
    if (!h.gmres) h.gmres.reset(new GmresWork());
    GmresWork& W = *h.gmres;
    W.ensure(n, cols, vg, s);
    // the reference's Z is zero-initialised (calloc) and its x update reads every column
    // with the coefficients ksi holds then (see k_gemv_add below)
    PRISM_CUDA(cudaMemsetAsync(h.V.get(), 0, (size_t)cols * n * sizeof(double), s));
    if (flexible) PRISM_CUDA(cudaMemsetAsync(h.Z.get(), 0, (size_t)cols * n * sizeof(double), s));
    PRISM_CUDA(cudaMemsetAsync(W.ksi.get(), 0, cols * sizeof(double), s));
    double* V = h.V.get();
    double* Z = flexible ? h.Z.get() : nullptr;
    double* y = h.y.get();
    double* vj = h.r.get();
    double* sc = h.red.scalars.get();
    uint32_t applies = 0, spmvs = 0, syncs = 0, body_nodes = 0;

    // one restart cycle as a graph, unless the caller asks for plain launches; the graph of an
    // earlier solve is replayed when it was captured from the same preconditioner object and
    // buffers
    CycleGraph* graph = nullptr;
    if (o.launch_mode != PRISM_LAUNCH_STREAM) {
        const void* bufs[7] = {h.V.get(), flexible ? h.Z.get() : nullptr, h.w.get(), W.vcur.get(), W.zcur.get(),
                               W.part.get(), h.A.val.get()};
        const uint64_t uid = P ? P->uid : 0;
        CycleGraph* c = W.graph.get();
        const bool same = c && c->precond_uid == uid && c->n == n && c->restart == mm && c->flexible == flexible &&
                          std::equal(bufs, bufs + 7, c->bufs);
        if (!same) {
            W.graph.reset();
            PRISM_CUDA(cudaStreamSynchronize(s));  // workspace set up before the capture reads its pointers
            W.graph = build_cycle_graph(h, W, flexible);
            if (W.graph) {
                W.graph->precond_uid = uid;
                W.graph->n = n;
                W.graph->restart = mm;
                W.graph->flexible = flexible;
                std::copy(bufs, bufs + 7, W.graph->bufs);
            }
        }
        graph = W.graph.get();
        if (graph) body_nodes = graph->nodes;
    }
    GmPtrs g = W.ptrs();
    GmState hs;

    PRISM_CUDA(cudaEventRecord(h.ev0, s));
    // r = A x; vj = b - r; Σ b², Σ vj²  (GMRES.cpp:152-154)
    h.spmv(x, y);
    ++spmvs;
    k_residual<<<vg, kBlock, 0, s>>>(n, b, y, vj, h.red.slot(SC_BB));
    PRISM_LAUNCHED();
    k_gm_init<<<1, 32, 0, s>>>(g.st, sc, o.tol, mm);
    PRISM_LAUNCHED();
    bool converged = false;
    int32_t k = -1;
    uint32_t m = mm;
    double rel = 0.0;
    while (!converged && k < max_cycles) {
        ++k;
        k_gm_start<<<vg, kBlock, 0, s>>>(n, vj, V, W.vcur.get(), g, mm);
        PRISM_LAUNCHED();
        if (m > 0) {
            if (graph) {
                PRISM_CUDA(cudaGraphLaunch(graph->exec, s));
            } else {
                for (uint32_t j = 0; j < m; ++j) {
                    arnoldi_step(h, s, W, flexible, 0, 0);
                    PRISM_CUDA(cudaMemcpyAsync(&hs, g.st, sizeof(GmState), cudaMemcpyDeviceToHost, s));
                    PRISM_CUDA(cudaStreamSynchronize(s));
                    ++syncs;
                    if (hs.state != GM_RUN) break;
                }
            }
        }
        // least squares R y = g, then x += Z ksi (flexible) or V ksi over all m+1 columns
        k_gm_finish<<<1, 32, 0, s>>>(g);
        PRISM_LAUNCHED();
        k_gemv_add<<<vg, kBlock, 0, s>>>(n, flexible ? Z : V, cols, W.ksi.get(), x);
        PRISM_LAUNCHED();
        // vj = b - A x; the next cycle restarts from the Givens estimate (GMRES.cpp:207-214)
        h.spmv(x, y);
        ++spmvs;
        k_residual<<<vg, kBlock, 0, s>>>(n, b, y, vj, h.red.slot(SC_BB));
        PRISM_LAUNCHED();
        // the restart test: the host's one read of the cycle
        PRISM_CUDA(cudaMemcpyAsync(&hs, g.st, sizeof(GmState), cudaMemcpyDeviceToHost, s));
        h.check_status();
        ++syncs;
        if (hs.state == GM_NONFINITE) throw Error(PRISM_ERR_NONFINITE, "non-finite Arnoldi norm");
        const uint32_t steps = m > 0 ? hs.steps : 0;
        applies += flexible ? steps : 0;
        spmvs += steps;
        rel = hs.rel;
        m = hs.m;  // the next cycle's length (GMRES.cpp:126: m survives from cycle to cycle)
        converged = rel < o.tol;
    }
    PRISM_CUDA(cudaEventRecord(h.ev1, s));
    PRISM_CUDA(cudaMemcpyAsync(h.pinned, sc, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    h.check_status();
    ++syncs;
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
        st->host_syncs = syncs;
        st->graph_nodes = graph ? body_nodes : 0;
    }
}

}  // namespace prism
