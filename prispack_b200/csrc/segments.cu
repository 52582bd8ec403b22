// A batch of independent systems solved together: the handle's matrix is block
// diagonal, rows [seg_ptr[s], seg_ptr[s+1]) forming system s, and so is any
// incomplete factorisation of it (an ICT / ILDLT / ILUT of a block-diagonal
// matrix eliminates each block on its own), so one SpMV and one pair of
// triangular sweeps serve every system at once -- the sweep kernels' slabs
// follow the block boundaries.  Each system runs the recurrence of
// CG<double>::solve (CG.cpp:34-83) on its own scalars: the Krylov reductions
// are per system (one CTA per system, fixed summation order, so repeated
// solves give identical bits), a system that has converged stops changing,
// and stats[s] reports exactly what a solve of system s alone reports.
#include <cmath>
#include <cstring>

#include "../../include/prism_solve.h"
#include "kernels.cuh"
#include "solve.cuh"

namespace prism {

namespace {

// Per-system scalars, each an array of nseg doubles.
enum SegScalar : int { SG_BB = 0, SG_RES, SG_RR, SG_WV, SG_DV, SG_DR, SG_DR2, kSegScalars };

template <int NV>
__device__ __forceinline__ void seg_store(double (&v)[NV], double* const (&out)[NV], uint32_t s) {
    __shared__ double smem[NV * 32];
    block_sum<NV>(v, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) out[q][s] = v[q];
    }
}

// r = b - y (r may be null); bb[s] = Σ b², res[s] = Σ (b - y)²
__global__ void __launch_bounds__(kBlock) k_seg_residual(uint32_t nseg, const uint32_t* __restrict__ sp,
                                                         const double* __restrict__ b, const double* __restrict__ y,
                                                         double* __restrict__ r, double* bb, double* res) {
    for (uint32_t s = blockIdx.x; s < nseg; s += gridDim.x) {
        double v[2] = {0.0, 0.0};
        for (uint32_t i = sp[s] + threadIdx.x; i < sp[s + 1]; i += blockDim.x) {
            const double bi = b[i], ri = bi - y[i];
            if (r) r[i] = ri;
            v[0] += bi * bi;
            v[1] += ri * ri;
        }
        double* const out[2] = {bb, res};
        seg_store<2>(v, out, s);
    }
}

// out[s] = Σ a b over the system's rows
__global__ void __launch_bounds__(kBlock) k_seg_dot(uint32_t nseg, const uint32_t* __restrict__ sp,
                                                    const double* __restrict__ a, const double* __restrict__ b,
                                                    double* out) {
    for (uint32_t s = blockIdx.x; s < nseg; s += gridDim.x) {
        double v[1] = {0.0};
        for (uint32_t i = sp[s] + threadIdx.x; i < sp[s + 1]; i += blockDim.x) v[0] += a[i] * b[i];
        double* const o[1] = {out};
        seg_store<1>(v, o, s);
    }
}

// vd[s] = Σ v d, dr[s] = Σ d r
__global__ void __launch_bounds__(kBlock) k_seg_dot2(uint32_t nseg, const uint32_t* __restrict__ sp,
                                                     const double* __restrict__ v, const double* __restrict__ d,
                                                     const double* __restrict__ r, double* vd, double* dr) {
    for (uint32_t s = blockIdx.x; s < nseg; s += gridDim.x) {
        double acc[2] = {0.0, 0.0};
        for (uint32_t i = sp[s] + threadIdx.x; i < sp[s + 1]; i += blockDim.x) {
            acc[0] += v[i] * d[i];
            acc[1] += d[i] * r[i];
        }
        double* const out[2] = {vd, dr};
        seg_store<2>(acc, out, s);
    }
}

// active systems: c = (w.v)/(d.v); d = w - c d.  dr[s] = Σ d r (frozen systems keep d)
__global__ void __launch_bounds__(kBlock) k_seg_direction(uint32_t nseg, const uint32_t* __restrict__ sp,
                                                          const double* __restrict__ w, double* __restrict__ d,
                                                          const double* __restrict__ r, const double* __restrict__ wv,
                                                          const double* __restrict__ dv,
                                                          const int* __restrict__ active, double* dr) {
    for (uint32_t s = blockIdx.x; s < nseg; s += gridDim.x) {
        const bool on = active[s] != 0 && dv[s] != 0.0;  // dv = 0: a zero right-hand side, nothing to do
        const double c = on ? wv[s] / dv[s] : 0.0;
        double v[1] = {0.0};
        for (uint32_t i = sp[s] + threadIdx.x; i < sp[s + 1]; i += blockDim.x) {
            double di = d[i];
            if (on) {
                di = w[i] - c * di;
                d[i] = di;
            }
            v[0] += di * r[i];
        }
        double* const o[1] = {dr};
        seg_store<1>(v, o, s);
    }
}

// active systems: a = (d.r)/(d.v); x += a d; r -= a v.  rr[s] = Σ r²
__global__ void __launch_bounds__(kBlock) k_seg_step(uint32_t nseg, const uint32_t* __restrict__ sp,
                                                     double* __restrict__ x, double* __restrict__ r,
                                                     const double* __restrict__ d, const double* __restrict__ v,
                                                     const double* __restrict__ dr, const double* __restrict__ dv,
                                                     const int* __restrict__ active, double* rr) {
    for (uint32_t s = blockIdx.x; s < nseg; s += gridDim.x) {
        const bool on = active[s] != 0 && dv[s] != 0.0;
        const double a = on ? dr[s] / dv[s] : 0.0;
        double acc[1] = {0.0};
        for (uint32_t i = sp[s] + threadIdx.x; i < sp[s + 1]; i += blockDim.x) {
            double ri = r[i];
            if (on) {
                x[i] = x[i] + a * d[i];
                ri = ri - a * v[i];
                r[i] = ri;
            }
            acc[0] += ri * ri;
        }
        double* const o[1] = {rr};
        seg_store<1>(acc, o, s);
    }
}

}  // namespace

struct SegWork {
    std::vector<uint32_t> seg;   // the segment table the device copy holds
    DevBuf<uint32_t> sp;
    DevBuf<double> sc;           // kSegScalars * nseg
    DevBuf<int> active;
    std::vector<double> host;
};

void seg_release(SegWork* w) { delete w; }

void segmented_fcg_solve(Handle& h, const prism_solve_opts& o, uint32_t nseg, const uint32_t* seg_ptr,
                         const double* b, double* x, prism_solve_stats* st) {
    const uint32_t n = h.A.n;
    if (nseg == 0) throw Error(PRISM_ERR_ARG, "no systems");
    if (seg_ptr[0] != 0 || seg_ptr[nseg] != n) throw Error(PRISM_ERR_ARG, "system offsets must run from 0 to n");
    for (uint32_t s = 0; s < nseg; ++s)
        if (seg_ptr[s + 1] <= seg_ptr[s]) throw Error(PRISM_ERR_ARG, "a system without rows");
    if (!h.seg || h.seg->seg.size() != (size_t)nseg + 1 ||
        std::memcmp(h.seg->seg.data(), seg_ptr, ((size_t)nseg + 1) * sizeof(uint32_t)) != 0) {
        // a row may only couple to rows of its own system
        const CsrHost& A = h.A_host;
        for (uint32_t s = 0; s < nseg; ++s)
            for (uint32_t i = seg_ptr[s]; i < seg_ptr[s + 1]; ++i)
                for (uint32_t k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k)
                    if (A.col[k] < seg_ptr[s] || A.col[k] >= seg_ptr[s + 1])
                        throw Error(PRISM_ERR_ARG, "row " + std::to_string(i) + " couples system " +
                                                       std::to_string(s) + " to another one");
        h.seg.reset();
        auto* w = new SegWork();
        h.seg = std::unique_ptr<SegWork, void (*)(SegWork*)>(w, seg_release);
        w->seg.assign(seg_ptr, seg_ptr + nseg + 1);
        w->sp.upload(seg_ptr, (size_t)nseg + 1, h.stream);
        w->sc.alloc((size_t)kSegScalars * nseg);
        w->active.alloc(nseg);
        w->host.assign((size_t)kSegScalars * nseg, 0.0);
    }
    SegWork& w = *h.seg;
    h.ensure_workspace();
    cudaStream_t s = h.stream;
    const bool flexible = o.solver == PRISM_SOLVER_FCG;
    Precond* P = h.P.get();
    double *r = h.r.get(), *wv = h.w.get(), *d = h.d.get(), *v = h.v.get(), *y = h.y.get();
    const uint32_t* sp = w.sp.get();
    auto sc = [&](int k) { return w.sc.get() + (size_t)k * nseg; };
    const int grid = (int)std::min<uint32_t>(nseg, 65535u);
    uint32_t applies = 0, spmvs = 0;
    std::vector<int> act(nseg, 1);
    PRISM_CUDA(cudaMemcpyAsync(w.active.get(), act.data(), nseg * sizeof(int), cudaMemcpyHostToDevice, s));

    PRISM_CUDA(cudaEventRecord(h.ev0, s));
    h.spmv(x, y);
    ++spmvs;
    k_seg_residual<<<grid, kBlock, 0, s>>>(nseg, sp, b, y, r, sc(SG_BB), sc(SG_RES));
    PRISM_LAUNCHED();
    if (P) { P->apply(s, r, wv); ++applies; }
    else PRISM_CUDA(cudaMemcpyAsync(wv, r, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    PRISM_CUDA(cudaMemcpyAsync(d, wv, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    h.spmv(d, v);
    ++spmvs;
    k_seg_dot2<<<grid, kBlock, 0, s>>>(nseg, sp, v, d, r, sc(SG_DV), sc(SG_DR));
    PRISM_LAUNCHED();
    k_seg_step<<<grid, kBlock, 0, s>>>(nseg, sp, x, r, d, v, sc(SG_DR), sc(SG_DV), w.active.get(), sc(SG_RR));
    PRISM_LAUNCHED();
    PRISM_CUDA(cudaMemcpyAsync(w.host.data(), w.sc.get(), (size_t)kSegScalars * nseg * sizeof(double),
                               cudaMemcpyDeviceToHost, s));
    h.check_status();
    std::vector<double> norm_b(nseg), norm(nseg, 0.0);
    std::vector<uint32_t> m(nseg, o.max_iter);
    std::vector<int> conv(nseg, 0);
    uint32_t remaining = nseg;
    for (uint32_t q = 0; q < nseg; ++q) {
        norm_b[q] = std::sqrt(w.host[(size_t)SG_BB * nseg + q]);
        if (norm_b[q] == 0.0) {  // b = 0: x = 0 solves it; nothing to iterate
            conv[q] = 1;
            m[q] = 0;
            act[q] = 0;
            --remaining;
        }
    }
    for (uint32_t i = 1; i < o.max_iter && remaining > 0; ++i) {
        if (i > 1) {
            PRISM_CUDA(cudaMemcpyAsync(w.host.data() + (size_t)SG_RR * nseg, sc(SG_RR), nseg * sizeof(double),
                                       cudaMemcpyDeviceToHost, s));
            h.check_status();
        }
        bool changed = false;
        for (uint32_t q = 0; q < nseg; ++q) {
            if (!act[q]) continue;
            norm[q] = std::sqrt(w.host[(size_t)SG_RR * nseg + q]) / norm_b[q];
            if (!std::isfinite(norm[q]))
                throw Error(PRISM_ERR_NONFINITE, "non-finite residual norm of system " + std::to_string(q) +
                                                     " in CG iteration " + std::to_string(i));
            if (norm[q] < o.tol) {
                conv[q] = 1;
                m[q] = i;
                act[q] = 0;
                --remaining;
                changed = true;
            }
        }
        if (remaining == 0) break;
        if (changed)
            PRISM_CUDA(cudaMemcpyAsync(w.active.get(), act.data(), nseg * sizeof(int), cudaMemcpyHostToDevice, s));
        if (flexible && P) { P->apply(s, r, wv); ++applies; }
        else PRISM_CUDA(cudaMemcpyAsync(wv, r, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        k_seg_dot<<<grid, kBlock, 0, s>>>(nseg, sp, wv, v, sc(SG_WV));
        PRISM_LAUNCHED();
        k_seg_direction<<<grid, kBlock, 0, s>>>(nseg, sp, wv, d, r, sc(SG_WV), sc(SG_DV), w.active.get(),
                                               sc(SG_DR2));
        PRISM_LAUNCHED();
        h.spmv(d, v);
        ++spmvs;
        k_seg_dot<<<grid, kBlock, 0, s>>>(nseg, sp, v, d, sc(SG_DV));
        PRISM_LAUNCHED();
        k_seg_step<<<grid, kBlock, 0, s>>>(nseg, sp, x, r, d, v, sc(SG_DR2), sc(SG_DV), w.active.get(),
                                          sc(SG_RR));
        PRISM_LAUNCHED();
    }
    h.spmv(x, y);
    ++spmvs;
    k_seg_residual<<<grid, kBlock, 0, s>>>(nseg, sp, b, y, nullptr, sc(SG_BB), sc(SG_RES));
    PRISM_LAUNCHED();
    PRISM_CUDA(cudaEventRecord(h.ev1, s));
    PRISM_CUDA(cudaMemcpyAsync(w.host.data(), w.sc.get(), 2 * (size_t)nseg * sizeof(double), cudaMemcpyDeviceToHost,
                               s));
    h.check_status();
    float ms = 0.f;
    PRISM_CUDA(cudaEventElapsedTime(&ms, h.ev0, h.ev1));
    if (st) {
        for (uint32_t q = 0; q < nseg; ++q) {
            const double bb = w.host[(size_t)SG_BB * nseg + q], res = w.host[(size_t)SG_RES * nseg + q];
            st[q].num_iter = (int32_t)(m[q] + 1);
            st[q].converged = conv[q];
            st[q].final_error = norm[q];
            st[q].true_rel_residual = bb > 0.0 ? std::sqrt(res) / std::sqrt(bb) : 0.0;
            st[q].precond_applies = applies;
            st[q].spmv_count = spmvs;
            st[q].device_ms = ms;
            st[q].forward_error = -1.0;  // no reference solution for block / batch solves
            st[q].host_syncs = 0;  // not counted for block / batch solves
            st[q].graph_nodes = 0;
        }
    }
}

}  // namespace prism
