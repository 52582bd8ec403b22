// sm_100a kernels of the solve phase.
//
// Everything here is HBM-bandwidth or latency bound integer/FP64 work: CSR
// SpMV, sync-free triangular sweeps and Krylov vector updates with fused,
// deterministic reductions.  None of it is GEMM-shaped, so none of it goes to
// the tensor cores.
#pragma once

#include "device_common.cuh"

namespace prism {


// ---------------------------------------------------------------------------
// Deterministic grid reduction ("last block finishes").
// Each block reduces NV values in a fixed tree, writes them to
// partial[block*NV + q]; the block that takes the last ticket sums all
// partials in a fixed order and stores out[q], then re-arms the ticket.
// Same grid size => bitwise identical result, run after run.
// ---------------------------------------------------------------------------

template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* smem /* [NV * 32] */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double x = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) smem[q * 32 + wid] = x;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double x = lane < nw ? smem[q * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            v[q] = x;  // valid in warp 0
        }
    }
    __syncthreads();
}

template <int NV>
__device__ __forceinline__ void grid_reduce(double (&v)[NV], ReduceSlot slot) {
    __shared__ double smem[NV * 32];
    __shared__ bool last;
    block_sum<NV>(v, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) slot.partial[blockIdx.x * NV + q] = v[q];
        __threadfence();
        unsigned t = atomicAdd(slot.ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
        for (int q = 0; q < NV; ++q) acc[q] += __ldcg(slot.partial + b * NV + q);
    }
    block_sum<NV>(acc, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) slot.out[q] = acc[q];
        *slot.ticket = 0u;
    }
}

// ---------------------------------------------------------------------------
// CSR SpMV, y = A x  (CSRMatrix::MatPVecWithRawPtr, CSRMatrix.h:360-377).
// G lanes per row, rows grid-strided.  Optionally fuses up to two dot
// products for the Krylov loop: Σ y_i z_i and Σ x_i q_i.
// ---------------------------------------------------------------------------
template <int G, int NDOT>
__global__ void __launch_bounds__(kBlock) k_spmv(uint32_t n, const uint32_t* __restrict__ rowptr,
                                                 const uint32_t* __restrict__ col, const double* __restrict__ val,
                                                 const double* __restrict__ x, double* __restrict__ y,
                                                 const double* __restrict__ z, const double* __restrict__ q,
                                                 ReduceSlot slot) {
    const int lane = threadIdx.x & (G - 1);
    const uint32_t groups = (gridDim.x * blockDim.x) / G;
    const uint32_t gid = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    const uint32_t sub = (threadIdx.x & 31) / G;  // group index inside the warp
    double acc[NDOT > 0 ? NDOT : 1];
#pragma unroll
    for (int t = 0; t < (NDOT > 0 ? NDOT : 1); ++t) acc[t] = 0.0;
    // the trip count is uniform across the warp (row0 is the warp's first group),
    // so the full-mask shuffles in group_sum are always reached by all 32 lanes
    for (uint32_t row0 = gid - sub; row0 < n; row0 += groups) {
        const uint32_t row = row0 + sub;
        double s = 0.0;
        if (row < n) {
            const uint32_t beg = __ldg(rowptr + row), end = __ldg(rowptr + row + 1);
            for (uint32_t k = beg + lane; k < end; k += G) s += __ldcs(val + k) * __ldg(x + __ldcs(col + k));
        }
        s = group_sum<G>(s);
        if (lane == 0 && row < n) {
            y[row] = s;
            if (NDOT >= 1) acc[0] += s * z[row];
            if (NDOT >= 2) acc[1] += x[row] * q[row];
        }
    }
    if (NDOT > 0) {
        double v[NDOT > 0 ? NDOT : 1];
#pragma unroll
        for (int t = 0; t < (NDOT > 0 ? NDOT : 1); ++t) v[t] = acc[t];
        grid_reduce<(NDOT > 0 ? NDOT : 1)>(v, slot);
    }
}

// ---------------------------------------------------------------------------
// Sync-free triangular sweep over a level-ordered row list.
//
//   out[r] = post( pre(in[r]) - Σ_k val[k] * out[col[k]] )
//
// Readiness is carried by the value itself: before the sweep every out[] slot
// holds kPending, a signalling-NaN bit pattern that no arithmetic result can
// take (results that are NaN are canonicalised).  A row polls its
// dependencies' slots until they differ from kPending -- one 8-byte
// single-copy-atomic word carries both the flag and the value, so no fence or
// second load is needed on the critical path.
//
// Rows are visited in level order: warp w takes positions w, w+W, w+2W, ...
// and a row only depends on rows of earlier levels, i.e. earlier positions,
// held by warps that are resident (the grid never exceeds the number of
// co-resident warps).  The lowest unfinished position therefore never waits,
// so the sweep always progresses.  Every wait is still bounded: after
// `wait_ns` without progress the warp raises *status = 6 (timeout), and all
// waiters leave as soon as they see a non-zero status.
// ---------------------------------------------------------------------------
constexpr unsigned long long kPending = 0x7FF4DEADBEEF5EEDull;
constexpr unsigned long long kCanonicalNaN = 0x7FF8000000000000ull;

enum : int { OP_DIV = 0, OP_MUL = 1, OP_NONE = 2, OP_PREDIV = 3 };

__global__ void k_fill_pending(uint32_t n, unsigned long long* __restrict__ p) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = kPending;
}

template <typename Low, int OP>
__global__ void __launch_bounds__(kBlock) k_sweep(uint32_t n, const uint32_t* __restrict__ order,
                                                  const uint32_t* __restrict__ rowptr, const uint32_t* __restrict__ col,
                                                  const Low* __restrict__ val, const double* __restrict__ diag,
                                                  const double* __restrict__ in, double* out, int* status,
                                                  unsigned long long wait_ns) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t p = warp; p < n; p += nwarps) {
        const uint32_t beg = __ldg(rowptr + p), end = __ldg(rowptr + p + 1);
        double s = 0.0;
        bool failed = false;
        for (uint32_t k = beg + lane; k < end; k += 32) {
            const uint32_t c = __ldg(col + k);
            const double a = (double)__ldg(val + k);
            unsigned long long bits = ld_relaxed_u64(out + c);
            if (bits == kPending) {
                const unsigned long long t0 = globaltimer_ns();
                unsigned spins = 0;
                do {
                    if ((++spins & 255u) == 0u) {
                        if (ld_relaxed_s32(status) != 0 || globaltimer_ns() - t0 > wait_ns) {
                            failed = true;
                            break;
                        }
                    }
                    bits = ld_relaxed_u64(out + c);
                } while (bits == kPending);
            }
            if (failed) break;
            s += a * __longlong_as_double((long long)bits);
        }
        if (__any_sync(0xffffffffu, failed)) {
            if (lane == 0) atomicCAS(status, 0, 6);
            return;
        }
        s = group_sum<32>(s);
        if (lane == 0) {
            const uint32_t r = __ldg(order + p);
            const double v = in[r];
            double res;
            if (OP == OP_DIV) res = (v - s) / diag[p];
            else if (OP == OP_MUL) res = (v - s) * diag[p];
            else if (OP == OP_NONE) res = v - s;
            else res = v / diag[p] - s;
            unsigned long long bits = (unsigned long long)__double_as_longlong(res);
            if (res != res) bits = kCanonicalNaN;
            st_relaxed_u64(out + r, bits);
        }
    }
}

// ---------------------------------------------------------------------------
// Krylov vector kernels (BaseVector::add / innerProduct / norm_2 semantics,
// BaseVector.h:279-530), each with its reduction fused.
// ---------------------------------------------------------------------------
// r = b - y (r may be null) ; out = { Σ b_i^2, Σ (b_i - y_i)^2 }
__global__ void __launch_bounds__(kBlock) k_residual(uint32_t n, const double* __restrict__ b,
                                                     const double* __restrict__ y, double* __restrict__ r,
                                                     ReduceSlot slot) {
    double v[2] = {0.0, 0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double bi = b[i];
        const double ri = bi - y[i];
        if (r) r[i] = ri;
        v[0] += bi * bi;
        v[1] += ri * ri;
    }
    grid_reduce<2>(v, slot);
}

// out = { Σ a_i b_i }
__global__ void __launch_bounds__(kBlock) k_dot(uint32_t n, const double* __restrict__ a,
                                                const double* __restrict__ b, ReduceSlot slot) {
    double v[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[0] += a[i] * b[i];
    grid_reduce<1>(v, slot);
}

// FCG direction update (CG.cpp:69-74): c = (w.v)/(d.v); d = w - c d; out = { Σ d_i r_i }
__global__ void __launch_bounds__(kBlock) k_fcg_direction(uint32_t n, const double* __restrict__ w,
                                                          double* __restrict__ d, const double* __restrict__ r,
                                                          const double* __restrict__ sc_wv,
                                                          const double* __restrict__ sc_dv, ReduceSlot slot) {
    const double c = *sc_wv / *sc_dv;
    double v[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double di = w[i] - c * d[i];
        d[i] = di;
        v[0] += di * r[i];
    }
    grid_reduce<1>(v, slot);
}

// FCG step (CG.cpp:77-79): a = (d.r)/(d.v); x += a d; r -= a v; out = { Σ r_i^2 }
__global__ void __launch_bounds__(kBlock) k_fcg_step(uint32_t n, double* __restrict__ x, double* __restrict__ r,
                                                     const double* __restrict__ d, const double* __restrict__ v,
                                                     const double* __restrict__ sc_dr,
                                                     const double* __restrict__ sc_dv, ReduceSlot slot) {
    const double a = *sc_dr / *sc_dv;
    double acc[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] = x[i] + a * d[i];
        const double ri = r[i] - a * v[i];
        r[i] = ri;
        acc[0] += ri * ri;
    }
    grid_reduce<1>(acc, slot);
}

}  // namespace prism
