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
// CSR SpMV, y = A x  (CSRMatrix::MatPVecWithRawPtr, CSRMatrix.h:360-377),
// optionally fused with up to two dot products for the Krylov loop:
// Σ y_i z_i and Σ x_i q_i (deterministic grid reduction).
//
// A G-lane group takes U rows per pass (rows T + sub + u * 32/G of the warp's
// tile of U * 32/G consecutive rows); all U rows' offsets, their first 8/G
// entries per lane and the x gathers are issued before any of them is used,
// so memory in flight, not latency, sets the pace.  Rows longer than 8
// entries finish in a loop.  The operator uses G = 1, U = 2 (one thread per
// row, two rows at a time: 61% of measured HBM bandwidth on 3D Poisson 128^3,
// against 37% for eight lanes per row); with G = 1 each row is summed in
// stored column order, as the reference's row loop does.
// ---------------------------------------------------------------------------
template <int G, int U, int NDOT>
static __global__ void __launch_bounds__(kBlock) k_spmv(uint32_t n, const uint32_t* __restrict__ rowptr,
                                                   const uint32_t* __restrict__ col, const double* __restrict__ val,
                                                   const double* __restrict__ x, double* __restrict__ y,
                                                   const double* __restrict__ z, const double* __restrict__ q,
                                                   ReduceSlot slot) {
    constexpr int GPW = 32 / G;            // groups per warp
    constexpr int CH = G >= 8 ? 1 : 8 / G; // entries per lane issued up front
    const int lane = threadIdx.x & (G - 1);
    const uint32_t sub = (threadIdx.x & 31) / G;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    double acc[NDOT > 0 ? NDOT : 1];
#pragma unroll
    for (int t = 0; t < (NDOT > 0 ? NDOT : 1); ++t) acc[t] = 0.0;
    for (uint32_t tile = warp * (uint32_t)(GPW * U); tile < n; tile += nwarps * (uint32_t)(GPW * U)) {
        uint32_t beg[U], end[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t r = tile + sub + (uint32_t)(u * GPW);
            beg[u] = r < n ? __ldg(rowptr + r) : 0u;
            end[u] = r < n ? __ldg(rowptr + r + 1) : 0u;
        }
        uint32_t c[U][CH];
        double a[U][CH];
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int h = 0; h < CH; ++h) {
                const uint32_t k = beg[u] + (uint32_t)lane + (uint32_t)(h * G);
                const bool in = k < end[u];
                c[u][h] = in ? __ldcs(col + k) : 0u;
                a[u][h] = in ? __ldcs(val + k) : 0.0;
            }
        double s[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            s[u] = 0.0;
#pragma unroll
            for (int h = 0; h < CH; ++h) s[u] += a[u][h] * __ldg(x + c[u][h]);
            for (uint32_t k = beg[u] + (uint32_t)lane + (uint32_t)(CH * G); k < end[u]; k += G)
                s[u] += __ldcs(val + k) * __ldg(x + __ldcs(col + k));
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t r = tile + sub + (uint32_t)(u * GPW);
            const double t = group_sum<G>(s[u]);
            if (lane == 0 && r < n) {
                y[r] = t;
                if (NDOT >= 1) acc[0] += t * z[r];
                if (NDOT >= 2) acc[1] += x[r] * q[r];
            }
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
// holds kPending, a signalling-NaN bit pattern that no arithmetic result takes
// (NaN results are canonicalised).  One 8-byte single-copy-atomic word carries
// both the flag and the value, so no fence and no second load sits on the
// critical path.
//
// Rows are visited in level order: warp w takes positions w, w+W, w+2W, ...
// A row depends only on rows of earlier levels, i.e. earlier positions, held
// by warps that are resident (cooperative launch), so the lowest unfinished
// position never waits and the sweep always progresses.
//
// Latency hiding: while a row waits, the warp has already loaded the next
// row's offsets, column indices, values, diagonal, right-hand side and the
// current value of every dependency (all independent of the wait).  When the
// warp turns to that row, only the dependencies that were still pending are
// polled, by their own lanes; the others cost nothing more.  Every wait is
// bounded: after `wait_ns` without progress the warp raises *status = 6
// (timeout) and every waiter leaves as soon as it sees a non-zero status.
// ---------------------------------------------------------------------------
constexpr unsigned long long kPending = 0x7FF4DEADBEEF5EEDull;
constexpr unsigned long long kCanonicalNaN = 0x7FF8000000000000ull;

enum : int { OP_DIV = 0, OP_MUL = 1, OP_NONE = 2, OP_PREDIV = 3 };

static __global__ void k_fill_pending(uint32_t n, unsigned long long* __restrict__ p) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = kPending;
}

// One row of a sweep as a warp holds it: lane k owns the k-th stored entry
// (rows longer than 32 entries continue in a loop); `bits` is the value of the
// lane's dependency as last seen (kPending if not produced yet).
struct SweepRow {
    uint32_t beg, end, r;
    uint32_t c;                 // this lane's dependency row (first 32 entries)
    double a;                   // its coefficient
    unsigned long long bits;    // its value, loaded when the row was prefetched
    double d, v;                // diagonal and right-hand side (lane 0)
};

// Loads a row's offsets, entries, diagonal, right-hand side and -- already --
// the current value of each dependency; all of it is independent of the
// wait, so it overlaps the previous row's wait.  `dep` is a callable loading
// a dependency's current bits.
template <typename Low, typename Dep>
__device__ __forceinline__ void prefetch_row(SweepRow& m, uint32_t p, int lane, const uint32_t* __restrict__ order,
                                             const uint32_t* __restrict__ rowptr, const uint32_t* __restrict__ col,
                                             const Low* __restrict__ val, const double* __restrict__ diag,
                                             const double* __restrict__ in, Dep&& dep) {
    m.beg = __ldg(rowptr + p);
    m.end = __ldg(rowptr + p + 1);
    m.r = __ldg(order + p);
    m.c = 0;
    m.a = 0.0;
    m.bits = 0ull;
    if (m.beg + lane < m.end) {
        m.c = __ldcs(col + m.beg + lane);
        m.a = (double)__ldcs(val + m.beg + lane);
        m.bits = dep(m.c);
    }
    if (lane == 0) {
        m.d = __ldg(diag + p);
        m.v = __ldg(in + m.r);
    }
}

// Finishes a prefetched row: polls only the dependencies that were still
// pending, reduces, and returns the row's value in lane 0 (false: a wait ran out).
template <typename Low, int OP, typename Wait>
__device__ __forceinline__ bool finish_row(const SweepRow& m, int lane, const uint32_t* __restrict__ col,
                                           const Low* __restrict__ val, Wait&& wait, unsigned long long& out_bits) {
    bool ok = true;
    double s = 0.0;
    if (m.beg + lane < m.end) {
        unsigned long long bits = m.bits;
        if (bits == kPending) ok = wait(m.c, bits);
        s = m.a * __longlong_as_double((long long)bits);
    }
    for (uint32_t k = m.beg + 32 + lane; ok && k < m.end; k += 32) {  // rows longer than a warp
        unsigned long long bits;
        ok = wait(__ldcs(col + k), bits);
        s += (double)__ldcs(val + k) * __longlong_as_double((long long)bits);
    }
    if (!__all_sync(0xffffffffu, ok)) return false;
    s = group_sum<32>(s);
    double res;
    if (OP == OP_DIV) res = (m.v - s) / m.d;
    else if (OP == OP_MUL) res = (m.v - s) * m.d;
    else if (OP == OP_NONE) res = m.v - s;
    else res = m.v / m.d - s;
    out_bits = (unsigned long long)__double_as_longlong(res);
    if (res != res) out_bits = kCanonicalNaN;
    return true;
}

// Spin on a word until it is no longer kPending; false when the wait gave up.
template <typename Load>
__device__ __forceinline__ bool spin_ready(Load&& load, unsigned long long& bits, const int* status,
                                           unsigned long long wait_ns) {
    bits = load();
    if (bits != kPending) return true;
    const unsigned long long t0 = globaltimer_ns();
    unsigned spins = 0;
    do {
        if ((++spins & 255u) == 0u) {
            if (ld_relaxed_s32(status) != 0 || globaltimer_ns() - t0 > wait_ns) return false;
        }
        bits = load();
    } while (bits == kPending);
    return true;
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
    auto dep = [&](uint32_t c) { return ld_relaxed_u64(out + c); };
    auto wait = [&](uint32_t c, unsigned long long& bits) {
        return spin_ready([&] { return ld_relaxed_u64(out + c); }, bits, status, wait_ns);
    };
    uint32_t p = warp;
    if (p >= n) return;
    SweepRow cur, nxt;
    prefetch_row<Low>(cur, p, lane, order, rowptr, col, val, diag, in, dep);
    while (true) {
        const uint32_t pn = p + nwarps;
        if (pn < n) prefetch_row<Low>(nxt, pn, lane, order, rowptr, col, val, diag, in, dep);
        unsigned long long rb;
        if (!finish_row<Low, OP>(cur, lane, col, val, wait, rb)) {
            if (lane == 0) atomicCAS(status, 0, 6);
            return;
        }
        if (lane == 0) st_relaxed_u64(out + cur.r, rb);
        if (pn >= n) break;
        cur = nxt;
        p = pn;
    }
}

// ---------------------------------------------------------------------------
// Slab-blocked sync-free sweep.
//
// CTA b owns the contiguous rows [rb, re) = [b*rows_per_cta, ...) and visits
// them in (level, row) order (positions [cta_pos[b], cta_pos[b+1]) of the slab
// layout); its warps take those positions round-robin.  The CTA keeps the
// values of its own rows in shared memory (the first `smem_rows` of them), so
// a dependency produced inside the slab is a shared-memory poll of a few tens
// of cycles; only dependencies owned by other slabs poll global memory.  Each
// finished row is written to both.  Readiness uses the same kPending encoding
// as k_sweep, in shared memory (initialised by the CTA itself) and in global
// memory (initialised by k_fill_pending before the launch).
//
// Progress: take the unfinished row of lowest level.  Its dependencies are
// finished; in its CTA every earlier position has a level no higher than its
// own, so those rows can finish too, and the warp that owns the position
// reaches it.  All CTAs are co-resident (cooperative launch), so no CTA waits
// for one that is not running.  Waits are bounded as in k_sweep.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long ld_shared_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.volatile.shared.u64 %0, [%1];" : "=l"(v) : "r"((unsigned)__cvta_generic_to_shared(p)) : "memory");
    return v;
}
__device__ __forceinline__ void st_shared_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.volatile.shared.u64 [%0], %1;" ::"r"((unsigned)__cvta_generic_to_shared(p)), "l"(v) : "memory");
}

template <typename Low, int OP>
static __global__ void __launch_bounds__(1024) k_sweep_slab(uint32_t n, uint32_t rows_per_cta, uint32_t smem_rows,
                                                     const uint32_t* __restrict__ cta_pos,
                                                     const uint32_t* __restrict__ order,
                                                     const uint32_t* __restrict__ rowptr,
                                                     const uint32_t* __restrict__ col, const Low* __restrict__ val,
                                                     const double* __restrict__ diag, const double* __restrict__ in,
                                                     double* out, int* status, unsigned long long wait_ns) {
    extern __shared__ unsigned long long xs[];
    const uint32_t b = blockIdx.x;
    const uint32_t rb = b * rows_per_cta;
    const uint32_t re = min(n, rb + rows_per_cta);
    const uint32_t owned = re > rb ? re - rb : 0;
    const uint32_t local_rows = min(owned, smem_rows);
    for (uint32_t i = threadIdx.x; i < local_rows; i += blockDim.x) xs[i] = kPending;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint32_t wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t p0 = cta_pos[b], p1 = cta_pos[b + 1];
    auto load = [&](uint32_t c) {
        const uint32_t lc = c - rb;  // wraps for c < rb
        return lc < local_rows ? ld_shared_u64(xs + lc) : ld_relaxed_u64(out + c);
    };
    auto wait = [&](uint32_t c, unsigned long long& bits) {
        return spin_ready([&] { return load(c); }, bits, status, wait_ns);
    };
    // Dependencies inside the slab are produced by neighbouring positions and
    // would still be pending when the row is read ahead, so they are polled
    // (in shared memory) only when the row is reached; dependencies owned by
    // other slabs, usually finished long before, are loaded ahead with the row.
    auto later = [&](uint32_t c) { return (c - rb) < owned ? kPending : ld_relaxed_u64(out + c); };
    uint32_t p = p0 + wid;
    if (p >= p1) return;
    SweepRow cur, nxt;
    prefetch_row<Low>(cur, p, lane, order, rowptr, col, val, diag, in, later);
    while (true) {
        const uint32_t pn = p + nw;
        if (pn < p1) prefetch_row<Low>(nxt, pn, lane, order, rowptr, col, val, diag, in, later);
        unsigned long long rbits;
        if (!finish_row<Low, OP>(cur, lane, col, val, wait, rbits)) {
            if (lane == 0) atomicCAS(status, 0, 6);
            return;
        }
        if (lane == 0) {
            const uint32_t lr = cur.r - rb;
            if (lr < local_rows) st_shared_u64(xs + lr, rbits);
            st_relaxed_u64(out + cur.r, rbits);
        }
        if (pn >= p1) break;
        cur = nxt;
        p = pn;
    }
}

// ---------------------------------------------------------------------------
// Krylov vector kernels (BaseVector::add / innerProduct / norm_2 semantics,
// BaseVector.h:279-530), each with its reduction fused.
// ---------------------------------------------------------------------------
// r = b - y (r may be null) ; out = { Σ b_i^2, Σ (b_i - y_i)^2 }
static __global__ void __launch_bounds__(kBlock) k_residual(uint32_t n, const double* __restrict__ b,
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
static __global__ void __launch_bounds__(kBlock) k_dot(uint32_t n, const double* __restrict__ a,
                                                const double* __restrict__ b, ReduceSlot slot) {
    double v[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[0] += a[i] * b[i];
    grid_reduce<1>(v, slot);
}

// FCG direction update (CG.cpp:69-74): c = (w.v)/(d.v); d = w - c d; out = { Σ d_i r_i }
static __global__ void __launch_bounds__(kBlock) k_fcg_direction(uint32_t n, const double* __restrict__ w,
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
static __global__ void __launch_bounds__(kBlock) k_fcg_step(uint32_t n, double* __restrict__ x, double* __restrict__ r,
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

namespace prism {
// ---------------------------------------------------------------------------
// GMRES kernels (GMRES<double>::solve, GMRES.cpp:122-221)
// ---------------------------------------------------------------------------
// dst = src * alpha (BaseVector::scale by a reciprocal, GMRES.cpp:158,188)
static __global__ void __launch_bounds__(kBlock) k_scale(uint32_t n, const double* __restrict__ src, double alpha,
                                                         double* __restrict__ dst) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[i] * alpha;
}

// x += B * ksi over ncols columns of a column-major n x ncols block, summed
// column by column per element (DenseMatrix::MatVec, DenseMatrix.cpp:208-243).
static __global__ void __launch_bounds__(kBlock) k_gemv_add(uint32_t n, const double* __restrict__ B, uint32_t ncols,
                                                            const double* __restrict__ ksi, double* __restrict__ x) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (uint32_t c = 0; c < ncols; ++c) acc += B[(size_t)c * n + i] * ksi[c];
        x[i] = x[i] + 1.0 * acc;
    }
}
}  // namespace prism

namespace prism {
// ---------------------------------------------------------------------------
// AMSED apply kernels (AMSEDPrecondition::MInvSolve / levelCInvRecursiveSolve,
// AMSEDPrecondition.cpp:1494-1587, 1976-2087)
// ---------------------------------------------------------------------------
// out[i] = in[perm[i]]  (prepareRightHand) / out[perm[i]] = in[i] (recoverRightHand)
static __global__ void __launch_bounds__(kBlock) k_permute(uint32_t n, const uint32_t* __restrict__ perm,
                                                           const double* __restrict__ in, double* __restrict__ out,
                                                           int scatter) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (scatter) out[perm[i]] = in[i];
        else out[i] = in[perm[i]];
    }
}

// y[i] -= Σ_k M[i,k] x[k]   (x2 -= E^T x1 with E^T stored explicitly; one warp-group per row)
template <int G>
static __global__ void __launch_bounds__(kBlock) k_spmv_sub(uint32_t n, const uint32_t* __restrict__ rowptr,
                                                            const uint32_t* __restrict__ col,
                                                            const double* __restrict__ val,
                                                            const double* __restrict__ x, double* __restrict__ y) {
    const int lane = threadIdx.x & (G - 1);
    const uint32_t groups = (gridDim.x * blockDim.x) / G;
    const uint32_t gid = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    const uint32_t sub = (threadIdx.x & 31) / G;
    for (uint32_t row0 = gid - sub; row0 < n; row0 += groups) {
        const uint32_t row = row0 + sub;
        double s = 0.0;
        if (row < n)
            for (uint32_t k = __ldg(rowptr + row) + lane; k < __ldg(rowptr + row + 1); k += G)
                s += __ldg(val + k) * __ldg(x + __ldg(col + k));
        s = group_sum<G>(s);
        if (lane == 0 && row < n) y[row] -= s;
    }
}

// y -= x
static __global__ void __launch_bounds__(kBlock) k_sub(uint32_t n, const double* __restrict__ x, double* __restrict__ y) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] -= x[i];
}

// Low-rank correction, first half: partial[b*r + c] = Σ_{j in block b} W[c*n + j] * x[j]
// (W column-major n x r, r <= kMaxRank).  Each block strides over rows; the r
// partial sums are reduced in a fixed order by k_lowrank_finish.
constexpr int kMaxRank = 128;
static __global__ void __launch_bounds__(kBlock) k_lowrank_dots(uint32_t n, uint32_t r, const double* __restrict__ W,
                                                                const double* __restrict__ x,
                                                                double* __restrict__ partial) {
    __shared__ double acc[kMaxRank][kBlock / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (uint32_t c = 0; c < r; ++c) {
        double s = 0.0;
        const double* wc = W + (size_t)c * n;
        for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
            s += wc[j] * x[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) acc[c][wid] = s;
    }
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < r; c += blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) s += acc[c][w];
        partial[(size_t)blockIdx.x * r + c] = s;
    }
}

// t[c] = H[c] * Σ_b partial[b*r + c]  (one block, fixed order)
static __global__ void k_lowrank_finish(uint32_t nblocks, uint32_t r, const double* __restrict__ partial,
                                        const double* __restrict__ H, double* __restrict__ t) {
    for (uint32_t c = threadIdx.x; c < r; c += blockDim.x) {
        double s = 0.0;
        for (uint32_t b = 0; b < nblocks; ++b) s += partial[(size_t)b * r + c];
        t[c] = s * H[c];
    }
}

// y[j] += Σ_c W[c*n + j] * t[c]   (DenseMatrix::MatVec then x2 += ..., column order per element)
static __global__ void __launch_bounds__(kBlock) k_lowrank_add(uint32_t n, uint32_t r, const double* __restrict__ W,
                                                               const double* __restrict__ t, double* __restrict__ y) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (uint32_t c = 0; c < r; ++c) s += W[(size_t)c * n + j] * t[c];
        y[j] += s;
    }
}
}  // namespace prism

namespace prism {
// ---------------------------------------------------------------------------
// Adjoint of x = A^{-1} b on A's stored pattern: dL/dA_ij = -lambda_i x_j,
// with lambda = A^{-T} dL/dx.  One thread per row, entries in stored order.
// ---------------------------------------------------------------------------
static __global__ void __launch_bounds__(kBlock) k_adjoint_outer(uint32_t n, const uint32_t* __restrict__ rowptr,
                                                                 const uint32_t* __restrict__ col,
                                                                 const double* __restrict__ lambda,
                                                                 const double* __restrict__ x,
                                                                 double* __restrict__ grad) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double li = -lambda[i];
        for (uint32_t k = rowptr[i]; k < rowptr[i + 1]; ++k) grad[k] = li * x[col[k]];
    }
}
}  // namespace prism
