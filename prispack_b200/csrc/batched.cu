// Block of right-hand sides: k <= 64 independent FCG solves that share A and
// the preconditioner, run as one sequence of launches.
//
// Layout.  Inside the solve every block vector is interleaved, X[row * k + c],
// so that one warp reads or writes a whole row of the block in one or two
// coalesced 256-byte transactions.  Lane l owns columns l and l + 32.  The
// caller's blocks are column-major (ld >= n) and are converted on entry and
// exit by a shared-memory tiled transpose.
//
// Why a block pays on the sweeps: a triangular sweep is a chain of dependency
// wavefronts whose latency (two L2 round trips each) does not depend on how
// many values a row carries.  With k columns one wavefront moves k values per
// row, so the same chain of latencies serves k solves.
//
// Each column follows the recurrence of CG<double>::solve (CG.cpp:34-83) on
// its own scalars; a column that has converged is frozen (its x and r stop
// changing, its direction stops changing) while the others go on, so every
// column ends with the iterate, iteration count and error the single solve
// would report.  Reductions are per column and deterministic (fixed-order
// block and grid sums).
#include <cmath>
#include <cstring>

#include "../../include/prism_solve.h"
#include "kernels.cuh"
#include "solve.cuh"

namespace prism {

namespace {

constexpr int kBK = 64;                                 // columns per block solve
constexpr int kBWarps = kBlock / 32;                    // warps per block
constexpr unsigned long long kBWaitNs = 1000000000ull;  // 1 s per dependency wait

// Scalar slots of the batched reductions, each kBK wide.
enum BScalar : int { BS_BB = 0, BS_RES = 1, BS_RR = 2, BS_WV = 3, BS_DV = 4, BS_DR = 5, BS_DR2 = 6, kBScalars = 8 };

struct BSlot {
    double* partial;   // [grid][NV][kBK]
    unsigned* ticket;  // 0 between launches
    double* out;       // [NV][kBK], consecutive slots
};

// Per-column block + grid reduction of NV values.  v[q][h] is this lane's
// partial sum for column lane + 32 h.  Same grid => same bits.
template <int NV>
__device__ __forceinline__ void bt_reduce(double (&v)[NV][2], BSlot slot) {
    static_assert(NV * kBK <= kBlock, "one thread per (value, column)");
    __shared__ double sm[kBWarps][NV][kBK];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        sm[wid][q][lane] = v[q][0];
        sm[wid][q][lane + 32] = v[q][1];
    }
    __syncthreads();
    const int t = threadIdx.x;
    if (t < NV * kBK) {
        const int q = t / kBK, c = t % kBK;
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kBWarps; ++w) s += sm[w][q][c];
        slot.partial[((size_t)blockIdx.x * NV + q) * kBK + c] = s;
        __threadfence();
    }
    __syncthreads();
    if (t == 0) last = atomicAdd(slot.ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (t < NV * kBK) {
        const int q = t / kBK, c = t % kBK;
        double s = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) s += __ldcg(slot.partial + ((size_t)b * NV + q) * kBK + c);
        slot.out[q * kBK + c] = s;
    }
    if (t == 0) *slot.ticket = 0u;
}

// column-major (ld) <-> interleaved, 32 rows x k columns per block through shared memory
__global__ void __launch_bounds__(kBlock) k_bt_pack(uint32_t n, uint32_t k, uint64_t ld,
                                                    const double* __restrict__ src, double* __restrict__ dst) {
    __shared__ double tile[32][kBK + 1];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (uint64_t r0 = (uint64_t)blockIdx.x * 32; r0 < n; r0 += (uint64_t)gridDim.x * 32) {
        const uint64_t r = r0 + lane;
        for (uint32_t c = wid; c < k; c += kBWarps) tile[lane][c] = r < n ? src[c * ld + r] : 0.0;
        __syncthreads();
        for (int i = wid; i < 32; i += kBWarps) {
            const uint64_t rr = r0 + i;
            if (rr < n) {
                if ((uint32_t)lane < k) dst[rr * k + lane] = tile[i][lane];
                if ((uint32_t)lane + 32 < k) dst[rr * k + lane + 32] = tile[i][lane + 32];
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kBlock) k_bt_unpack(uint32_t n, uint32_t k, uint64_t ld,
                                                      const double* __restrict__ src, double* __restrict__ dst) {
    __shared__ double tile[32][kBK + 1];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (uint64_t r0 = (uint64_t)blockIdx.x * 32; r0 < n; r0 += (uint64_t)gridDim.x * 32) {
        for (int i = wid; i < 32; i += kBWarps) {
            const uint64_t rr = r0 + i;
            if (rr < n) {
                if ((uint32_t)lane < k) tile[i][lane] = src[rr * k + lane];
                if ((uint32_t)lane + 32 < k) tile[i][lane + 32] = src[rr * k + lane + 32];
            }
        }
        __syncthreads();
        const uint64_t r = r0 + lane;
        if (r < n)
            for (uint32_t c = wid; c < k; c += kBWarps) dst[c * ld + r] = tile[lane][c];
        __syncthreads();
    }
}

// Y = A X (interleaved, warp per row); NDOT = 1: Σ y z per column; NDOT = 2: also Σ x q.
template <int NDOT>
__global__ void __launch_bounds__(kBlock) k_bt_spmm(uint32_t n, uint32_t k, const uint32_t* __restrict__ rowptr,
                                                    const uint32_t* __restrict__ col, const double* __restrict__ val,
                                                    const double* __restrict__ X, double* __restrict__ Y,
                                                    const double* __restrict__ Z, const double* __restrict__ Q,
                                                    BSlot slot) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const bool h0 = (uint32_t)lane < k, h1 = (uint32_t)lane + 32 < k;
    double acc[NDOT > 0 ? NDOT : 1][2] = {};
    for (uint32_t row = warp; row < n; row += nwarps) {
        const uint32_t beg = __ldg(rowptr + row), end = __ldg(rowptr + row + 1);
        double s0 = 0.0, s1 = 0.0;
        for (uint32_t e0 = beg; e0 < end; e0 += 32) {
            uint32_t cc = 0;
            double aa = 0.0;
            if (e0 + lane < end) {
                cc = __ldcs(col + e0 + lane);
                aa = __ldcs(val + e0 + lane);
            }
            const int cnt = (int)min(32u, end - e0);
            for (int t = 0; t < cnt; ++t) {
                const uint64_t c = __shfl_sync(0xffffffffu, cc, t);
                const double a = __shfl_sync(0xffffffffu, aa, t);
                if (h0) s0 += a * __ldg(X + c * k + lane);
                if (h1) s1 += a * __ldg(X + c * k + lane + 32);
            }
        }
        const uint64_t o = (uint64_t)row * k;
        if (h0) {
            Y[o + lane] = s0;
            if (NDOT >= 1) acc[0][0] += s0 * Z[o + lane];
            if (NDOT >= 2) acc[NDOT - 1][0] += X[o + lane] * Q[o + lane];
        }
        if (h1) {
            Y[o + lane + 32] = s1;
            if (NDOT >= 1) acc[0][1] += s1 * Z[o + lane + 32];
            if (NDOT >= 2) acc[NDOT - 1][1] += X[o + lane + 32] * Q[o + lane + 32];
        }
    }
    if (NDOT > 0) bt_reduce<(NDOT > 0 ? NDOT : 1)>(acc, slot);
}

// R = B - Y (R may be null); out = { Σ b², Σ (b - y)² } per column
__global__ void __launch_bounds__(kBlock) k_bt_residual(uint32_t n, uint32_t k, const double* __restrict__ B,
                                                        const double* __restrict__ Y, double* __restrict__ R,
                                                        BSlot slot) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    double v[2][2] = {};
    for (uint32_t row = warp; row < n; row += nwarps) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint32_t c = lane + 32 * h;
            if (c < k) {
                const uint64_t i = (uint64_t)row * k + c;
                const double b = B[i], r = b - Y[i];
                if (R) R[i] = r;
                v[0][h] += b * b;
                v[1][h] += r * r;
            }
        }
    }
    bt_reduce<2>(v, slot);
}

// out = { Σ a b } per column
__global__ void __launch_bounds__(kBlock) k_bt_dot(uint32_t n, uint32_t k, const double* __restrict__ A,
                                                   const double* __restrict__ B, BSlot slot) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    double v[1][2] = {};
    for (uint32_t row = warp; row < n; row += nwarps) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint32_t c = lane + 32 * h;
            if (c < k) v[0][h] += A[(uint64_t)row * k + c] * B[(uint64_t)row * k + c];
        }
    }
    bt_reduce<1>(v, slot);
}

// Active columns: c = (w.v)/(d.v); d = w - c d.  Out: Σ d r per column (frozen columns keep d).
__global__ void __launch_bounds__(kBlock) k_bt_fcg_direction(uint32_t n, uint32_t k, const double* __restrict__ W,
                                                             double* __restrict__ D, const double* __restrict__ R,
                                                             const double* __restrict__ wv,
                                                             const double* __restrict__ dv,
                                                             const int* __restrict__ active, BSlot slot) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    double coef[2] = {0.0, 0.0};
    bool on[2] = {false, false};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const uint32_t c = lane + 32 * h;
        if (c < k && active[c]) {
            on[h] = true;
            coef[h] = wv[c] / dv[c];
        }
    }
    double v[1][2] = {};
    for (uint32_t row = warp; row < n; row += nwarps) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint32_t c = lane + 32 * h;
            if (c < k) {
                const uint64_t i = (uint64_t)row * k + c;
                double d = D[i];
                if (on[h]) {
                    d = W[i] - coef[h] * d;
                    D[i] = d;
                }
                v[0][h] += d * R[i];
            }
        }
    }
    bt_reduce<1>(v, slot);
}

// Active columns: a = (d.r)/(d.v); x += a d; r -= a v.  Out: Σ r² per column.
__global__ void __launch_bounds__(kBlock) k_bt_fcg_step(uint32_t n, uint32_t k, double* __restrict__ X,
                                                        double* __restrict__ R, const double* __restrict__ D,
                                                        const double* __restrict__ V, const double* __restrict__ dr,
                                                        const double* __restrict__ dv, const int* __restrict__ active,
                                                        BSlot slot) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    double a[2] = {0.0, 0.0};
    bool on[2] = {false, false};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const uint32_t c = lane + 32 * h;
        if (c < k && active[c]) {
            on[h] = true;
            a[h] = dr[c] / dv[c];
        }
    }
    double v[1][2] = {};
    for (uint32_t row = warp; row < n; row += nwarps) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint32_t c = lane + 32 * h;
            if (c < k) {
                const uint64_t i = (uint64_t)row * k + c;
                double r = R[i];
                if (on[h]) {
                    X[i] += a[h] * D[i];
                    r -= a[h] * V[i];
                    R[i] = r;
                }
                v[0][h] += r * r;
            }
        }
    }
    bt_reduce<1>(v, slot);
}

__global__ void k_bt_fill_pending(uint64_t count, unsigned long long* __restrict__ p) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = kPending;
}

// ---------------------------------------------------------------------------
// Block triangular sweep: the rows of a level-ordered sweep (see k_sweep),
// warp per row, lane l computing columns l and l + 32 of the row:
//   out[r][c] = post( pre(in[r][c]) - Σ_e val[e] * out[col[e]][c] ).
// A row's stored entries are fetched once by the warp; the dependency values
// are loaded eight entries at a time before any of them is waited on, so the
// waits of one row overlap.  Readiness is the kPending encoding of k_sweep,
// per value; each lane waits only on its own columns.  Waits are bounded
// (status 6).  Positions are taken round-robin by co-resident warps
// (cooperative launch): the unfinished position of lowest level never waits
// on an unfinished one, so the sweep always progresses.
// ---------------------------------------------------------------------------
template <typename Low, int OP>
__global__ void __launch_bounds__(kBlock) k_bt_sweep(uint32_t n, uint32_t k, const uint32_t* __restrict__ order,
                                                     const uint32_t* __restrict__ rowptr,
                                                     const uint32_t* __restrict__ col, const Low* __restrict__ val,
                                                     const double* __restrict__ diag, const double* __restrict__ in,
                                                     double* out, int* status, unsigned long long wait_ns) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const bool h0 = (uint32_t)lane < k, h1 = (uint32_t)lane + 32 < k;
    for (uint32_t p = warp; p < n; p += nwarps) {
        const uint32_t beg = __ldg(rowptr + p), end = __ldg(rowptr + p + 1);
        const uint64_t r = __ldg(order + p);
        const double dg = (OP == OP_NONE) ? 1.0 : __ldg(diag + p);
        const double v0 = h0 ? __ldg(in + r * k + lane) : 0.0;
        const double v1 = h1 ? __ldg(in + r * k + lane + 32) : 0.0;
        double s0 = 0.0, s1 = 0.0;
        bool ok = true;
        for (uint32_t e0 = beg; e0 < end; e0 += 32) {
            uint32_t cc = 0;
            double aa = 0.0;
            if (e0 + lane < end) {
                cc = __ldcs(col + e0 + lane);
                aa = (double)__ldcs(val + e0 + lane);
            }
            const int cnt = (int)min(32u, end - e0);
            for (int t0 = 0; t0 < cnt; t0 += 8) {
                // issue the loads of eight entries, then wait on the pending ones
                uint64_t cj[8];
                double a[8];
                unsigned long long b0[8], b1[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int t = t0 + j;
                    cj[j] = __shfl_sync(0xffffffffu, cc, t & 31);
                    a[j] = __shfl_sync(0xffffffffu, aa, t & 31);
                    b0[j] = (t < cnt && h0) ? ld_relaxed_u64(out + cj[j] * k + lane) : 0ull;
                    b1[j] = (t < cnt && h1) ? ld_relaxed_u64(out + cj[j] * k + lane + 32) : 0ull;
                }
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    if (t0 + j < cnt) {
                        const double* p0 = out + cj[j] * k + lane;
                        if (ok && b0[j] == kPending)
                            ok = spin_ready([&] { return ld_relaxed_u64(p0); }, b0[j], status, wait_ns);
                        if (ok && b1[j] == kPending)
                            ok = spin_ready([&] { return ld_relaxed_u64(p0 + 32); }, b1[j], status, wait_ns);
                        s0 += a[j] * __longlong_as_double((long long)b0[j]);
                        s1 += a[j] * __longlong_as_double((long long)b1[j]);
                    }
                }
            }
        }
        if (!__all_sync(0xffffffffu, ok)) {
            if (lane == 0) atomicCAS(status, 0, 6);
            return;
        }
        double res0, res1;
        if (OP == OP_DIV) { res0 = (v0 - s0) / dg; res1 = (v1 - s1) / dg; }
        else if (OP == OP_MUL) { res0 = (v0 - s0) * dg; res1 = (v1 - s1) * dg; }
        else if (OP == OP_NONE) { res0 = v0 - s0; res1 = v1 - s1; }
        else { res0 = v0 / dg - s0; res1 = v1 / dg - s1; }
        unsigned long long o0 = (unsigned long long)__double_as_longlong(res0);
        unsigned long long o1 = (unsigned long long)__double_as_longlong(res1);
        if (res0 != res0) o0 = kCanonicalNaN;
        if (res1 != res1) o1 = kCanonicalNaN;
        if (h0) st_relaxed_u64(out + r * k + lane, o0);
        if (h1) st_relaxed_u64(out + r * k + lane + 32, o1);
    }
}

template <typename Low>
void* bt_sweep_kernel(int op) {
    switch (op) {
        case SWEEP_DIV: return (void*)k_bt_sweep<Low, OP_DIV>;
        case SWEEP_MUL: return (void*)k_bt_sweep<Low, OP_MUL>;
        case SWEEP_NONE: return (void*)k_bt_sweep<Low, OP_NONE>;
        default: return (void*)k_bt_sweep<Low, OP_PREDIV>;
    }
}

int bt_grid(const Handle& h, uint32_t n) {
    long want = ((long)n + kBWarps - 1) / kBWarps;
    long cap = (long)h.info.sms * 4;
    if (want < 1) want = 1;
    return (int)(want < cap ? want : cap);
}

}  // namespace

// ============================================================================
// Batch workspace
// ============================================================================
struct BatchWork {
    uint32_t n = 0, k = 0;
    DevBuf<double> B, X, R, W, D, V, Y, T;
    DevBuf<double> partial, sc;
    DevBuf<unsigned> ticket;
    DevBuf<int> active;
    double* pinned = nullptr;   // kBScalars * kBK
    int* pinned_active = nullptr;
    ~BatchWork() {
        if (pinned) cudaFreeHost(pinned);
        if (pinned_active) cudaFreeHost(pinned_active);
    }
    BSlot slot(int s) { return BSlot{partial.get(), ticket.get(), sc.get() + s * kBK}; }
};

void batch_release(BatchWork* w) { delete w; }

static BatchWork& batch_work(Handle& h, uint32_t k) {
    const uint32_t n = h.A.n;
    if (!h.batch || h.batch->n != n || h.batch->k < k) {
        h.batch.reset();
        auto* w = new BatchWork();
        h.batch = std::unique_ptr<BatchWork, void (*)(BatchWork*)>(w, batch_release);
        w->n = n;
        w->k = k;
        const size_t nk = (size_t)n * k;
        for (DevBuf<double>* b : {&w->B, &w->X, &w->R, &w->W, &w->D, &w->V, &w->Y, &w->T}) b->alloc(nk);
        w->partial.alloc((size_t)h.info.sms * 4 * 2 * kBK);
        w->sc.alloc(kBScalars * kBK);
        w->ticket.alloc(1);
        PRISM_CUDA(cudaMemsetAsync(w->ticket.get(), 0, sizeof(unsigned), h.stream));
        w->active.alloc(kBK);
        PRISM_CUDA(cudaMallocHost(&w->pinned, kBScalars * kBK * sizeof(double)));
        PRISM_CUDA(cudaMallocHost(&w->pinned_active, kBK * sizeof(int)));
    }
    return *h.batch;
}

// ============================================================================
// Launch helpers
// ============================================================================
void launch_bt_fill(cudaStream_t st, const Handle& h, uint64_t count, double* p) {
    if (!count) return;
    long want = (long)((count + kBlock - 1) / kBlock);
    long cap = (long)h.info.sms * 8;
    k_bt_fill_pending<<<(int)(want < cap ? want : cap), kBlock, 0, st>>>(count,
                                                                         reinterpret_cast<unsigned long long*>(p));
    PRISM_LAUNCHED();
}

void launch_bt_sweep(const Handle& h, cudaStream_t st, const DevSweep& s, uint32_t k, const double* in, double* out) {
    if (!s.n) return;
    if (s.layout != LAYOUT_LEVEL) throw Error(PRISM_ERR_ARG, "block sweep needs the level-order layout");
    void* fn = s.fp32 ? bt_sweep_kernel<float>(s.op) : bt_sweep_kernel<double>(s.op);
    int occ = 0;
    PRISM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kBlock, 0));
    if (occ < 1) occ = 1;
    const int per_sm = occ < h.info.sweep_blocks_per_sm ? occ : h.info.sweep_blocks_per_sm;
    long want = ((long)s.n * 32 + kBlock - 1) / kBlock;
    long cap = (long)h.info.sms * per_sm;
    int grid = (int)(want < cap ? want : cap);
    uint32_t n = s.n, kk = k;
    const uint32_t* order = s.order.get();
    const uint32_t* rowptr = s.rowptr.get();
    const uint32_t* col = s.col.get();
    const void* val = s.fp32 ? (const void*)s.val32.get() : (const void*)s.val64.get();
    const double* diag = s.diag.get();
    int* status = h.status.get();
    unsigned long long wait = kBWaitNs;
    void* args[] = {&n, &kk, &order, &rowptr, &col, &val, &diag, &in, &out, &status, &wait};
    PRISM_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kBlock), args, 0, st));
    PRISM_LAUNCHED();
}

void launch_bt_pack(cudaStream_t st, const Handle& h, uint32_t n, uint32_t k, uint64_t ld, const double* src,
                    double* dst) {
    long want = ((long)n + 31) / 32;
    long cap = (long)h.info.sms * 8;
    k_bt_pack<<<(int)(want < cap ? want : cap), kBlock, 0, st>>>(n, k, ld, src, dst);
    PRISM_LAUNCHED();
}

void launch_bt_unpack(cudaStream_t st, const Handle& h, uint32_t n, uint32_t k, uint64_t ld, const double* src,
                      double* dst) {
    long want = ((long)n + 31) / 32;
    long cap = (long)h.info.sms * 8;
    k_bt_unpack<<<(int)(want < cap ? want : cap), kBlock, 0, st>>>(n, k, ld, src, dst);
    PRISM_LAUNCHED();
}

// ============================================================================
// Triangular preconditioner on a block (level-order sweeps; the slab layout
// that the single-vector tuner may have chosen is re-uploaded in level order
// once, on first use)
// ============================================================================
void TriangularPrecond::apply_batched(cudaStream_t st, uint32_t k, const double* in, double* out) {
    const uint32_t n = h_.A.n;
    auto level_order = [&](const DevSweep& tuned, DevSweep& mine, bool lower) -> const DevSweep& {
        if (tuned.layout == LAYOUT_LEVEL) return tuned;
        if (mine.n != tuned.n) {
            if (f_->fp32) mine.upload(lower ? f_->lower32 : f_->upper32, h_.info, LAYOUT_LEVEL, h_.stream);
            else mine.upload(lower ? f_->lower64 : f_->upper64, h_.info, LAYOUT_LEVEL, h_.stream);
            refresh_level_copy(mine, lower);  // after a device refactorisation: its values
        }
        return mine;
    };
    const DevSweep& lo = level_order(lower_, lower_lv_, true);
    const DevSweep& up = level_order(upper_, upper_lv_, false);
    const size_t nk = (size_t)n * k;
    if (tmpk_.size() < nk) tmpk_.alloc(nk);
    launch_bt_fill(st, h_, nk, tmpk_.get());
    if (in != out) launch_bt_fill(st, h_, nk, out);
    launch_bt_sweep(h_, st, lo, k, in, tmpk_.get());
    if (in == out) launch_bt_fill(st, h_, nk, out);
    launch_bt_sweep(h_, st, up, k, tmpk_.get(), out);
}

// ============================================================================
// Batched apply and FCG
// ============================================================================
void batched_apply(Handle& h, uint32_t k, const double* in_d, double* out_d, uint64_t ld) {
    if (!h.P) throw Error(PRISM_ERR_NOT_READY, "no preconditioner set up");
    const uint32_t n = h.A.n;
    BatchWork& w = batch_work(h, k);
    cudaStream_t s = h.stream;
    launch_bt_pack(s, h, n, k, ld, in_d, w.R.get());
    h.P->apply_batched(s, k, w.R.get(), w.W.get());
    launch_bt_unpack(s, h, n, k, ld, w.W.get(), out_d);
    h.check_status();
}

static void spmm(Handle& h, BatchWork& w, uint32_t k, const double* X, double* Y, int ndot = 0,
                 const double* Z = nullptr, const double* Q = nullptr, int slot = 0) {
    const uint32_t n = h.A.n;
    const int g = bt_grid(h, n);
    cudaStream_t s = h.stream;
    if (ndot == 0)
        k_bt_spmm<0><<<g, kBlock, 0, s>>>(n, k, h.A.rowptr.get(), h.A.col.get(), h.A.val.get(), X, Y, Z, Q, w.slot(0));
    else if (ndot == 1)
        k_bt_spmm<1><<<g, kBlock, 0, s>>>(n, k, h.A.rowptr.get(), h.A.col.get(), h.A.val.get(), X, Y, Z, Q,
                                          w.slot(slot));
    else
        k_bt_spmm<2><<<g, kBlock, 0, s>>>(n, k, h.A.rowptr.get(), h.A.col.get(), h.A.val.get(), X, Y, Z, Q,
                                          w.slot(slot));
    PRISM_LAUNCHED();
}

void batched_fcg_solve(Handle& h, const prism_solve_opts& o, uint32_t k, const double* B_d, double* X_d, uint64_t ld,
                       prism_solve_stats* st) {
    const uint32_t n = h.A.n;
    BatchWork& w = batch_work(h, k);
    cudaStream_t s = h.stream;
    const bool flexible = o.solver == PRISM_SOLVER_FCG;
    Precond* P = h.P.get();
    double *B = w.B.get(), *X = w.X.get(), *R = w.R.get(), *W = w.W.get(), *D = w.D.get(), *V = w.V.get(),
           *Y = w.Y.get();
    double* sc = w.sc.get();
    const int g = bt_grid(h, n);
    const size_t nk = (size_t)n * k;
    uint32_t applies = 0, spmvs = 0;
    auto precond = [&]() {
        if (P) { P->apply_batched(s, k, R, W); ++applies; }
        else PRISM_CUDA(cudaMemcpyAsync(W, R, nk * sizeof(double), cudaMemcpyDeviceToDevice, s));
    };
    std::vector<int> act(k, 1);
    for (uint32_t c = 0; c < kBK; ++c) w.pinned_active[c] = c < k ? 1 : 0;
    PRISM_CUDA(cudaMemcpyAsync(w.active.get(), w.pinned_active, kBK * sizeof(int), cudaMemcpyHostToDevice, s));

    PRISM_CUDA(cudaEventRecord(h.ev0, s));
    launch_bt_pack(s, h, n, k, ld, B_d, B);
    launch_bt_pack(s, h, n, k, ld, X_d, X);
    // R = B - A X ; Σ b²
    spmm(h, w, k, X, Y);
    ++spmvs;
    k_bt_residual<<<g, kBlock, 0, s>>>(n, k, B, Y, R, w.slot(BS_BB));
    PRISM_LAUNCHED();
    precond();
    PRISM_CUDA(cudaMemcpyAsync(D, W, nk * sizeof(double), cudaMemcpyDeviceToDevice, s));
    // V = A D ; Σ v·d, Σ d·r
    spmm(h, w, k, D, V, 2, D, R, BS_DV);
    ++spmvs;
    k_bt_fcg_step<<<g, kBlock, 0, s>>>(n, k, X, R, D, V, sc + BS_DR * kBK, sc + BS_DV * kBK, w.active.get(),
                                       w.slot(BS_RR));
    PRISM_LAUNCHED();
    PRISM_CUDA(cudaMemcpyAsync(w.pinned, sc, kBScalars * kBK * sizeof(double), cudaMemcpyDeviceToHost, s));
    h.check_status();
    std::vector<double> norm_b(k), norm(k, -1.0);
    std::vector<uint32_t> m(k, o.max_iter);
    std::vector<int> conv(k, 0);
    for (uint32_t c = 0; c < k; ++c) norm_b[c] = std::sqrt(w.pinned[BS_BB * kBK + c]);
    uint32_t remaining = k;
    for (uint32_t i = 1; i < o.max_iter; ++i) {
        if (i > 1) {
            PRISM_CUDA(cudaMemcpyAsync(w.pinned + BS_RR * kBK, sc + BS_RR * kBK, kBK * sizeof(double),
                                       cudaMemcpyDeviceToHost, s));
            h.check_status();
        }
        bool changed = false;
        for (uint32_t c = 0; c < k; ++c) {
            if (!act[c]) continue;
            norm[c] = std::sqrt(w.pinned[BS_RR * kBK + c]) / norm_b[c];
            if (!std::isfinite(norm[c]))
                throw Error(PRISM_ERR_NONFINITE, "non-finite residual norm of right-hand side " + std::to_string(c) +
                                                     " in CG iteration " + std::to_string(i));
            if (norm[c] < o.tol) {
                conv[c] = 1;
                m[c] = i;
                act[c] = 0;
                --remaining;
                changed = true;
            }
        }
        if (remaining == 0) break;
        if (changed) {
            for (uint32_t c = 0; c < k; ++c) w.pinned_active[c] = act[c];
            PRISM_CUDA(cudaMemcpyAsync(w.active.get(), w.pinned_active, kBK * sizeof(int), cudaMemcpyHostToDevice, s));
        }
        if (flexible) precond();
        else PRISM_CUDA(cudaMemcpyAsync(W, R, nk * sizeof(double), cudaMemcpyDeviceToDevice, s));
        k_bt_dot<<<g, kBlock, 0, s>>>(n, k, W, V, w.slot(BS_WV));
        PRISM_LAUNCHED();
        k_bt_fcg_direction<<<g, kBlock, 0, s>>>(n, k, W, D, R, sc + BS_WV * kBK, sc + BS_DV * kBK, w.active.get(),
                                                w.slot(BS_DR2));
        PRISM_LAUNCHED();
        spmm(h, w, k, D, V, 1, D, nullptr, BS_DV);
        ++spmvs;
        k_bt_fcg_step<<<g, kBlock, 0, s>>>(n, k, X, R, D, V, sc + BS_DR2 * kBK, sc + BS_DV * kBK, w.active.get(),
                                           w.slot(BS_RR));
        PRISM_LAUNCHED();
    }
    // true FP64 residuals
    spmm(h, w, k, X, Y);
    ++spmvs;
    k_bt_residual<<<g, kBlock, 0, s>>>(n, k, B, Y, nullptr, w.slot(BS_BB));
    PRISM_LAUNCHED();
    launch_bt_unpack(s, h, n, k, ld, X, X_d);
    PRISM_CUDA(cudaEventRecord(h.ev1, s));
    PRISM_CUDA(cudaMemcpyAsync(w.pinned, sc, 2 * kBK * sizeof(double), cudaMemcpyDeviceToHost, s));
    h.check_status();
    float ms = 0.f;
    PRISM_CUDA(cudaEventElapsedTime(&ms, h.ev0, h.ev1));
    if (st) {
        for (uint32_t c = 0; c < k; ++c) {
            st[c].num_iter = (int32_t)(m[c] + 1);
            st[c].converged = conv[c];
            st[c].final_error = norm[c];
            st[c].true_rel_residual = std::sqrt(w.pinned[BS_RES * kBK + c]) / std::sqrt(w.pinned[BS_BB * kBK + c]);
            st[c].precond_applies = applies;
            st[c].spmv_count = spmvs;
            st[c].device_ms = ms;
            st[c].forward_error = -1.0;  // no reference solution for block / batch solves
            st[c].host_syncs = 0;  // not counted for block / batch solves
            st[c].graph_nodes = 0;
        }
    }
}

}  // namespace prism
