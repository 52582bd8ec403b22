// Device-resident operator, triangular preconditioners and the FCG driver.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <future>

#include "../../include/prism_solve.h"
#include "kernels.cuh"
#include "solve.cuh"
#include "stream_sweep.cuh"

namespace prism {

std::atomic<uint64_t>& launch_counter() {
    static std::atomic<uint64_t> c{0};
    return c;
}

namespace {
constexpr unsigned long long kWaitNs = 1000000000ull;  // 1 s per dependency wait
constexpr int kSpmvSubG = 8;                           // lanes per row in k_spmv_sub
constexpr int kSpmvG = 1, kSpmvU = 2;                  // k_spmv: lanes per row, rows per group and pass
// the shapes A's SpMV may take (lanes per row, rows per group and pass): one lane per row
// suits short rows such as stencils, a group of lanes per row longer ones
constexpr int kSpmvShapes = 6;
constexpr int kSpmvShapeG[kSpmvShapes] = {1, 1, 2, 4, 8, 16};
constexpr int kSpmvShapeU[kSpmvShapes] = {2, 4, 2, 1, 1, 1};
}  // namespace

int vec_grid(const Handle& h, uint32_t n) {
    long want = ((long)n + kBlock - 1) / kBlock;
    long cap = (long)h.info.sms * 4;
    if (want < 1) want = 1;
    return (int)(want < cap ? want : cap);
}

void launch_fill(cudaStream_t st, const Handle& h, uint32_t n, double* p) {
    if (!n) return;
    k_fill_pending<<<vec_grid(h, n), kBlock, 0, st>>>(n, reinterpret_cast<unsigned long long*>(p));
    PRISM_LAUNCHED();
}

static void* slab_kernel(bool fp32, int op) {
    if (fp32) {
        switch (op) {
            case SWEEP_DIV: return (void*)k_sweep_slab<float, OP_DIV>;
            case SWEEP_MUL: return (void*)k_sweep_slab<float, OP_MUL>;
            case SWEEP_NONE: return (void*)k_sweep_slab<float, OP_NONE>;
            default: return (void*)k_sweep_slab<float, OP_PREDIV>;
        }
    }
    switch (op) {
        case SWEEP_DIV: return (void*)k_sweep_slab<double, OP_DIV>;
        case SWEEP_MUL: return (void*)k_sweep_slab<double, OP_MUL>;
        case SWEEP_NONE: return (void*)k_sweep_slab<double, OP_NONE>;
        default: return (void*)k_sweep_slab<double, OP_PREDIV>;
    }
}

static constexpr int kSlabThreads = 1024;

// acc32: single-precision arithmetic (float factor values only)
static void* stream_kernel(bool fp32, int op, bool acc32) {
    if (acc32) {
        switch (op) {
            case SWEEP_DIV: return (void*)k_sweep_stream<float, OP_DIV, float>;
            case SWEEP_MUL: return (void*)k_sweep_stream<float, OP_MUL, float>;
            case SWEEP_NONE: return (void*)k_sweep_stream<float, OP_NONE, float>;
            default: return (void*)k_sweep_stream<float, OP_PREDIV, float>;
        }
    }
    if (fp32) {
        switch (op) {
            case SWEEP_DIV: return (void*)k_sweep_stream<float, OP_DIV, double>;
            case SWEEP_MUL: return (void*)k_sweep_stream<float, OP_MUL, double>;
            case SWEEP_NONE: return (void*)k_sweep_stream<float, OP_NONE, double>;
            default: return (void*)k_sweep_stream<float, OP_PREDIV, double>;
        }
    }
    switch (op) {
        case SWEEP_DIV: return (void*)k_sweep_stream<double, OP_DIV, double>;
        case SWEEP_MUL: return (void*)k_sweep_stream<double, OP_MUL, double>;
        case SWEEP_NONE: return (void*)k_sweep_stream<double, OP_NONE, double>;
        default: return (void*)k_sweep_stream<double, OP_PREDIV, double>;
    }
}

void launch_sweep_prepare(const Handle& h, cudaStream_t st, const DevSweep& s, const double* in, double* out) {
    if (!s.n) return;
    if (s.layout != LAYOUT_STREAM) {
        launch_fill(st, h, s.n, out);
        return;
    }
    if (s.paired) {
        // the prep reads other rows of `in`: when in == out, the outputs are marked afterwards
        const int mark = in != out ? 1 : 0;
        if (s.acc32)
            k_stream_prep_pair<float><<<vec_grid(h, s.n), kBlock, 0, st>>>(
                s.n, s.str_in_slot.get(), s.pair_ptr.get(), s.pair_dep.get(), s.pair_coef.get(), in,
                reinterpret_cast<float*>(s.str_blob.get()), reinterpret_cast<unsigned long long*>(out), mark);
        else
            k_stream_prep_pair<double><<<vec_grid(h, s.n), kBlock, 0, st>>>(
                s.n, s.str_in_slot.get(), s.pair_ptr.get(), s.pair_dep.get(), s.pair_coef.get(), in,
                reinterpret_cast<double*>(s.str_blob.get()), reinterpret_cast<unsigned long long*>(out), mark);
        PRISM_LAUNCHED();
        if (!mark) launch_fill(st, h, s.n, out);
        return;
    }
    if (s.acc32)
        k_stream_prep<float><<<vec_grid(h, s.n), kBlock, 0, st>>>(s.n, s.str_in_slot.get(), in,
                                                                  reinterpret_cast<float*>(s.str_blob.get()),
                                                                  reinterpret_cast<unsigned long long*>(out));
    else
        k_stream_prep<double><<<vec_grid(h, s.n), kBlock, 0, st>>>(s.n, s.str_in_slot.get(), in,
                                                                   reinterpret_cast<double*>(s.str_blob.get()),
                                                                   reinterpret_cast<unsigned long long*>(out));
    PRISM_LAUNCHED();
}

void launch_sweep_kernel(const Handle& h, cudaStream_t st, const DevSweep& s, const double* in, double* out) {
    if (!s.n) return;
    if (s.layout == LAYOUT_STREAM) {
        (void)in;
        StreamArgs a;
        a.blob = s.str_blob.get();
        a.meta = reinterpret_cast<const uint4*>(s.str_meta.get());
        a.cta_round = s.str_cta_round.get();
        a.slab_start = s.str_slab_start.get();
        a.halo_ptr = s.str_halo_ptr.get();
        a.halo_row = s.str_halo_row.get();
        a.halo_sw = s.str_halo_sw.get();
        a.n = s.n;
        a.ring_bytes = s.str_ring;
        a.meta_slots = s.str_meta_slots;
        a.slots = s.str_slots;
        a.out = out;
        a.status = h.status.get();
        a.wait_ns = kWaitNs;
        void* args[] = {&a};
        PRISM_CUDA(cudaLaunchCooperativeKernel(stream_kernel(s.fp32, s.op, s.acc32), dim3(s.str_ctas), dim3(kStrThreads), args,
                                               s.str_smem, st));
        PRISM_LAUNCHED();
        return;
    }
    if (s.num_ctas > 0) {
        void* fn = slab_kernel(s.fp32, s.op);
        uint32_t n = s.n, rpc = s.rows_per_cta, smem_rows = s.smem_rows;
        const uint32_t* cta_pos = s.cta_pos.get();
        const uint32_t* order = s.order.get();
        const uint32_t* rowptr = s.rowptr.get();
        const uint32_t* col = s.col.get();
        const void* val = s.fp32 ? (const void*)s.val32.get() : (const void*)s.val64.get();
        const double* diag = s.diag.get();
        int* status = h.status.get();
        unsigned long long wait = kWaitNs;
        void* args[] = {&n, &rpc, &smem_rows, &cta_pos, &order, &rowptr, &col, &val, &diag, &in, &out, &status, &wait};
        PRISM_CUDA(cudaLaunchCooperativeKernel(fn, dim3(s.num_ctas), dim3(kSlabThreads), args,
                                               (size_t)s.smem_rows * sizeof(double), st));
        PRISM_LAUNCHED();
        return;
    }
    long want = ((long)s.n * 32 + kBlock - 1) / kBlock;
    long cap = (long)h.info.sms * h.info.sweep_blocks_per_sm;
    int grid = (int)(want < cap ? want : cap);
    void* fn = nullptr;
    if (s.fp32) {
        switch (s.op) {
            case SWEEP_DIV: fn = (void*)k_sweep<float, OP_DIV>; break;
            case SWEEP_MUL: fn = (void*)k_sweep<float, OP_MUL>; break;
            case SWEEP_NONE: fn = (void*)k_sweep<float, OP_NONE>; break;
            default: fn = (void*)k_sweep<float, OP_PREDIV>; break;
        }
    } else {
        switch (s.op) {
            case SWEEP_DIV: fn = (void*)k_sweep<double, OP_DIV>; break;
            case SWEEP_MUL: fn = (void*)k_sweep<double, OP_MUL>; break;
            case SWEEP_NONE: fn = (void*)k_sweep<double, OP_NONE>; break;
            default: fn = (void*)k_sweep<double, OP_PREDIV>; break;
        }
    }
    uint32_t n = s.n;
    const uint32_t* order = s.order.get();
    const uint32_t* rowptr = s.rowptr.get();
    const uint32_t* col = s.col.get();
    const void* val = s.fp32 ? (const void*)s.val32.get() : (const void*)s.val64.get();
    const double* diag = s.diag.get();
    int* status = h.status.get();
    unsigned long long wait = kWaitNs;
    void* args[] = {&n, &order, &rowptr, &col, &val, &diag, &in, &out, &status, &wait};
    // Cooperative launch: all blocks co-resident, which the level-order
    // progress argument of k_sweep relies on.
    PRISM_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kBlock), args, 0, st));
    PRISM_LAUNCHED();
}

void launch_sweep(const Handle& h, cudaStream_t st, const DevSweep& s, const double* in, double* out) {
    if (s.layout == LAYOUT_STREAM) launch_sweep_prepare(h, st, s, in, out);
    launch_sweep_kernel(h, st, s, in, out);
}

void launch_spmv(const Handle& h, cudaStream_t st, uint32_t nrows, const uint32_t* rowptr, const uint32_t* col,
                 const double* val, const double* x, double* y, int sub) {
    if (!nrows) return;
    long cap = (long)h.info.sms * 8;
    ReduceSlot none{nullptr, nullptr, nullptr};
    if (sub) {
        long want = ((long)nrows * kSpmvSubG + kBlock - 1) / kBlock;
        k_spmv_sub<kSpmvSubG><<<(int)(want < cap ? want : cap), kBlock, 0, st>>>(nrows, rowptr, col, val, x, y);
    } else {
        const long rows_per_block = (long)(kBlock / 32) * (32 / kSpmvG) * kSpmvU;
        long want = ((long)nrows + rows_per_block - 1) / rows_per_block;
        k_spmv<kSpmvG, kSpmvU, 0><<<(int)(want < cap ? want : cap), kBlock, 0, st>>>(nrows, rowptr, col, val, x, y,
                                                                                   nullptr, nullptr, none);
    }
    PRISM_LAUNCHED();
}

void launch_adjoint_outer(const Handle& h, cudaStream_t st, const double* lambda, const double* x, double* grad) {
    k_adjoint_outer<<<vec_grid(h, h.A.n), kBlock, 0, st>>>(h.A.n, h.A.rowptr.get(), h.A.col.get(), lambda, x, grad);
    PRISM_LAUNCHED();
}

// ============================================================================
// Bounded-wait self test: a two-row sweep whose first position depends on the
// second one, run by a single warp.  The warp reaches position 0 first, so the
// value it waits for is never produced; the wait must run out after wait_ns,
// raise status 6 and return, leaving the context usable (checked by a normal
// sweep afterwards).
// ============================================================================
int selftest_wait_timeout(int device, unsigned long long wait_ns, int* device_status) {
    PRISM_CUDA(cudaSetDevice(device));
    cudaStream_t st;
    PRISM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    // position 0 = row 0 (depends on row 1), position 1 = row 1 (no dependency)
    const uint32_t h_order[2] = {0, 1}, h_rowptr[3] = {0, 1, 1}, h_col[1] = {1};
    const double h_val[1] = {0.5}, h_diag[2] = {1.0, 1.0}, h_in[2] = {1.0, 2.0};
    DevBuf<uint32_t> order(2), rowptr(3), col(1);
    DevBuf<double> val(1), diag(2), in(2), out(2);
    DevBuf<int> status(1);
    order.upload(h_order, 2, st); rowptr.upload(h_rowptr, 3, st); col.upload(h_col, 1, st);
    val.upload(h_val, 1, st); diag.upload(h_diag, 2, st); in.upload(h_in, 2, st);
    PRISM_CUDA(cudaMemsetAsync(status.get(), 0, sizeof(int), st));
    k_fill_pending<<<1, 32, 0, st>>>(2, reinterpret_cast<unsigned long long*>(out.get()));
    PRISM_LAUNCHED();
    k_sweep<double, OP_NONE><<<1, 32, 0, st>>>(2, order.get(), rowptr.get(), col.get(), val.get(), diag.get(),
                                               in.get(), out.get(), status.get(), wait_ns);
    PRISM_LAUNCHED();
    int s = -1;
    PRISM_CUDA(cudaMemcpyAsync(&s, status.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    PRISM_CUDA(cudaStreamSynchronize(st));
    *device_status = s;
    // the context is still usable: the same rows in a valid order solve normally
    const uint32_t g_order[2] = {1, 0}, g_rowptr[3] = {0, 0, 1};
    order.upload(g_order, 2, st); rowptr.upload(g_rowptr, 3, st);
    PRISM_CUDA(cudaMemsetAsync(status.get(), 0, sizeof(int), st));
    k_fill_pending<<<1, 32, 0, st>>>(2, reinterpret_cast<unsigned long long*>(out.get()));
    PRISM_LAUNCHED();
    k_sweep<double, OP_NONE><<<1, 32, 0, st>>>(2, order.get(), rowptr.get(), col.get(), val.get(), diag.get(),
                                               in.get(), out.get(), status.get(), wait_ns);
    PRISM_LAUNCHED();
    double h_out[2] = {0, 0};
    int s2 = -1;
    PRISM_CUDA(cudaMemcpyAsync(h_out, out.get(), sizeof(h_out), cudaMemcpyDeviceToHost, st));
    PRISM_CUDA(cudaMemcpyAsync(&s2, status.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    PRISM_CUDA(cudaStreamSynchronize(st));
    PRISM_CUDA(cudaStreamDestroy(st));
    // row 1 = 2, row 0 = 1 - 0.5 * 2 = 0
    if (s2 != 0 || h_out[0] != 0.0 || h_out[1] != 2.0)
        throw Error(PRISM_ERR_CUDA, "context unusable after a timed-out wait");
    return 0;
}

// ============================================================================
// Handle
// ============================================================================
void init_device_info(DeviceInfo& info, int device) {
    info.device = device;
    PRISM_CUDA(cudaDeviceGetAttribute(&info.sms, cudaDevAttrMultiProcessorCount, device));
    int occ = 0, occ2 = 0;
    PRISM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_sweep<double, OP_DIV>, kBlock, 0));
    PRISM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, k_sweep<float, OP_DIV>, kBlock, 0));
    occ = occ < occ2 ? occ : occ2;
    // a fraction of the co-resident capacity: enough warps to cover a wavefront,
    // few enough pollers to leave L2 bandwidth to the producers
    int want = 4;
    if (const char* e = std::getenv("PRISM_SWEEP_BLOCKS_PER_SM")) want = std::atoi(e);
    if (want < 1) want = 1;
    info.sweep_blocks_per_sm = occ < want ? (occ > 0 ? occ : 1) : want;
    PRISM_CUDA(cudaDeviceGetAttribute(&info.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    if (const char* e = std::getenv("PRISM_SWEEP_KERNEL")) {
        const std::string k(e);
        info.sweep_kernel = k == "global" ? 1 : (k == "slab" ? 2 : (k == "stream" ? 3 : 0));
    }
    if (const char* e = std::getenv("PRISM_SLAB_MIN_ROWS")) info.slab_min_rows = (uint32_t)std::atoi(e);
    if (const char* e = std::getenv("PRISM_SLAB_MAX_ROWS")) info.slab_max_rows = (uint32_t)std::atoi(e);
    if (info.slab_min_rows < 32) info.slab_min_rows = 32;
    // the slab kernel runs one 1024-thread CTA per SM with up to the whole opt-in shared memory
    if (const char* e = std::getenv("PRISM_STREAM_MIN_ROWS")) info.stream_min_rows = (uint32_t)std::atoi(e);
    if (const char* e = std::getenv("PRISM_STREAM_PAIR")) {  // 0 never, 1 the tuner decides, 2 always
        const int v = std::atoi(e);
        info.stream_pair = v < 0 ? 0 : (v > 2 ? 2 : v);
    }
    if (info.stream_min_rows < 32) info.stream_min_rows = 32;
    for (bool f32 : {false, true})
        for (int op = 0; op < 4; ++op) {
            PRISM_CUDA(cudaFuncSetAttribute(slab_kernel(f32, op), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            info.max_smem_optin));
            PRISM_CUDA(cudaFuncSetAttribute(stream_kernel(f32, op, false), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            info.max_smem_optin));
            if (f32)
                PRISM_CUDA(cudaFuncSetAttribute(stream_kernel(true, op, true),
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, info.max_smem_optin));
        }
}

Handle::~Handle() {
    P.reset();
    if (pinned) cudaFreeHost(pinned);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (own_stream && stream) cudaStreamDestroy(stream);
}

void Handle::ensure_workspace() {
    const uint32_t n = A.n;
    if (r.size() < n) {
        r.alloc(n); w.alloc(n); d.alloc(n); v.alloc(n); y.alloc(n);
    }
}

namespace {
template <int G, int U>
void spmv_shape_launch(const Handle& h, const double* x, double* yout, int ndot, const double* z, const double* q,
                       ReduceSlot slot) {
    const uint32_t n = h.A.n;
    const long rows_per_block = (long)(kBlock / 32) * (32 / G) * U;
    long want = ((long)n + rows_per_block - 1) / rows_per_block;
    long cap = (long)h.info.sms * 8;
    int grid = (int)(want < cap ? want : cap);
    if (grid > Reducer::kMaxGrid) grid = Reducer::kMaxGrid;
    const uint32_t* rp = h.A.rowptr.get();
    const uint32_t* ci = h.A.col.get();
    const double* va = h.A.val.get();
    if (ndot == 0) k_spmv<G, U, 0><<<grid, kBlock, 0, h.stream>>>(n, rp, ci, va, x, yout, z, q, slot);
    else if (ndot == 1) k_spmv<G, U, 1><<<grid, kBlock, 0, h.stream>>>(n, rp, ci, va, x, yout, z, q, slot);
    else k_spmv<G, U, 2><<<grid, kBlock, 0, h.stream>>>(n, rp, ci, va, x, yout, z, q, slot);
    PRISM_LAUNCHED();
}
}  // namespace

void Handle::spmv(const double* x, double* yout, int ndot, const double* z, const double* q, int scalar) {
    if (!A.n) return;
    const ReduceSlot slot = red.slot(scalar);
    switch (spmv_shape) {
        case 1: spmv_shape_launch<kSpmvShapeG[1], kSpmvShapeU[1]>(*this, x, yout, ndot, z, q, slot); break;
        case 2: spmv_shape_launch<kSpmvShapeG[2], kSpmvShapeU[2]>(*this, x, yout, ndot, z, q, slot); break;
        case 3: spmv_shape_launch<kSpmvShapeG[3], kSpmvShapeU[3]>(*this, x, yout, ndot, z, q, slot); break;
        case 4: spmv_shape_launch<kSpmvShapeG[4], kSpmvShapeU[4]>(*this, x, yout, ndot, z, q, slot); break;
        case 5: spmv_shape_launch<kSpmvShapeG[5], kSpmvShapeU[5]>(*this, x, yout, ndot, z, q, slot); break;
        default: spmv_shape_launch<kSpmvShapeG[0], kSpmvShapeU[0]>(*this, x, yout, ndot, z, q, slot); break;
    }
}

void Handle::spmv_shape_of(int* lanes_per_row, int* rows_per_pass) const {
    const int s = spmv_shape >= 0 && spmv_shape < kSpmvShapes ? spmv_shape : 0;
    if (lanes_per_row) *lanes_per_row = kSpmvShapeG[s];
    if (rows_per_pass) *rows_per_pass = kSpmvShapeU[s];
}

// Times A x with each shape (one warm-up and three timed launches, the plain product
// without fused dot products) and keeps the fastest; PRISM_SPMV_SHAPE (0..5) forces one.
void Handle::tune_spmv() {
    spmv_shape = 0;
    if (const char* e = std::getenv("PRISM_SPMV_SHAPE")) {
        const int v = std::atoi(e);
        spmv_shape = v >= 0 && v < kSpmvShapes ? v : 0;
        return;
    }
    if (A.n == 0) return;
    DevBuf<double> x(A.n), y(A.n);
    std::vector<double> ones(A.n, 1.0);
    x.upload(ones.data(), A.n, stream);
    float best = 0.f;
    int best_s = 0;
    for (int s = 0; s < kSpmvShapes; ++s) {
        spmv_shape = s;
        spmv(x.get(), y.get());
        PRISM_CUDA(cudaEventRecord(ev0, stream));
        for (int it = 0; it < 3; ++it) spmv(x.get(), y.get());
        PRISM_CUDA(cudaEventRecord(ev1, stream));
        PRISM_CUDA(cudaEventSynchronize(ev1));
        float ms = 0.f;
        PRISM_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        if (s == 0 || ms < best) {
            best = ms;
            best_s = s;
        }
    }
    spmv_shape = best_s;
}

void Handle::check_status() {
    int s = 0;
    PRISM_CUDA(cudaMemcpyAsync(&s, status.get(), sizeof(int), cudaMemcpyDeviceToHost, stream));
    PRISM_CUDA(cudaStreamSynchronize(stream));
    if (s != 0) {
        PRISM_CUDA(cudaMemsetAsync(status.get(), 0, sizeof(int), stream));
        throw Error(s, "device-side wait ran out of time in a triangular sweep (status " + std::to_string(s) + ")");
    }
}

// ============================================================================
// Sweeps and triangular preconditioners
// ============================================================================
void DevSweep::release() {
    order.release(); rowptr.release(); col.release(); cta_pos.release();
    val64.release(); diag.release(); val32.release();
    str_blob.release(); str_meta.release(); str_cta_round.release(); str_slab_start.release(); str_in_slot.release();
    str_halo_ptr.release(); str_halo_row.release(); str_halo_sw.release();
    num_ctas = rows_per_cta = smem_rows = 0;
    str_ctas = str_ring = str_meta_slots = str_slots = str_rounds = str_smem = 0;
    str_nnz = 0;
    str_round_cap = 0;
    pair_ptr.release(); pair_dep.release(); pair_coef.release();
    paired = false;
    n = num_levels = 0;  // empty: nothing launches on a released sweep
}

template <typename Low>
StreamPlan plan_stream(const Sweep<Low>& sweep, const DeviceInfo& info, bool acc32, bool pair) {
    // One persistent CTA per SM (fewer for small sweeps); shared memory holds the
    // round table, the value slots and, in what is left, the ring the round
    // records stream through.
    StreamPlan P;
    const uint32_t nn = sweep.n;
    if (nn == 0) return P;
    Sweep<Low> ps;
    if (pair) pair_sweep<Low>(sweep, ps, P.pm);
    const Sweep<Low>& s0 = pair ? ps : sweep;
    const uint32_t ctas_req = stream_slab_count(nn, (uint32_t)info.sms, info.stream_min_rows);
    const std::vector<uint32_t> start = slab_ranges<Low>(s0, ctas_req);
    const uint64_t smem = (uint64_t)info.max_smem_optin;
    StreamLayout& L = P.L;
    const bool a32 = acc32 && std::is_same<Low, float>::value;
    const uint32_t slot_bytes = a32 ? 4 : 8;  // one value slot
    const uint32_t vb = (uint32_t)sizeof(Low);
    const uint64_t base_smem = stream_smem(0, 0, slot_bytes, vb, 0).total;  // everything but table and slots
    if (smem <= base_smem) return P;
    const uint32_t slot_cap = (uint32_t)std::min<uint64_t>(kNoSlot, (smem - base_smem) / slot_bytes / 2);
    // While round i is computed the row threads hold rounds i and i + 1 and wait for
    // round i + 2's record: two live records and room for a third, which a circular ring
    // of four of the largest records always has in one piece.  Where a round's record
    // is too large for that (rows of many entries), the rounds are cut shorter.
    uint32_t cap = 0;
    uint64_t fixed = 0;
    bool fits = false;
    for (int attempt = 0; attempt < 4 && !fits; ++attempt) {
        L = StreamLayout();
        if (!stream_layout<Low>(s0, start, slot_cap, slot_bytes, L, nullptr, nullptr, nullptr, cap)) return P;
        if (L.max_rounds_per_cta > smem / 16 || L.slots > kNoSlot) return P;
        fixed = stream_smem(L.max_rounds_per_cta, L.slots, slot_bytes, vb, 0).total;
        fits = fixed + 4ull * L.max_round_bytes <= smem;
        if (!fits) {
            if (fixed + 4096 >= smem) return P;
            const uint64_t room = (smem - fixed) / 4 * 7 / 8 >> attempt;  // margin for rounds and slots
            cap = (uint32_t)std::max<uint64_t>(room & ~15ull, 1024);
        }
    }
    if (!fits) return P;
    P.ok = true;
    P.paired = pair;
    P.fp32 = std::is_same<Low, float>::value;
    P.a32 = a32;
    P.n = s0.n;
    P.num_levels = s0.num_levels;
    P.op = s0.op;
    P.ctas = (uint32_t)start.size() - 1;
    P.ctas_req = ctas_req;
    P.slot_bytes = slot_bytes;
    P.cap = cap;
    P.ring = (uint32_t)((smem - fixed) & ~15ull);
    P.smem = stream_smem(L.max_rounds_per_cta, L.slots, slot_bytes, vb, P.ring).total;  // <= smem
    P.nnz = s0.val.size();
    return P;
}
template StreamPlan plan_stream<double>(const Sweep<double>&, const DeviceInfo&, bool, bool);
template StreamPlan plan_stream<float>(const Sweep<float>&, const DeviceInfo&, bool, bool);

void DevSweep::commit_stream(StreamPlan&& P, cudaStream_t st) {
    const StreamLayout& L = P.L;
    release();
    n = P.n;
    num_levels = P.num_levels;
    op = P.op;
    fp32 = P.fp32;
    acc32 = P.a32;
    layout = LAYOUT_STREAM;
    str_ctas = P.ctas;
    str_ctas_req = P.ctas_req;
    str_slot_bytes = P.slot_bytes;
    str_round_cap = P.cap;
    str_ring = P.ring;
    str_meta_slots = L.max_rounds_per_cta;
    str_slots = L.slots;
    str_rounds = L.num_rounds;
    str_smem = P.smem;
    str_nnz = P.nnz;
    str_blob.upload(L.blob.data(), L.blob.size(), st);
    str_meta.upload(L.meta.data(), L.meta.size(), st);
    str_cta_round.upload(L.cta_round.data(), L.cta_round.size(), st);
    str_slab_start.upload(L.slab_start.data(), L.slab_start.size(), st);
    str_in_slot.upload(L.in_slot.data(), L.in_slot.size(), st);
    str_halo_ptr.upload(L.halo_ptr.data(), L.halo_ptr.size(), st);
    str_halo_row.upload(L.halo_row.data(), L.halo_row.size(), st);
    str_halo_sw.upload(L.halo_sw.data(), L.halo_sw.size(), st);
    if (str_halo_row.size() == 0) str_halo_row.alloc(1);  // valid pointers for the kernel
    if (str_halo_sw.size() == 0) str_halo_sw.alloc(1);
    if (P.paired) {
        paired = true;
        pair_ptr.upload(P.pm.ptr.data(), P.pm.ptr.size(), st);
        pair_dep.upload(P.pm.dep.data(), P.pm.dep.size(), st);
        pair_coef.upload(P.pm.coef.data(), P.pm.coef.size(), st);
        if (pair_dep.size() == 0) pair_dep.alloc(1);  // valid pointers for the prep
        if (pair_coef.size() == 0) pair_coef.alloc(1);
    }
    PRISM_CUDA(cudaStreamSynchronize(st));
}

template <typename Low>
bool DevSweep::upload(const Sweep<Low>& sweep, const DeviceInfo& info, int lay, cudaStream_t st, bool pair) {
    if (lay == LAYOUT_STREAM) {
        StreamPlan P = plan_stream<Low>(sweep, info, acc32, pair);
        if (!P.ok) return false;
        commit_stream(std::move(P), st);
        return true;
    }
    const Sweep<Low>& s0 = sweep;
    release();
    layout = lay;
    n = s0.n;
    num_levels = s0.num_levels;
    op = s0.op;
    fp32 = std::is_same<Low, float>::value;
    const Sweep<Low>* s = &s0;
    Sweep<Low> slab;
    std::vector<uint32_t> cpos;
    if (lay == LAYOUT_SLAB && n > 0) {
        // As many rows per slab as shared memory holds: the dependencies of a
        // row reach back about one grid plane, so large slabs keep most of them
        // (and the critical path through them) inside one CTA, where a
        // dependency costs a shared-memory poll instead of an L2 round trip.
        const uint32_t cap = (uint32_t)(info.max_smem_optin / sizeof(double));
        uint32_t per = std::max<uint32_t>(std::min<uint32_t>(cap, info.slab_max_rows), info.slab_min_rows);
        uint32_t ctas = (n + per - 1) / per;
        if (ctas > (uint32_t)info.sms) ctas = (uint32_t)info.sms;
        if (ctas < 1) ctas = 1;
        rows_per_cta = (n + ctas - 1) / ctas;
        num_ctas = (n + rows_per_cta - 1) / rows_per_cta;
        smem_rows = std::min<uint32_t>(rows_per_cta, (uint32_t)(info.max_smem_optin / sizeof(double)));
        slab_layout<Low>(s0, num_ctas, rows_per_cta, cpos, slab);
        s = &slab;
        cta_pos.upload(cpos.data(), cpos.size(), st);
    } else {
        layout = LAYOUT_LEVEL;
    }
    order.upload(s->order.data(), s->order.size(), st);
    rowptr.upload(s->rowptr.data(), s->rowptr.size(), st);
    col.upload(s->col.data(), s->col.size(), st);
    diag.upload(s->diag.data(), s->diag.size(), st);
    if (fp32) val32.upload(reinterpret_cast<const float*>(s->val.data()), s->val.size(), st);
    else val64.upload(reinterpret_cast<const double*>(s->val.data()), s->val.size(), st);
    // keep at least one element so kernels always get valid pointers
    if (col.size() == 0) col.alloc(1);
    if (fp32 && val32.size() == 0) val32.alloc(1);
    if (!fp32 && val64.size() == 0) val64.alloc(1);
    PRISM_CUDA(cudaStreamSynchronize(st));
    return true;
}

uint32_t stream_slab_count(uint32_t n, uint32_t num_ctas, uint32_t min_rows) {
    if (min_rows < 1) min_rows = 1;
    uint32_t c = std::min<uint32_t>(num_ctas, (n + min_rows - 1) / min_rows);
    return c < 1 ? 1 : c;
}

template <typename Low>
bool DevSweep::stream_order(const Sweep<Low>& sweep, StreamOrder& o) const {
    if (layout != LAYOUT_STREAM || sweep.n != n) return false;
    Sweep<Low> ps;
    PairMap pm;
    if (paired) pair_sweep<Low>(sweep, ps, pm);
    const Sweep<Low>& s = paired ? ps : sweep;
    StreamLayout L;
    std::string why;
    if (!stream_layout<Low>(s, slab_ranges<Low>(s, str_ctas_req), kNoSlot, str_slot_bytes, L, &why, &o, nullptr,
                            str_round_cap))
        throw Error(PRISM_ERR_CUDA, "streamed layout could not be rebuilt: " + why);
    if (paired) {
        o.mptr = std::move(pm.ptr);
        o.mdep = std::move(pm.dep);
        o.mcoef = std::move(pm.coef);
    }
    return true;
}
template bool DevSweep::stream_order<double>(const Sweep<double>&, StreamOrder&) const;
template bool DevSweep::stream_order<float>(const Sweep<float>&, StreamOrder&) const;

template <typename Low>
void stream_sweep_run(int device, const Sweep<Low>& s, bool acc32, uint32_t num_ctas, const double* in,
                      double* out) {
    Handle h;
    init_device_info(h.info, device);
    h.info.sms = (int)std::min<uint32_t>(num_ctas, (uint32_t)h.info.sms);
    h.info.stream_min_rows = 32;
    PRISM_CUDA(cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking));
    h.own_stream = true;
    h.status.alloc(1);
    PRISM_CUDA(cudaMemsetAsync(h.status.get(), 0, sizeof(int), h.stream));
    DevSweep d;
    d.acc32 = acc32 && std::is_same<Low, float>::value;
    if (!d.upload(s, h.info, LAYOUT_STREAM, h.stream))
        throw Error(PRISM_ERR_UNSUPPORTED, "the sweep does not fit the streamed layout");
    DevBuf<double> din(s.n), dout(s.n);
    din.upload(in, s.n, h.stream);
    launch_sweep(h, h.stream, d, din.get(), dout.get());
    PRISM_CUDA(cudaMemcpyAsync(out, dout.get(), s.n * sizeof(double), cudaMemcpyDeviceToHost, h.stream));
    h.check_status();
}
template void stream_sweep_run<double>(int, const Sweep<double>&, bool, uint32_t, const double*, double*);
template void stream_sweep_run<float>(int, const Sweep<float>&, bool, uint32_t, const double*, double*);

// Sweep-kernel autotuner: uploads the sweep in each device layout in turn
// (level order for k_sweep, slabs for k_sweep_slab, streamed rounds for
// k_sweep_stream), times a few launches of each, output marking included, on
// a fixed right-hand side with CUDA events, and keeps the fastest.  Which
// kernel wins depends on how many rows a wavefront holds and how far
// dependencies reach.
template <typename Low>
void tune_sweep(Handle& h, DevSweep& d, const Sweep<Low>& s, bool acc32, bool pair) {
    const int mode = h.info.sweep_kernel;
    d.acc32 = acc32 && std::is_same<Low, float>::value;
    // Pairing keeps the arithmetic's precision class only where the derived coefficients are
    // stored in the arithmetic's own type: double values (FP64) or float values with float
    // arithmetic; float values with double arithmetic (<float,double>) stay unpaired.
    const bool pp = pair && h.info.stream_pair != 0 && (d.acc32 || std::is_same<Low, double>::value);
    if (s.n == 0) {
        d.upload(s, h.info, LAYOUT_LEVEL, h.stream);
        return;
    }
    // candidates: {layout, paired}.  Single-precision arithmetic: only the streamed kernel
    // has it (the other layouts, where the streamed one does not fit, compute in double).
    std::vector<std::pair<int, bool>> cand;
    if (pp && h.info.stream_pair == 2) {  // paired where it fits
        cand.push_back({LAYOUT_STREAM, true});
    } else if (d.acc32 || mode == 3) {
        cand.push_back({LAYOUT_STREAM, false});
        if (pp) cand.push_back({LAYOUT_STREAM, true});
    } else if (mode != 0) {
        cand.push_back({mode == 2 ? LAYOUT_SLAB : LAYOUT_LEVEL, false});
    } else {
        cand = {{LAYOUT_LEVEL, false}, {LAYOUT_SLAB, false}, {LAYOUT_STREAM, false}};
        if (pp) cand.push_back({LAYOUT_STREAM, true});
    }
    if (cand.size() == 1) {
        if (!d.upload(s, h.info, cand[0].first, h.stream, cand[0].second)) d.upload(s, h.info, LAYOUT_LEVEL, h.stream);
        return;
    }
    DevBuf<double> in(s.n), out(s.n);
    std::vector<double> rhs(s.n);
    for (uint32_t i = 0; i < s.n; ++i) rhs[i] = 1.0 + (double)(i % 7) * 0.125;
    in.upload(rhs.data(), s.n, h.stream);
    cudaEvent_t e0, e1;
    PRISM_CUDA(cudaEventCreate(&e0));
    PRISM_CUDA(cudaEventCreate(&e1));
    float best = 0.f;
    int best_c = -1;
    // the streamed candidates' host layouts are built concurrently
    std::vector<std::future<StreamPlan>> plans(cand.size());
    for (int c = 0; c < (int)cand.size(); ++c)
        if (cand[c].first == LAYOUT_STREAM) {
            const bool pc = cand[c].second, a32 = d.acc32;
            plans[c] = std::async(std::launch::async, [&s, &h, a32, pc] { return plan_stream<Low>(s, h.info, a32, pc); });
        }
    DevSweep kept;  // the fastest candidate so far, kept uploaded
    for (int c = 0; c < (int)cand.size(); ++c) {
        DevSweep t;
        t.acc32 = d.acc32;
        if (cand[c].first == LAYOUT_STREAM) {
            StreamPlan P = plans[c].get();
            if (!P.ok) continue;
            t.commit_stream(std::move(P), h.stream);
        } else if (!t.upload(s, h.info, cand[c].first, h.stream, cand[c].second)) {
            continue;
        }
        float tot = 0.f;
        for (int it = 0; it < 4; ++it) {
            PRISM_CUDA(cudaEventRecord(e0, h.stream));
            launch_sweep_prepare(h, h.stream, t, in.get(), out.get());
            launch_sweep_kernel(h, h.stream, t, in.get(), out.get());
            PRISM_CUDA(cudaEventRecord(e1, h.stream));
            PRISM_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            PRISM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (it > 0) tot += ms;  // first launch is a warm-up
        }
        h.check_status();
        if (best_c < 0 || tot < best) {
            best = tot;
            best_c = c;
            kept = std::move(t);
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best_c < 0) {  // nothing fitted (streamed layouts only): level order, double arithmetic
        d.upload(s, h.info, LAYOUT_LEVEL, h.stream);
        return;
    }
    d = std::move(kept);
    d.tuned_ms = best / 3.f;
}
template void tune_sweep<double>(Handle&, DevSweep&, const Sweep<double>&, bool, bool);
template void tune_sweep<float>(Handle&, DevSweep&, const Sweep<float>&, bool, bool);

namespace {
std::atomic<uint64_t> g_precond_uid{0};
}
Precond::Precond() : uid(++g_precond_uid) {}

TriangularPrecond::TriangularPrecond(Handle& h, std::shared_ptr<const HostFactor> f) : h_(h), f_(std::move(f)) {
    // the streamed kernel may run the sweeps paired (refactor() tunes them again unpaired)
    if (f_->fp32) {
        tune_sweep(h_, lower_, f_->lower32, f_->apply32, true);
        tune_sweep(h_, upper_, f_->upper32, f_->apply32, true);
    } else {
        tune_sweep(h_, lower_, f_->lower64, false, true);
        tune_sweep(h_, upper_, f_->upper64, false, true);
    }
    tmp_.alloc(h_.A.n);  // here rather than at the first apply, which may be under graph capture
}

void TriangularPrecond::apply(cudaStream_t st, const double* in, double* out) {
    const uint32_t n = h_.A.n;
    if (tmp_.size() < n) tmp_.alloc(n);
    if (!lower_.self_filling()) launch_fill(st, h_, n, tmp_.get());
    if (in != out && !upper_.self_filling()) launch_fill(st, h_, n, out);
    launch_sweep(h_, st, lower_, in, tmp_.get());
    if (in == out && !upper_.self_filling()) launch_fill(st, h_, n, out);
    launch_sweep(h_, st, upper_, tmp_.get(), out);
}

bool TriangularPrecond::run_sweep(cudaStream_t st, int sweep, const double* in, double* out, int prepare) {
    const DevSweep& s = sweep == 0 ? lower_ : upper_;
    if (prepare != 0) launch_sweep_prepare(h_, st, s, in, out);
    if (prepare != 2) launch_sweep_kernel(h_, st, s, in, out);
    return true;
}

bool TriangularPrecond::sweep_info(int sweep, uint32_t* n, uint64_t* nnz, uint32_t* vbytes, uint32_t* levels,
                                   uint32_t* kernel) const {
    const DevSweep& s = sweep == 0 ? lower_ : upper_;
    if (kernel) *kernel = s.layout == LAYOUT_STREAM ? 3 : (s.layout == LAYOUT_SLAB ? 2 : 1);
    if (n) *n = s.n;
    if (nnz) *nnz = s.entries();
    if (vbytes) *vbytes = s.fp32 ? 4 : 8;
    if (levels) *levels = s.num_levels;
    return true;
}

bool TriangularPrecond::sweep_order(int sweep, StreamOrder& o) const {
    const DevSweep& s = sweep == 0 ? lower_ : upper_;
    if (f_->fp32) return s.stream_order<float>(sweep == 0 ? f_->lower32 : f_->upper32, o);
    return s.stream_order<double>(sweep == 0 ? f_->lower64 : f_->upper64, o);
}

int export_host_factor(const HostFactor& f, int which, uint32_t* n, uint64_t* nnz, uint32_t* rowptr, uint32_t* col,
                       double* val, double* diag) {
    if (which != 0 && !(which == 1 && f.kind == PRISM_PRECOND_ILUT)) return PRISM_ERR_ARG;
    const CsrT<double>& m = which == 0 ? f.f0 : f.f1;
    if (n) *n = m.n;
    if (nnz) *nnz = m.nnz();
    if (rowptr) std::memcpy(rowptr, m.rowptr.data(), m.rowptr.size() * sizeof(uint32_t));
    if (col) std::memcpy(col, m.col.data(), m.col.size() * sizeof(uint32_t));
    if (val) std::memcpy(val, m.val.data(), m.val.size() * sizeof(double));
    if (diag && !f.diag.empty()) std::memcpy(diag, f.diag.data(), f.diag.size() * sizeof(double));
    return 0;
}

int TriangularPrecond::export_factor(int which, uint32_t* n, uint64_t* nnz, uint32_t* rowptr, uint32_t* col,
                                     double* val, double* diag) const {
    if (rf_) return export_refactored(which, n, nnz, rowptr, col, val, diag);
    return export_host_factor(*f_, which, n, nnz, rowptr, col, val, diag);
}

// ============================================================================
// Flexible / normal preconditioned CG  (CG<double>::solve, CG.cpp:34-83)
//
// Same recurrence, same stopping test on the recursive residual, same
// iteration count convention (numIter = m + 1).  The reference recomputes
// v = A d at the top of every iteration (CG.cpp:68) although d has not
// changed since v = A d at the end of the previous one (CG.cpp:75); the
// SpMV and the d.v reduction are deterministic here, so that product and its
// d.v are reused instead of recomputed: one SpMV per iteration, not two.
// ============================================================================
void fcg_solve(Handle& h, const prism_solve_opts& o, const double* b, double* x, prism_solve_stats* st) {
    const uint32_t n = h.A.n;
    h.ensure_workspace();
    cudaStream_t s = h.stream;
    const bool flexible = o.solver == PRISM_SOLVER_FCG;
    Precond* P = h.P.get();
    double* r = h.r.get();
    double* w = h.w.get();
    double* d = h.d.get();
    double* v = h.v.get();
    double* y = h.y.get();
    double* sc = h.red.scalars.get();
    const int vg = vec_grid(h, n);
    uint32_t applies = 0, spmvs = 0, syncs = 0;

    PRISM_CUDA(cudaEventRecord(h.ev0, s));
    // r = b - A x ; Σ b²
    h.spmv(x, y);
    ++spmvs;
    k_residual<<<vg, kBlock, 0, s>>>(n, b, y, r, h.red.slot(SC_BB));
    PRISM_LAUNCHED();
    // w = M^{-1} r ; d = w
    if (P) { P->apply(s, r, w); ++applies; }
    else PRISM_CUDA(cudaMemcpyAsync(w, r, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    PRISM_CUDA(cudaMemcpyAsync(d, w, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    // v = A d ; Σ v·d , Σ d·r
    h.spmv(d, v, 2, d, r, SC_DV);
    ++spmvs;
    // x += a d ; r -= a v ; Σ r²
    k_fcg_step<<<vg, kBlock, 0, s>>>(n, x, r, d, v, sc + SC_DR, sc + SC_DV, h.red.slot(SC_RR));
    PRISM_LAUNCHED();

    PRISM_CUDA(cudaMemcpyAsync(h.pinned, sc, kNumScalars * sizeof(double), cudaMemcpyDeviceToHost, s));
    h.check_status();
    ++syncs;
    const double norm_b = std::sqrt(h.pinned[SC_BB]);
    uint32_t m = o.max_iter;
    double norm = -1.0;
    bool converged = false;
    for (uint32_t i = 1; i < o.max_iter; ++i) {
        if (i > 1) {
            PRISM_CUDA(cudaMemcpyAsync(h.pinned + SC_RR, sc + SC_RR, sizeof(double), cudaMemcpyDeviceToHost, s));
            h.check_status();
            ++syncs;
        }
        norm = std::sqrt(h.pinned[SC_RR]) / norm_b;
        if (!std::isfinite(norm)) throw Error(PRISM_ERR_NONFINITE, "non-finite residual norm in CG iteration " + std::to_string(i));
        if (norm < o.tol) {
            converged = true;
            m = i;
            break;
        }
        if (flexible && P) { P->apply(s, r, w); ++applies; }
        else PRISM_CUDA(cudaMemcpyAsync(w, r, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        // v still holds A d and sc[DV] its d.v: c = (w.v)/(d.v); d = w - c d; Σ d·r
        k_dot<<<vg, kBlock, 0, s>>>(n, w, v, h.red.slot(SC_WV));
        PRISM_LAUNCHED();
        k_fcg_direction<<<vg, kBlock, 0, s>>>(n, w, d, r, sc + SC_WV, sc + SC_DV, h.red.slot(SC_DR2));
        PRISM_LAUNCHED();
        // v = A d ; Σ v·d
        h.spmv(d, v, 1, d, nullptr, SC_DV);
        ++spmvs;
        k_fcg_step<<<vg, kBlock, 0, s>>>(n, x, r, d, v, sc + SC_DR2, sc + SC_DV, h.red.slot(SC_RR));
        PRISM_LAUNCHED();
    }
    // true FP64 residual
    h.spmv(x, y);
    ++spmvs;
    k_residual<<<vg, kBlock, 0, s>>>(n, b, y, nullptr, h.red.slot(SC_BB));
    PRISM_LAUNCHED();
    PRISM_CUDA(cudaEventRecord(h.ev1, s));
    PRISM_CUDA(cudaMemcpyAsync(h.pinned, sc, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    h.check_status();
    ++syncs;
    float ms = 0.f;
    PRISM_CUDA(cudaEventElapsedTime(&ms, h.ev0, h.ev1));
    if (st) {
        st->num_iter = (int32_t)(m + 1);
        st->converged = converged;
        st->final_error = norm;
        st->true_rel_residual = std::sqrt(h.pinned[SC_RES]) / std::sqrt(h.pinned[SC_BB]);
        st->precond_applies = applies;
        st->spmv_count = spmvs;
        st->device_ms = ms;
        st->host_syncs = syncs;
        st->graph_nodes = 0;
    }
}

double forward_error(Handle& h, const double* x, const double* xref) {
    const uint32_t n = h.A.n;
    if (!n) return 0.0;
    // { Σ xref_i^2, Σ (xref_i - x_i)^2 } into the two scratch scalars
    k_residual<<<vec_grid(h, n), kBlock, 0, h.stream>>>(n, xref, x, nullptr, h.red.slot(SC_TMP));
    PRISM_LAUNCHED();
    double v[2] = {0.0, 0.0};
    PRISM_CUDA(cudaMemcpyAsync(v, h.red.scalars.get() + SC_TMP, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                               h.stream));
    PRISM_CUDA(cudaStreamSynchronize(h.stream));
    return v[0] > 0.0 ? std::sqrt(v[1]) / std::sqrt(v[0]) : std::sqrt(v[1]);
}

}  // namespace prism
