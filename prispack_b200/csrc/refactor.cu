// Device numeric refactorisation of an IC / ILDLT factor on its own pattern.
//
// The host factorisation (IncompleteCholesky::setup, IncompleteCholesky.cpp:
// 96-246; IncompleteLDLT::setup, IncompleteLDLT.cpp:39-186) is left-looking:
// column j starts from the matrix entries of row j on or below the diagonal,
// subtracts L_ik * L_jk (* D_k) for every finished column k with an entry in
// row j, in the order of its linked lists, drops small entries, and divides by
// the pivot.  Which entries survive depends on the values, but once the
// pattern is fixed, the order of every operation on a kept entry depends only
// on the pattern, and the host records it (RefactorPlan).  k_refactor replays
// it for new matrix values: one warp per column, columns taken in order by
// co-resident warps (cooperative launch), a finished column published with a
// release store of the refactorisation's epoch and awaited with bounded
// acquire polls, the column's accumulators in shared memory, every
// floating-point operation the host's, in the host's order, correctly
// rounded and never contracted.  With the matrix the factor was built from it
// reproduces the host factor bit for bit; with new values it computes the
// incomplete factor of the same pattern.
//
// The factor values then go into every device layout of the preconditioner's
// sweeps through maps built once from the factor's pattern: the level-order and
// slab layouts' value and diagonal arrays, and the streamed layout's round
// records (coefficients, and each row's diagonal or its reciprocal).
#include <algorithm>
#include <cmath>
#include <memory>

#include "kernels.cuh"
#include "solve.cuh"

namespace prism {

namespace {
constexpr int kRfWarps = kBlock / 32;
constexpr unsigned long long kRfWaitNs = 1000000000ull;  // 1 s per dependency wait
constexpr uint32_t kRfMaxCol = 1024;                      // longest column a warp holds in shared memory

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

struct RfArgs {
    uint32_t n, max_col, smax, epoch;
    const uint32_t* lt_rowptr;
    const uint32_t* lt_col;
    const uint32_t* a_col;
    const double* a_val;
    const uint32_t* a_ptr;
    const uint32_t* a_pos;
    const uint32_t* up_ptr;
    const uint32_t* up_k;
    const uint32_t* up_start;
    const uint32_t* sched;   // the columns in order of their depth in the dependency graph
    const uint64_t* uo;      // per column: offset of its first update entry in `slot`
    const uint16_t* slot;    // per update entry: its row's slot in the column, or kRfDrop
    uint32_t* done;     // per column: the epoch that finished it
    int* status;        // 0, PRISM_ERR_NOT_SPD, PRISM_ERR_ZERO_PIVOT or PRISM_ERR_TIMEOUT
    int* bad_col;       // the first column that raised it
    unsigned long long wait_ns;
};
constexpr uint16_t kRfDrop = 0xFFFFu;  // an update entry whose row is not in the column

// Per-warp shared memory of k_refactor: the column's accumulators and rows (max_col each),
// a chunk's products and their slots (smax each), and per update of the chunk its L_jk,
// D_k, start and first product.
__host__ __device__ inline size_t rf_warp_bytes(uint32_t max_col, uint32_t smax) {
    return ((size_t)max_col * (8 + 4) + (size_t)smax * (8 + 2) + 32 * (8 + 8 + 4 + 4) + 15) & ~(size_t)15;
}

// The column of each slot's row (slot 0: row j), in increasing order, and binary search.
struct RfCol {
    const uint32_t* rows;
    uint32_t m;
    __device__ int find(uint32_t i) const {
        uint32_t lo = 0, hi = m;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (rows[mid] < i) lo = mid + 1;
            else hi = mid;
        }
        return (lo < m && rows[lo] == i) ? (int)lo : -1;
    }
};

// Once per pattern: the slot in column j of every entry an update brings in (the entries
// of column k from row j down), laid out column after column, update after update.
__global__ void __launch_bounds__(kBlock) k_rf_slots(const RfArgs a, int ldlt) {
    extern __shared__ __align__(16) unsigned char rf_smem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t* rows = reinterpret_cast<uint32_t*>(rf_smem) + (size_t)wid * a.max_col;
    const uint32_t nwarps = gridDim.x * kRfWarps;
    for (uint32_t j = blockIdx.x * kRfWarps + wid; j < a.n; j += nwarps) {
        const uint32_t b = a.lt_rowptr[j], e = a.lt_rowptr[j + 1];
        const uint32_t m = ldlt ? e - b + 1 : e - b, off0 = ldlt ? b - 1 : b;
        for (uint32_t s = lane; s < m; s += 32) rows[s] = s == 0 ? j : a.lt_col[off0 + s];
        __syncwarp();
        const RfCol col{rows, m};
        uint64_t f = a.uo[j];
        for (uint32_t u = a.up_ptr[j]; u < a.up_ptr[j + 1]; ++u) {
            const uint32_t k = a.up_k[u], st = a.up_start[u], c = a.lt_rowptr[k + 1] - st;
            for (uint32_t t = lane; t < c; t += 32) {
                const int s = col.find(a.lt_col[st + t]);
                const_cast<uint16_t*>(a.slot)[f + t] = s < 0 ? kRfDrop : (uint16_t)s;
            }
            f += c;
        }
        __syncwarp();
    }
}

// Column j of the factor, one warp per column, columns taken in the order of `sched`
// (by depth in the dependency graph: a column's updates come from shallower columns, so
// the columns in flight at any time span a few levels of the graph, not a few planes of
// the natural order).  The updates are taken in chunks of up to
// 32 (the lanes wait for their columns k and load L_jk, D_k in parallel) whose entries fit
// `smax`: first every product L_ik L_jk (D_k) of the chunk into shared memory, all loads
// independent, then the subtractions in the host's update order.
template <typename Low, bool LDLT>
__global__ void __launch_bounds__(kBlock) k_refactor(const RfArgs a, Low* __restrict__ lt, double* __restrict__ D) {
    extern __shared__ __align__(16) unsigned char rf_smem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned char* base = rf_smem + (size_t)wid * rf_warp_bytes(a.max_col, a.smax);
    double* acc = reinterpret_cast<double*>(base);
    double* tv = acc + a.max_col;
    double* cL = tv + a.smax;
    double* cD = cL + 32;
    uint32_t* rows = reinterpret_cast<uint32_t*>(cD + 32);
    uint32_t* cst = rows + a.max_col;
    uint32_t* coff = cst + 32;
    uint16_t* tsl = reinterpret_cast<uint16_t*>(coff + 32);
    const uint32_t nwarps = gridDim.x * kRfWarps;
    auto fail = [&](int code, uint32_t col) {
        if (atomicCAS(a.status, 0, code) == 0) *a.bad_col = (int)col;
    };
    for (uint32_t w = blockIdx.x * kRfWarps + wid; w < a.n; w += nwarps) {
        const uint32_t j = a.sched[w];
        const uint32_t b = a.lt_rowptr[j], e = a.lt_rowptr[j + 1];
        // IC: the column's first entry is its diagonal; ILDLT stores none (slot 0 is row j anyway)
        const uint32_t m = LDLT ? e - b + 1 : e - b;
        const uint32_t off0 = LDLT ? b - 1 : b;  // entry of slot s is off0 + s (s >= 1)
        for (uint32_t s = lane; s < m; s += 32) {
            rows[s] = s == 0 ? j : a.lt_col[off0 + s];
            acc[s] = 0.0;
        }
        __syncwarp();
        const RfCol col{rows, m};
        // the matrix entries of row j at or below the diagonal, in stored order (duplicates add up)
        if (lane == 0) {
            for (uint32_t q = a.a_ptr[j]; q < a.a_ptr[j + 1]; ++q) {
                const uint32_t p = a.a_pos[q];
                const int s = col.find(a.a_col[p]);
                if (s >= 0) acc[s] = __dadd_rn(acc[s], a.a_val[p]);
            }
        }
        __syncwarp();
        bool ok = __all_sync(0xFFFFFFFFu, ld_relaxed_s32(a.status) == 0);  // the same in every lane
        uint64_t f0 = a.uo[j];
        const uint32_t uend = a.up_ptr[j + 1];
        for (uint32_t u0 = a.up_ptr[j]; u0 < uend && ok;) {
            const uint32_t u = u0 + lane;
            uint32_t c = 0, st = 0;
            double L = 0.0, dk = 0.0;
            bool mine = true;
            if (u < uend) {
                const uint32_t k = a.up_k[u];
                st = a.up_start[u];
                c = a.lt_rowptr[k + 1] - st;
                if (ld_acquire_u32(a.done + k) != a.epoch) {
                    const unsigned long long t0 = globaltimer_ns();
                    unsigned spins = 0;
                    while (ld_acquire_u32(a.done + k) != a.epoch) {
                        if ((++spins & 15u) == 0u &&
                            (ld_relaxed_s32(a.status) != 0 || globaltimer_ns() - t0 > a.wait_ns)) {
                            mine = false;
                            break;
                        }
                    }
                }
                if (mine) {
                    L = (double)lt[st];
                    if (LDLT) dk = D[k];
                }
            }
            if (!__all_sync(0xFFFFFFFFu, mine)) {
                ok = false;
                break;
            }
            // the chunk: the longest prefix of these updates whose entries fit smax (each
            // update alone does: c <= max_col <= smax)
            uint32_t incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                if (lane >= o) incl += t;
            }
            const unsigned fit = __ballot_sync(0xFFFFFFFFu, u < uend && incl <= a.smax);
            const int nu = __popc(fit);
            const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, nu - 1);
            if (lane < nu) {
                cL[lane] = L;
                cD[lane] = dk;
                cst[lane] = st;
                coff[lane] = incl - c;
            }
            __syncwarp();
            // every product of the chunk, with its slot
#pragma unroll 4
            for (uint32_t t = lane; t < total; t += 32) {
                int lo = 0, hi = nu - 1;  // the update of product t: the last coff <= t
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (coff[mid] <= t) lo = mid;
                    else hi = mid - 1;
                }
                const double Lik = (double)lt[cst[lo] + (t - coff[lo])];
                tv[t] = LDLT ? __dmul_rn(__dmul_rn(Lik, cL[lo]), cD[lo]) : __dmul_rn(Lik, cL[lo]);
                tsl[t] = a.slot[f0 + t];
            }
            __syncwarp();
            // the subtractions, update after update (a row appears once per update)
            for (int q = 0; q < nu; ++q) {
                const uint32_t b0 = coff[q], b1 = q + 1 < nu ? coff[q + 1] : total;
                for (uint32_t t = b0 + lane; t < b1; t += 32) {
                    const uint16_t sl = tsl[t];
                    if (sl != kRfDrop) acc[sl] = __dsub_rn(acc[sl], tv[t]);
                }
                __syncwarp();
            }
            u0 += nu;
            f0 += total;
        }
        if (!ok) {
            if (lane == 0) fail(PRISM_ERR_TIMEOUT, j);
            return;
        }
        // the pivot, then the column divided by it
        double piv = acc[0];
        if (LDLT) {
            if (fabs(piv) < 1e-15 && lane == 0) fail(PRISM_ERR_ZERO_PIVOT, j);
            if (lane == 0) D[j] = piv;
        } else {
            if (!(piv > 0.0) && lane == 0) fail(PRISM_ERR_NOT_SPD, j);
            piv = __dsqrt_rn(piv);
            if (lane == 0) lt[b] = (Low)piv;
        }
        for (uint32_t s = 1 + lane; s < m; s += 32) lt[off0 + s] = (Low)__ddiv_rn(acc[s], piv);
        __threadfence();  // every lane's values before the column is published
        __syncwarp();
        if (lane == 0) st_release_u32(a.done + j, a.epoch);
    }
}

// dst[cdst[t]] = src[csrc[t]]: new coefficients into a layout.  An index outside its
// array is not followed: the first such t is recorded (t + 1) in *bad for the host.
template <typename Low>
__global__ void __launch_bounds__(kBlock) k_rf_coef(uint32_t count, const uint32_t* __restrict__ cdst,
                                                    const uint32_t* __restrict__ csrc, const Low* __restrict__ src,
                                                    uint64_t src_n, Low* __restrict__ dst, uint64_t dst_n,
                                                    unsigned* bad) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        const uint32_t d = cdst[t], s = csrc[t];
        if (d >= dst_n || s >= src_n) {
            atomicCAS(bad, 0u, t + 1);
            continue;
        }
        dst[d] = src[s];
    }
}

// New diagonals into a layout: d = (double)lt[idx] (IC) or D[idx] (ILDLT), stored as d or
// 1/d (the streamed records of the dividing operations), in D2 (double or float).
template <typename Low, typename D2>
__global__ void __launch_bounds__(kBlock) k_rf_diag(uint32_t count, const uint32_t* __restrict__ ddst,
                                                    const uint32_t* __restrict__ dsrc, const Low* __restrict__ lt,
                                                    const double* __restrict__ D, uint64_t src_n, int ic, int recip,
                                                    D2* __restrict__ dst, uint64_t dst_n, unsigned* bad) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        const uint32_t di = ddst[t], si = dsrc[t];
        if (di >= dst_n || si >= src_n) {
            atomicCAS(bad, 0u, t + 1);
            continue;
        }
        const double d = ic ? (double)lt[si] : D[si];
        dst[di] = (D2)(recip ? 1.0 / d : d);
    }
}

int rf_grid(const Handle& h, uint64_t items) {
    uint64_t want = (items + kBlock - 1) / kBlock;
    const uint64_t cap = (uint64_t)h.info.sms * 8;
    if (want < 1) want = 1;
    return (int)(want < cap ? want : cap);
}
}  // namespace

// The maps of one device sweep: coefficient positions (in factor-value units) and
// diagonal positions (in the layout's diagonal units) with the factor entries they
// come from.
struct SweepValueMap {
    DevBuf<uint32_t> cdst, csrc, ddst, dsrc;
    uint32_t ncoef = 0, ndiag = 0;
};

struct RefactorState {
    uint32_t epoch = 0;
    DevBuf<uint32_t> lt_rowptr, lt_col, a_ptr, a_pos, up_ptr, up_k, up_start, done;
    DevBuf<uint32_t> sched;   // columns by depth in the dependency graph
    DevBuf<uint64_t> uo;      // per column: its first update entry
    DevBuf<uint16_t> slot;    // per update entry: the slot of its row in the column
    uint32_t smax = 0;
    DevBuf<float> lt32;
    DevBuf<double> lt64, D;
    DevBuf<int> status;       // [status, first bad column]
    DevBuf<unsigned> bad;     // first out-of-range map entry: [coefficients, diagonals]
    SweepValueMap lower, upper, lower_lv, upper_lv;
    bool refactored = false;  // the device factor differs from the host one
};
void refactor_release(RefactorState* r) { delete r; }

namespace {
void upload_map(SweepValueMap& M, const std::vector<uint32_t>& cd, const std::vector<uint32_t>& cs,
                const std::vector<uint32_t>& dd, const std::vector<uint32_t>& ds, cudaStream_t st) {
    M.ncoef = (uint32_t)cd.size();
    M.ndiag = (uint32_t)dd.size();
    M.cdst.upload(cd.data(), cd.size(), st);
    M.csrc.upload(cs.data(), cs.size(), st);
    M.ddst.upload(dd.data(), dd.size(), st);
    M.dsrc.upload(ds.data(), ds.size(), st);
}

// The map of device sweep d, uploaded from host sweep s (idx: the same sweep with factor
// entry indices as values and diagonal sources as diag).
template <typename Low>
void build_map(const DevSweep& d, const Sweep<Low>& s, const Sweep<double>& idx, SweepValueMap& M, cudaStream_t st) {
    std::vector<uint32_t> cd, cs, dd, ds;
    const bool has_diag = s.op != SWEEP_NONE;
    if (d.layout == LAYOUT_STREAM) {
        StreamLayout L;
        std::vector<uint32_t> cmap;
        std::string why;
        if (!stream_layout<Low>(s, slab_ranges<Low>(s, d.str_ctas_req), kNoSlot, d.str_slot_bytes, L, &why, nullptr,
                                &cmap, d.str_round_cap))
            throw Error(PRISM_ERR_CUDA, "streamed layout could not be rebuilt: " + why);
        cd.reserve(cmap.size() / 2);
        cs.reserve(cmap.size() / 2);
        for (size_t t = 0; t < cmap.size(); t += 2) {
            cd.push_back(cmap[t]);
            cs.push_back((uint32_t)idx.val[cmap[t + 1]]);
        }
        if (has_diag) {
            // each row's diagonal sits right after its right-hand side in its record
            for (uint32_t p = 0; p < idx.n; ++p) {
                dd.push_back(L.in_slot[idx.order[p]] + 1);
                ds.push_back((uint32_t)idx.diag[p]);
            }
        }
    } else {
        const Sweep<double>* src = &idx;
        Sweep<double> slab;
        if (d.layout == LAYOUT_SLAB) {
            std::vector<uint32_t> cpos;
            slab_layout<double>(idx, d.num_ctas, d.rows_per_cta, cpos, slab);
            src = &slab;
        }
        cd.resize(src->val.size());
        cs.resize(src->val.size());
        for (size_t t = 0; t < src->val.size(); ++t) {
            cd[t] = (uint32_t)t;
            cs[t] = (uint32_t)src->val[t];
        }
        if (has_diag) {
            dd.resize(src->n);
            ds.resize(src->n);
            for (uint32_t p = 0; p < src->n; ++p) {
                dd[p] = p;
                ds[p] = (uint32_t)src->diag[p];
            }
        }
    }
    upload_map(M, cd, cs, dd, ds, st);
}

// New values into device sweep d through its map (lt: lt_n factor values, D: n pivots);
// `bad` (two words, zero before) receives the first out-of-range map entry of each kernel.
template <typename Low>
void apply_map(const Handle& h, cudaStream_t st, DevSweep& d, const SweepValueMap& M, const Low* lt, uint64_t lt_n,
               const double* D, bool ic, unsigned* bad) {
    if (!d.n) return;
    if (M.ncoef) {
        const bool stream = d.layout == LAYOUT_STREAM;
        Low* dst = stream ? reinterpret_cast<Low*>(d.str_blob.get())
                          : (std::is_same<Low, float>::value ? reinterpret_cast<Low*>(d.val32.get())
                                                             : reinterpret_cast<Low*>(d.val64.get()));
        const uint64_t dst_n = stream ? d.str_blob.size() / sizeof(Low)
                                      : (std::is_same<Low, float>::value ? d.val32.size() : d.val64.size());
        k_rf_coef<Low><<<rf_grid(h, M.ncoef), kBlock, 0, st>>>(M.ncoef, M.cdst.get(), M.csrc.get(), lt, lt_n, dst,
                                                               dst_n, bad);
        PRISM_LAUNCHED();
    }
    if (M.ndiag) {
        const int recip = d.layout == LAYOUT_STREAM && (d.op == SWEEP_DIV || d.op == SWEEP_PREDIV);
        const uint64_t src_n = ic ? lt_n : d.n;
        if (d.layout == LAYOUT_STREAM && d.acc32) {
            k_rf_diag<Low, float><<<rf_grid(h, M.ndiag), kBlock, 0, st>>>(
                M.ndiag, M.ddst.get(), M.dsrc.get(), lt, D, src_n, ic, recip,
                reinterpret_cast<float*>(d.str_blob.get()), d.str_blob.size() / sizeof(float), bad + 1);
        } else {
            const bool stream = d.layout == LAYOUT_STREAM;
            double* dst = stream ? reinterpret_cast<double*>(d.str_blob.get()) : d.diag.get();
            const uint64_t dst_n = stream ? d.str_blob.size() / sizeof(double) : d.diag.size();
            k_rf_diag<Low, double><<<rf_grid(h, M.ndiag), kBlock, 0, st>>>(M.ndiag, M.ddst.get(), M.dsrc.get(), lt,
                                                                            D, src_n, ic, recip, dst, dst_n, bad + 1);
        }
        PRISM_LAUNCHED();
    }
}
}  // namespace

namespace {
// the scatter kernels' record of an out-of-range map entry, as an error
void check_maps(RefactorState& R, cudaStream_t st, const char* what) {
    unsigned b[2] = {0, 0};
    PRISM_CUDA(cudaMemcpyAsync(b, R.bad.get(), 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    PRISM_CUDA(cudaStreamSynchronize(st));
    if (b[0] || b[1])
        throw Error(PRISM_ERR_CUDA, std::string("refactorisation: a value map of ") + what +
                                        " points outside its arrays (coefficient entry " + std::to_string(b[0]) +
                                        ", diagonal entry " + std::to_string(b[1]) + ")");
}
}  // namespace

void TriangularPrecond::refactor() {
    const HostFactor& F = *f_;
    if ((F.kind != 1 && F.kind != 3) || !F.plan)
        throw Error(PRISM_ERR_UNSUPPORTED, "device refactorisation covers IC and ILDLT factors");
    const RefactorPlan& P = *F.plan;
    if (P.n != h_.A.n) throw Error(PRISM_ERR_ARG, "the factor does not belong to this operator");
    if (P.max_col > kRfMaxCol)
        throw Error(PRISM_ERR_UNSUPPORTED, "a factor column longer than " + std::to_string(kRfMaxCol) + " entries");
    cudaStream_t st = h_.stream;
    const bool ldlt = F.kind == 3;
    // A paired sweep's coefficients combine several factor entries, which the value maps
    // below cannot rebuild: such sweeps are tuned again without pairing first.
    if (!rf_ && (lower_.paired || upper_.paired)) {
        if (F.fp32) {
            if (lower_.paired) tune_sweep(h_, lower_, F.lower32, F.apply32, false);
            if (upper_.paired) tune_sweep(h_, upper_, F.upper32, F.apply32, false);
        } else {
            if (lower_.paired) tune_sweep(h_, lower_, F.lower64, false, false);
            if (upper_.paired) tune_sweep(h_, upper_, F.upper64, false, false);
        }
    }
    if (!rf_) {
        rf_.reset(new RefactorState());
        RefactorState& R = *rf_;
        R.lt_rowptr.upload(F.f0.rowptr.data(), F.f0.rowptr.size(), st);
        R.lt_col.upload(F.f0.col.data(), std::max<size_t>(F.f0.col.size(), 1), st);
        R.a_ptr.upload(P.a_ptr.data(), P.a_ptr.size(), st);
        R.a_pos.upload(P.a_pos.data(), std::max<size_t>(P.a_pos.size(), 1), st);
        R.up_ptr.upload(P.up_ptr.data(), P.up_ptr.size(), st);
        R.up_k.upload(P.up_k.data(), std::max<size_t>(P.up_k.size(), 1), st);
        R.up_start.upload(P.up_start.data(), std::max<size_t>(P.up_start.size(), 1), st);
        R.done.alloc(P.n);
        PRISM_CUDA(cudaMemsetAsync(R.done.get(), 0, (size_t)P.n * sizeof(uint32_t), st));
        // where each column's update entries start, and (on the device, once) their slots
        std::vector<uint64_t> uo((size_t)P.n + 1, 0);
        for (uint32_t j = 0; j < P.n; ++j) {
            uint64_t c = 0;
            for (uint32_t u = P.up_ptr[j]; u < P.up_ptr[j + 1]; ++u)
                c += F.f0.rowptr[P.up_k[u] + 1] - P.up_start[u];
            uo[j + 1] = uo[j] + c;
        }
        R.uo.upload(uo.data(), uo.size(), st);
        // depth of each column in the dependency graph (its updates come from columns k < j),
        // and the columns ordered by depth, then index
        std::vector<uint32_t> depth(P.n, 0), sched(std::max<uint32_t>(P.n, 1), 0);
        uint32_t maxd = 0;
        for (uint32_t j = 0; j < P.n; ++j) {
            uint32_t d = 0;
            for (uint32_t u = P.up_ptr[j]; u < P.up_ptr[j + 1]; ++u) d = std::max(d, depth[P.up_k[u]] + 1);
            depth[j] = d;
            maxd = std::max(maxd, d);
        }
        std::vector<uint32_t> start((size_t)maxd + 2, 0);
        for (uint32_t j = 0; j < P.n; ++j) ++start[depth[j] + 1];
        for (uint32_t d = 0; d <= maxd; ++d) start[d + 1] += start[d];
        for (uint32_t j = 0; j < P.n; ++j) sched[start[depth[j]]++] = j;
        R.sched.upload(sched.data(), sched.size(), st);
        R.slot.alloc(std::max<uint64_t>(uo[P.n], 1));
        R.smax = std::max<uint32_t>(512, (P.max_col + 31) / 32 * 32);
        const size_t nnz = std::max<size_t>(F.f0.col.size(), 1);
        if (F.fp32) R.lt32.alloc(nnz);
        else R.lt64.alloc(nnz);
        R.D.alloc(std::max<uint32_t>(P.n, 1));
        R.status.alloc(2);
        R.bad.alloc(2);
        Sweep<double> ilo, iup;
        factor_index_sweeps(F, ilo, iup);
        if (F.fp32) {
            build_map<float>(lower_, F.lower32, ilo, R.lower, st);
            build_map<float>(upper_, F.upper32, iup, R.upper, st);
        } else {
            build_map<double>(lower_, F.lower64, ilo, R.lower, st);
            build_map<double>(upper_, F.upper64, iup, R.upper, st);
        }
        PRISM_CUDA(cudaStreamSynchronize(st));
    }
    RefactorState& R = *rf_;
    RfArgs a;
    a.n = P.n;
    a.max_col = std::max<uint32_t>(P.max_col, 1);
    a.smax = R.smax;
    a.sched = R.sched.get();
    a.uo = R.uo.get();
    a.slot = R.slot.get();
    a.lt_rowptr = R.lt_rowptr.get();
    a.lt_col = R.lt_col.get();
    a.a_col = h_.A.col.get();
    a.a_val = h_.A.val.get();
    a.a_ptr = R.a_ptr.get();
    a.a_pos = R.a_pos.get();
    a.up_ptr = R.up_ptr.get();
    a.up_k = R.up_k.get();
    a.up_start = R.up_start.get();
    a.done = R.done.get();
    a.status = R.status.get();
    a.bad_col = R.status.get() + 1;
    a.wait_ns = kRfWaitNs;
    if (R.epoch == 0) {  // the slots, once per pattern
        const size_t ssm = (size_t)kRfWarps * a.max_col * sizeof(uint32_t);
        PRISM_CUDA(cudaFuncSetAttribute(k_rf_slots, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssm));
        const uint64_t want = ((uint64_t)P.n + kRfWarps - 1) / kRfWarps;
        const int g = (int)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)h_.info.sms * 4));
        k_rf_slots<<<g, kBlock, ssm, st>>>(a, ldlt ? 1 : 0);
        PRISM_LAUNCHED();
        PRISM_CUDA(cudaStreamSynchronize(st));
    }
    ++R.epoch;
    a.epoch = R.epoch;
    PRISM_CUDA(cudaMemsetAsync(R.status.get(), 0, 2 * sizeof(int), st));
    const size_t smem = (size_t)kRfWarps * rf_warp_bytes(a.max_col, a.smax);
    void* fn = F.fp32 ? (ldlt ? (void*)k_refactor<float, true> : (void*)k_refactor<float, false>)
                      : (ldlt ? (void*)k_refactor<double, true> : (void*)k_refactor<double, false>);
    PRISM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    PRISM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kBlock, smem));
    if (occ < 1) throw Error(PRISM_ERR_UNSUPPORTED, "the refactorisation kernel does not fit on an SM");
    const uint64_t want = ((uint64_t)P.n + kRfWarps - 1) / kRfWarps;
    const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)h_.info.sms * occ));
    void* lt = F.fp32 ? (void*)R.lt32.get() : (void*)R.lt64.get();
    double* D = R.D.get();
    void* args[] = {&a, &lt, &D};
    PRISM_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kBlock), args, smem, st));
    PRISM_LAUNCHED();
    int hs[2] = {0, 0};
    PRISM_CUDA(cudaMemcpyAsync(hs, R.status.get(), 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    PRISM_CUDA(cudaStreamSynchronize(st));
    if (hs[0] == PRISM_ERR_NOT_SPD)
        throw Error(PRISM_ERR_NOT_SPD, "refactorisation: non-positive pivot in column " + std::to_string(hs[1]));
    if (hs[0] == PRISM_ERR_ZERO_PIVOT)
        throw Error(PRISM_ERR_ZERO_PIVOT, "refactorisation: zero pivot in column " + std::to_string(hs[1]));
    if (hs[0] != 0) throw Error(hs[0], "refactorisation: a dependency wait ran out in column " + std::to_string(hs[1]));
    // the new values into every device layout of the two sweeps
    const bool ic = F.kind == 1;
    const uint64_t lt_n = F.f0.col.size();
    PRISM_CUDA(cudaMemsetAsync(R.bad.get(), 0, 2 * sizeof(unsigned), st));
    if (F.fp32) {
        apply_map<float>(h_, st, lower_, R.lower, R.lt32.get(), lt_n, D, ic, R.bad.get());
        apply_map<float>(h_, st, upper_, R.upper, R.lt32.get(), lt_n, D, ic, R.bad.get());
    } else {
        apply_map<double>(h_, st, lower_, R.lower, R.lt64.get(), lt_n, D, ic, R.bad.get());
        apply_map<double>(h_, st, upper_, R.upper, R.lt64.get(), lt_n, D, ic, R.bad.get());
    }
    check_maps(R, st, "the sweeps");
    // the level-order copies of the block solves are uploaded again on their next use, with
    // the new values (refresh_level_copy)
    lower_lv_.release();
    upper_lv_.release();
    R.refactored = true;
    PRISM_CUDA(cudaStreamSynchronize(st));
}

void TriangularPrecond::refresh_level_copy(DevSweep& d, bool lower) {
    if (!rf_ || !rf_->refactored) return;
    const HostFactor& F = *f_;
    RefactorState& R = *rf_;
    cudaStream_t st = h_.stream;
    Sweep<double> ilo, iup;
    factor_index_sweeps(F, ilo, iup);
    SweepValueMap& M = lower ? R.lower_lv : R.upper_lv;
    const uint64_t lt_n = F.f0.col.size();
    PRISM_CUDA(cudaMemsetAsync(R.bad.get(), 0, 2 * sizeof(unsigned), st));
    if (F.fp32) {
        build_map<float>(d, lower ? F.lower32 : F.upper32, lower ? ilo : iup, M, st);
        apply_map<float>(h_, st, d, M, R.lt32.get(), lt_n, R.D.get(), F.kind == 1, R.bad.get());
    } else {
        build_map<double>(d, lower ? F.lower64 : F.upper64, lower ? ilo : iup, M, st);
        apply_map<double>(h_, st, d, M, R.lt64.get(), lt_n, R.D.get(), F.kind == 1, R.bad.get());
    }
    check_maps(R, st, "a level-order copy");
}

int TriangularPrecond::export_refactored(int which, uint32_t* n, uint64_t* nnz, uint32_t* rowptr, uint32_t* col,
                                         double* val, double* diag) const {
    const HostFactor& F = *f_;
    const RefactorState& R = *rf_;
    if (which != 0) return 9;
    const uint32_t nn = F.f0.n;
    const size_t m = F.f0.col.size();
    if (n) *n = nn;
    if (nnz) *nnz = m;
    if (rowptr) std::copy(F.f0.rowptr.begin(), F.f0.rowptr.end(), rowptr);
    if (col) std::copy(F.f0.col.begin(), F.f0.col.end(), col);
    if (val) {
        if (F.fp32) {
            std::vector<float> v(m);
            PRISM_CUDA(cudaMemcpy(v.data(), R.lt32.get(), m * sizeof(float), cudaMemcpyDeviceToHost));
            for (size_t t = 0; t < m; ++t) val[t] = (double)v[t];
        } else {
            PRISM_CUDA(cudaMemcpy(val, R.lt64.get(), m * sizeof(double), cudaMemcpyDeviceToHost));
        }
    }
    if (diag && F.kind == 3) PRISM_CUDA(cudaMemcpy(diag, R.D.get(), nn * sizeof(double), cudaMemcpyDeviceToHost));
    return 0;
}

}  // namespace prism
