// extern "C" boundary of the solve phase (declared in include/prism_solve.h).
// Every entry point catches everything: no C++ exception crosses the ABI.
#include <cstring>
#include <string>

#include "../../include/prism_solve.h"
#include "solve.cuh"

using prism::Error;
using prism::Handle;

namespace {
thread_local std::string g_last_error;

int fail(int status, const std::string& msg) {
    g_last_error = msg;
    return status;
}

template <typename F>
int guarded(F&& f) {
    try {
        g_last_error.clear();
        return f();
    } catch (const Error& e) {
        return fail(e.status, e.what());
    } catch (const std::bad_alloc&) {
        return fail(PRISM_ERR_ALLOC, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(PRISM_ERR_ARG, e.what());
    } catch (...) {
        return fail(PRISM_ERR_ARG, "unknown error");
    }
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};
}  // namespace

namespace prism {
int record_error(int status, const char* msg) {
    if (status == PRISM_OK) g_last_error.clear();
    else g_last_error = msg;
    return status;
}
}  // namespace prism

struct prism_handle_s : Handle {};

struct prism_factor_s {
    std::shared_ptr<const prism::HostFactor> f;      // IC / ILUT / ILDLT
    std::shared_ptr<const prism::HostAmsed> amsed;   // AMSED / MSLR
};

static prism::AmsedOptions to_options(const prism_amsed_opts* o) {
    prism::AmsedOptions a;
    a.levels = o->levels;
    a.lanczos_steps = o->lanczos_steps;
    a.low_rank = o->low_rank;
    a.eig_bound = o->eig_bound;
    a.lowrank_type = o->lowrank_type;
    a.lanczos_type = o->lanczos_type;
    a.reorder = o->reorder;
    a.factor_tol = o->factor_tol;
    a.minsep = o->minsep;
    a.seed = o->seed;
    return a;
}

static bool valid_precision(int32_t p) { return p == PRISM_FP64 || p == PRISM_FP32 || p == PRISM_FP32_APPLY; }

static std::shared_ptr<prism::HostAmsed> build_amsed(const prism::CsrHost& A, const prism_amsed_opts* o,
                                                     int32_t precision, int* rc, std::string* err, int family = 5) {
    auto h = std::make_shared<prism::HostAmsed>();
    h->fp32 = precision != PRISM_FP64;
    h->apply32 = precision == PRISM_FP32_APPLY;
    h->opt = to_options(o);
    h->opt.family = family;
    if (h->fp32) {
        h->s32 = std::make_shared<prism::AmsedSetup<float>>();
        *rc = prism::amsed_setup<float>(A, h->opt, *h->s32, err);
    } else {
        h->s64 = std::make_shared<prism::AmsedSetup<double>>();
        *rc = prism::amsed_setup<double>(A, h->opt, *h->s64, err);
    }
    return h;
}

static int32_t set_tri(prism_handle h, int kind, double tol, uint32_t lfill, int32_t precision) {
    if (!h) return fail(PRISM_ERR_ARG, "null handle");
    if (!valid_precision(precision)) return fail(PRISM_ERR_ARG, "precision must be PRISM_FP64, PRISM_FP32 or PRISM_FP32_APPLY");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        h->P.reset();
        auto f = std::make_shared<prism::HostFactor>();
        std::string err;
        int rc = prism::build_triangular(kind, h->A_host, tol, lfill, precision != PRISM_FP64, *f, &err);
        if (rc) return fail(rc, err);
        f->apply32 = precision == PRISM_FP32_APPLY;
        h->P = std::make_unique<prism::TriangularPrecond>(*h, std::move(f));
        return PRISM_OK;
    });
}


// A gather-form triangular sweep from caller arrays (dependencies on one side of the diagonal).
template <typename Low>
static void gather_sweep(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
                         const double* diag, int op, bool lower, prism::Sweep<Low>& s) {
    const uint64_t nnz = rowptr[n];
    std::vector<uint32_t> rp(rowptr, rowptr + n + 1), ci(col, col + nnz);
    std::vector<Low> v(nnz);
    for (uint64_t k = 0; k < nnz; ++k) v[k] = (Low)val[k];
    std::vector<double> d;
    if (diag) d.assign(diag, diag + n);
    prism::build_sweep<Low>(n, rp, ci, v, diag ? &d : nullptr, op, lower, s);
}

static int check_gather_form(uint32_t n, const uint32_t* rowptr, const uint32_t* col, int32_t lower) {
    for (uint32_t r = 0; r < n; ++r) {
        if (rowptr[r + 1] < rowptr[r]) return fail(PRISM_ERR_ARG, "row offsets decrease");
        for (uint32_t k = rowptr[r]; k < rowptr[r + 1]; ++k)
            if (col[k] >= n || (lower ? col[k] >= r : col[k] <= r))
                return fail(PRISM_ERR_ARG, "dependency on the wrong side of the diagonal");
    }
    return PRISM_OK;
}

static int copy_order(const prism::StreamOrder& o, uint32_t n, uint32_t* eptr, uint32_t* edep, double* ecoef,
                      uint32_t* kptr, uint32_t* kdep, double* kcoef) {
    if (o.eptr.size() != (size_t)n + 1) return fail(PRISM_ERR_ARG, "order size");
    std::memcpy(eptr, o.eptr.data(), o.eptr.size() * sizeof(uint32_t));
    std::memcpy(kptr, o.kptr.data(), o.kptr.size() * sizeof(uint32_t));
    if (edep) std::memcpy(edep, o.edep.data(), o.edep.size() * sizeof(uint32_t));
    if (ecoef) std::memcpy(ecoef, o.ecoef.data(), o.ecoef.size() * sizeof(double));
    if (kdep) std::memcpy(kdep, o.kdep.data(), o.kdep.size() * sizeof(uint32_t));
    if (kcoef) std::memcpy(kcoef, o.kcoef.data(), o.kcoef.size() * sizeof(double));
    return PRISM_OK;
}

template <typename Low>
static int stream_selftest(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
                           const double* diag, int op, bool lower, uint32_t num_ctas, uint32_t rows_per_cta,
                           uint32_t slot_bytes, const double* in, double* out, uint32_t max_round_bytes = 0,
                           uint32_t* record_bytes = nullptr) {
    const uint64_t nnz = rowptr[n];
    std::vector<uint32_t> rp(rowptr, rowptr + n + 1), ci(col, col + nnz);
    std::vector<Low> v(nnz);
    for (uint64_t k = 0; k < nnz; ++k) v[k] = (Low)val[k];
    std::vector<double> d;
    if (diag) d.assign(diag, diag + n);
    prism::Sweep<Low> s;
    prism::build_sweep<Low>(n, rp, ci, v, diag ? &d : nullptr, op, lower, s);
    // rows_per_cta = 0: the slab boundaries the device layout would choose
    std::vector<uint32_t> start;
    if (rows_per_cta == 0) {
        start = prism::slab_ranges<Low>(s, num_ctas);
    } else {
        if ((uint64_t)num_ctas * rows_per_cta < n) return fail(PRISM_ERR_UNSUPPORTED, "slabs do not cover the rows");
        for (uint32_t b = 0; b <= num_ctas; ++b)
            start.push_back((uint32_t)std::min<uint64_t>((uint64_t)b * rows_per_cta, n));
    }
    prism::StreamLayout L;
    std::string why;
    if (!prism::stream_layout<Low>(s, start, prism::kNoSlot, slot_bytes, L, &why, nullptr, nullptr, max_round_bytes))
        return fail(PRISM_ERR_UNSUPPORTED, why);
    if (record_bytes) *record_bytes = L.max_round_bytes;
    why = prism::stream_layout_replay<Low>(s, L, in, out);
    if (!why.empty()) return fail(PRISM_ERR_ARG, "stream layout: " + why);
    return PRISM_OK;
}

extern "C" {

const char* prism_last_error(void) { return g_last_error.c_str(); }

int32_t prism_version(void) { return 100; }

uint64_t prism_kernel_launch_count(void) { return prism::launch_counter().load(); }

int32_t prism_selftest_wait_timeout(int32_t device, uint64_t wait_ns, int32_t* device_status) {
    if (!device_status) return fail(PRISM_ERR_ARG, "null output");
    if (wait_ns == 0 || wait_ns > 2000000000ull) return fail(PRISM_ERR_ARG, "wait_ns must be in (0, 2 s]");
    return guarded([&]() -> int {
        int s = -1;
        DeviceGuard g(device);
        prism::selftest_wait_timeout(device, wait_ns, &s);
        *device_status = s;
        return PRISM_OK;
    });
}

int32_t prism_lowrank_block_run(int32_t device, uint32_t nrem, uint32_t rank, uint32_t k, const double* W,
                                const double* H, const double* X, double* Y, int32_t tensor) {
    if (!W || !H || !X || !Y || nrem == 0) return fail(PRISM_ERR_ARG, "null array or empty block");
    if (rank == 0 || rank > 128 || k == 0 || k > 64) return fail(PRISM_ERR_ARG, "rank must be in [1, 128], k in [1, 64]");
    return guarded([&]() -> int {
        DeviceGuard g(device);
        prism::lowrank_block_run(device, nrem, rank, k, W, H, X, Y, tensor != 0);
        return PRISM_OK;
    });
}

int32_t prism_stream_sweep_order(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
                                 const double* diag, int32_t op, int32_t lower, int32_t precision, uint32_t num_ctas,
                                 uint32_t* eptr, uint32_t* edep, double* ecoef, uint32_t* kptr, uint32_t* kdep,
                                 double* kcoef) {
    if (!rowptr || !col || !val || !eptr || !kptr || n == 0) return fail(PRISM_ERR_ARG, "null array or empty sweep");
    if (op < 0 || op > 3 || (op != 2 && !diag)) return fail(PRISM_ERR_ARG, "bad op / missing diagonal");
    if (!valid_precision(precision) || num_ctas == 0) return fail(PRISM_ERR_ARG, "bad precision or slab count");
    return guarded([&]() -> int {
        int rc = check_gather_form(n, rowptr, col, lower);
        if (rc) return rc;
        const uint32_t slot_bytes = precision == PRISM_FP32_APPLY ? 4 : 8;
        const uint32_t ctas = prism::stream_slab_count(n, num_ctas, 32);
        prism::StreamOrder o;
        prism::StreamLayout L;
        std::string why;
        bool ok;
        if (precision != PRISM_FP64) {
            prism::Sweep<float> s;
            gather_sweep<float>(n, rowptr, col, val, diag, op, lower != 0, s);
            ok = prism::stream_layout<float>(s, prism::slab_ranges<float>(s, ctas), prism::kNoSlot, slot_bytes, L,
                                             &why, &o);
        } else {
            prism::Sweep<double> s;
            gather_sweep<double>(n, rowptr, col, val, diag, op, lower != 0, s);
            ok = prism::stream_layout<double>(s, prism::slab_ranges<double>(s, ctas), prism::kNoSlot, 8, L, &why, &o);
        }
        if (!ok) return fail(PRISM_ERR_UNSUPPORTED, why);
        return copy_order(o, n, eptr, edep, ecoef, kptr, kdep, kcoef);
    });
}

int32_t prism_stream_sweep_run(int32_t device, uint32_t n, const uint32_t* rowptr, const uint32_t* col,
                               const double* val, const double* diag, int32_t op, int32_t lower, int32_t precision,
                               uint32_t num_ctas, const double* in, double* out) {
    if (!rowptr || !col || !val || !in || !out || n == 0) return fail(PRISM_ERR_ARG, "null array or empty sweep");
    if (op < 0 || op > 3 || (op != 2 && !diag)) return fail(PRISM_ERR_ARG, "bad op / missing diagonal");
    if (!valid_precision(precision) || num_ctas == 0) return fail(PRISM_ERR_ARG, "bad precision or slab count");
    return guarded([&]() -> int {
        int rc = check_gather_form(n, rowptr, col, lower);
        if (rc) return rc;
        DeviceGuard g(device);
        if (precision != PRISM_FP64) {
            prism::Sweep<float> s;
            gather_sweep<float>(n, rowptr, col, val, diag, op, lower != 0, s);
            prism::stream_sweep_run<float>(device, s, precision == PRISM_FP32_APPLY, num_ctas, in, out);
        } else {
            prism::Sweep<double> s;
            gather_sweep<double>(n, rowptr, col, val, diag, op, lower != 0, s);
            prism::stream_sweep_run<double>(device, s, false, num_ctas, in, out);
        }
        return PRISM_OK;
    });
}

int32_t prism_stream_sweep_pair(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
                                const double* diag, int32_t op, int32_t lower, int32_t precision, uint64_t* pnnz,
                                uint32_t* prow, uint32_t* pcol, double* pval, uint64_t* mnnz, uint32_t* mptr,
                                uint32_t* mdep, double* mcoef) {
    if (!rowptr || !col || !val || !pnnz || !mnnz || n == 0) return fail(PRISM_ERR_ARG, "null array or empty sweep");
    if (op < 0 || op > 3 || (op != 2 && !diag)) return fail(PRISM_ERR_ARG, "bad op / missing diagonal");
    if (!valid_precision(precision)) return fail(PRISM_ERR_ARG, "bad precision");
    return guarded([&]() -> int {
        int rc = check_gather_form(n, rowptr, col, lower);
        if (rc) return rc;
        auto emit = [&](auto& s) {
            using S = std::decay_t<decltype(s)>;
            S ps;
            prism::PairMap pm;
            prism::pair_sweep(s, ps, pm);
            *pnnz = ps.col.size();
            *mnnz = pm.dep.size();
            if (prow) {  // gather form by row
                std::vector<uint32_t> pos(n);
                for (uint32_t p = 0; p < n; ++p) pos[ps.order[p]] = p;
                prow[0] = 0;
                for (uint32_t r = 0; r < n; ++r) {
                    const uint32_t p = pos[r], len = ps.rowptr[p + 1] - ps.rowptr[p];
                    prow[r + 1] = prow[r] + len;
                    for (uint32_t t = 0; t < len; ++t) {
                        if (pcol) pcol[prow[r] + t] = ps.col[ps.rowptr[p] + t];
                        if (pval) pval[prow[r] + t] = (double)ps.val[ps.rowptr[p] + t];
                    }
                }
            }
            if (mptr) std::copy(pm.ptr.begin(), pm.ptr.end(), mptr);
            if (mdep) std::copy(pm.dep.begin(), pm.dep.end(), mdep);
            if (mcoef) std::copy(pm.coef.begin(), pm.coef.end(), mcoef);
        };
        if (precision != PRISM_FP64) {
            prism::Sweep<float> s;
            gather_sweep<float>(n, rowptr, col, val, diag, op, lower != 0, s);
            emit(s);
        } else {
            prism::Sweep<double> s;
            gather_sweep<double>(n, rowptr, col, val, diag, op, lower != 0, s);
            emit(s);
        }
        return PRISM_OK;
    });
}

int32_t prism_precond_sweep_rhs_map(prism_handle h, int32_t sweep, int32_t* paired, uint64_t* mnnz, uint32_t* mptr,
                                    uint32_t* mdep, double* mcoef) {
    if (!h || !paired || !mnnz) return fail(PRISM_ERR_ARG, "null handle or output");
    if (!h->P) return fail(PRISM_ERR_NOT_READY, "no preconditioner");
    return guarded([&]() -> int {
        uint32_t rows = 0;
        if (!h->P->sweep_info(sweep, &rows, nullptr, nullptr, nullptr, nullptr))
            return fail(PRISM_ERR_ARG, "no such sweep");
        prism::StreamOrder o;
        if (!h->P->sweep_order(sweep, o)) return fail(PRISM_ERR_UNSUPPORTED, "the sweep does not run the streamed kernel");
        *paired = o.mptr.empty() ? 0 : 1;
        *mnnz = o.mdep.size();
        if (mptr) {
            if (o.mptr.empty()) std::fill(mptr, mptr + rows + 1, 0u);
            else std::copy(o.mptr.begin(), o.mptr.end(), mptr);
        }
        if (mdep) std::copy(o.mdep.begin(), o.mdep.end(), mdep);
        if (mcoef) std::copy(o.mcoef.begin(), o.mcoef.end(), mcoef);
        return PRISM_OK;
    });
}

int32_t prism_precond_sweep_order(prism_handle h, int32_t sweep, uint32_t* n, uint32_t* eptr, uint32_t* edep,
                                  double* ecoef, uint32_t* kptr, uint32_t* kdep, double* kcoef, double* diag,
                                  int32_t* op, int32_t* lower) {
    if (!h || !n) return fail(PRISM_ERR_ARG, "null handle or size");
    if (!h->P) return fail(PRISM_ERR_NOT_READY, "no preconditioner");
    return guarded([&]() -> int {
        uint32_t rows = 0;
        if (!h->P->sweep_info(sweep, &rows, nullptr, nullptr, nullptr, nullptr))
            return fail(PRISM_ERR_ARG, "no such sweep");
        *n = rows;
        if (!eptr && !kptr) return PRISM_OK;
        if (!eptr || !kptr) return fail(PRISM_ERR_ARG, "eptr and kptr go together");
        prism::StreamOrder o;
        if (!h->P->sweep_order(sweep, o)) return fail(PRISM_ERR_UNSUPPORTED, "the sweep does not run the streamed kernel");
        if (diag) std::memcpy(diag, o.diag.data(), o.diag.size() * sizeof(double));
        if (op) *op = o.op;
        if (lower) *lower = o.lower ? 1 : 0;
        return copy_order(o, rows, eptr, edep, ecoef, kptr, kdep, kcoef);
    });
}

int32_t prism_selftest_stream_layout(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
                                     const double* diag, int32_t op, int32_t lower, int32_t precision,
                                     uint32_t num_ctas, uint32_t rows_per_cta, const double* in, double* out) {
    return prism_selftest_stream_layout_capped(n, rowptr, col, val, diag, op, lower, precision, num_ctas,
                                               rows_per_cta, 0, in, out, nullptr);
}

int32_t prism_selftest_stream_layout_capped(uint32_t n, const uint32_t* rowptr, const uint32_t* col,
                                            const double* val, const double* diag, int32_t op, int32_t lower,
                                            int32_t precision, uint32_t num_ctas, uint32_t rows_per_cta,
                                            uint32_t max_round_bytes, const double* in, double* out,
                                            uint32_t* record_bytes) {
    if (!rowptr || !col || !val || !in || !out) return fail(PRISM_ERR_ARG, "null array");
    if (op < 0 || op > 3 || (op != 2 && !diag)) return fail(PRISM_ERR_ARG, "bad op / missing diagonal");
    return guarded([&]() -> int {
        for (uint32_t r = 0; r < n; ++r)
            for (uint32_t k = rowptr[r]; k < rowptr[r + 1]; ++k)
                if (col[k] >= n || (lower ? col[k] >= r : col[k] <= r))
                    return fail(PRISM_ERR_ARG, "dependency on the wrong side of the diagonal");
        const uint32_t slot_bytes = precision == PRISM_FP32_APPLY ? 4 : 8;
        if (precision != PRISM_FP64)
            return stream_selftest<float>(n, rowptr, col, val, diag, op, lower != 0, num_ctas, rows_per_cta,
                                          slot_bytes, in, out, max_round_bytes, record_bytes);
        return stream_selftest<double>(n, rowptr, col, val, diag, op, lower != 0, num_ctas, rows_per_cta, 8, in,
                                       out, max_round_bytes, record_bytes);
    });
}

int32_t prism_mtx_read(const char* path, int32_t base, int32_t part, uint32_t* rows, uint32_t* cols, uint64_t* nnz,
                       uint32_t* rowptr, uint32_t* col, double* val) {
    if (!path || !rows || !cols || !nnz) return fail(PRISM_ERR_ARG, "null argument");
    if (base < 0 || (part != 0 && part != 1)) return fail(PRISM_ERR_ARG, "index base must be >= 0, part 0 or 1");
    return guarded([&]() -> int {
        uint32_t r = 0, c = 0;
        std::vector<uint32_t> rp, ci;
        std::vector<double> v;
        std::string err;
        int rc = prism::read_mtx(path, (uint32_t)base, part, r, c, rp, ci, v, &err);
        if (rc) return fail(PRISM_ERR_ARG, "Matrix Market: " + err);
        *rows = r;
        *cols = c;
        *nnz = ci.size();
        if (rowptr) std::memcpy(rowptr, rp.data(), rp.size() * sizeof(uint32_t));
        if (col) std::memcpy(col, ci.data(), ci.size() * sizeof(uint32_t));
        if (val) std::memcpy(val, v.data(), v.size() * sizeof(double));
        return PRISM_OK;
    });
}

int32_t prism_mtx_read_dense(const char* path, uint32_t* rows, uint32_t* cols, double* values) {
    if (!path || !rows || !cols) return fail(PRISM_ERR_ARG, "null argument");
    return guarded([&]() -> int {
        uint32_t r = 0, c = 0;
        std::vector<double> v;
        std::string err;
        int rc = prism::read_mtx_dense(path, r, c, v, &err);
        if (rc) return fail(PRISM_ERR_ARG, "Matrix Market: " + err);
        *rows = r;
        *cols = c;
        if (values) std::memcpy(values, v.data(), v.size() * sizeof(double));
        return PRISM_OK;
    });
}

int32_t prism_laplacian_dims(int32_t nx, int32_t ny, int32_t nz, uint32_t* n, uint32_t* nnz) {
    if (!n || !nnz) return fail(PRISM_ERR_ARG, "null output pointer");
    if (!prism::laplacian_dims(nx, ny, nz, n, nnz)) return fail(PRISM_ERR_ARG, "grid dimensions out of range");
    return PRISM_OK;
}

int32_t prism_laplacian_fill(int32_t nx, int32_t ny, int32_t nz, double ax, double ay, double az, double shift,
                             uint32_t* rowptr, uint32_t* col, double* val) {
    uint32_t n, nnz;
    if (!rowptr || !col || !val) return fail(PRISM_ERR_ARG, "null output pointer");
    if (!prism::laplacian_dims(nx, ny, nz, &n, &nnz)) return fail(PRISM_ERR_ARG, "grid dimensions out of range");
    return guarded([&]() -> int {
        prism::laplacian_fill(nx, ny, nz, ax, ay, az, shift, rowptr, col, val);
        return PRISM_OK;
    });
}

int32_t prism_create(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val, int32_t device,
                     prism_handle* out) {
    if (!out) return fail(PRISM_ERR_ARG, "null output handle");
    *out = nullptr;
    if (n == 0) return fail(PRISM_ERR_ARG, "empty matrix (n == 0)");
    if (!rowptr || !col || !val) return fail(PRISM_ERR_ARG, "null CSR array");
    std::string bad = prism::validate_csr(n, rowptr, col);
    if (!bad.empty()) return fail(PRISM_ERR_BAD_MATRIX, bad);
    return guarded([&]() -> int {
        int ndev = 0;
        PRISM_CUDA(cudaGetDeviceCount(&ndev));
        if (device < 0 || device >= ndev)
            return fail(PRISM_ERR_ARG, "device " + std::to_string(device) + " not present (" + std::to_string(ndev) + " devices)");
        DeviceGuard g(device);
        auto* h = new prism_handle_s();
        try {
            prism::init_device_info(h->info, device);
            PRISM_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
            h->own_stream = true;
            PRISM_CUDA(cudaEventCreate(&h->ev0));
            PRISM_CUDA(cudaEventCreate(&h->ev1));
            PRISM_CUDA(cudaMallocHost(&h->pinned, prism::Handle::kScalarCapacity * sizeof(double)));
            const uint64_t nnz = rowptr[n];
            h->A_host.n = n;
            h->A_host.rowptr.assign(rowptr, rowptr + n + 1);
            h->A_host.col.assign(col, col + nnz);
            h->A_host.val.assign(val, val + nnz);
            h->A.n = n;
            h->A.nnz = nnz;
            h->A.rowptr.upload(rowptr, (size_t)n + 1, h->stream);
            h->A.col.upload(col, nnz, h->stream);
            h->A.val.upload(val, nnz, h->stream);
            h->red.partial.alloc(prism::Reducer::kMaxGrid * 2);
            h->red.ticket.alloc(1);
            h->red.scalars.alloc(prism::Handle::kScalarCapacity);
            h->status.alloc(1);
            PRISM_CUDA(cudaMemsetAsync(h->red.ticket.get(), 0, sizeof(unsigned), h->stream));
            PRISM_CUDA(cudaMemsetAsync(h->red.scalars.get(), 0, prism::Handle::kScalarCapacity * sizeof(double),
                                       h->stream));
            PRISM_CUDA(cudaMemsetAsync(h->status.get(), 0, sizeof(int), h->stream));
            PRISM_CUDA(cudaStreamSynchronize(h->stream));
            h->tune_spmv();
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        return PRISM_OK;
    });
}

int32_t prism_destroy(prism_handle h) {
    if (!h) return PRISM_OK;
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        cudaStreamSynchronize(h->stream);
        delete h;
        return PRISM_OK;
    });
}

int32_t prism_set_stream(prism_handle h, void* stream) {
    if (!h) return fail(PRISM_ERR_ARG, "null handle");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        PRISM_CUDA(cudaStreamSynchronize(h->stream));
        if (h->own_stream) PRISM_CUDA(cudaStreamDestroy(h->stream));
        h->own_stream = false;
        h->stream = static_cast<cudaStream_t>(stream);
        return PRISM_OK;
    });
}

int32_t prism_dims(prism_handle h, uint32_t* n, uint64_t* nnz) {
    if (!h) return fail(PRISM_ERR_ARG, "null handle");
    if (n) *n = h->A.n;
    if (nnz) *nnz = h->A.nnz;
    return PRISM_OK;
}

int32_t prism_spmv_device(prism_handle h, const double* x_d, double* y_d) {
    if (!h) return fail(PRISM_ERR_ARG, "null handle");
    if (!x_d || !y_d) return fail(PRISM_ERR_ARG, "null vector");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        h->spmv(x_d, y_d);
        PRISM_CUDA(cudaStreamSynchronize(h->stream));
        return PRISM_OK;
    });
}

int32_t prism_spmv_shape(prism_handle h, int32_t* lanes_per_row, int32_t* rows_per_pass) {
    if (!h || !lanes_per_row || !rows_per_pass) return fail(PRISM_ERR_ARG, "null handle or output");
    int g = 0, u = 0;
    h->spmv_shape_of(&g, &u);
    *lanes_per_row = g;
    *rows_per_pass = u;
    return PRISM_OK;
}

int32_t prism_spmv(prism_handle h, const double* x, double* y) {
    if (!h) return fail(PRISM_ERR_ARG, "null handle");
    if (!x || !y) return fail(PRISM_ERR_ARG, "null vector");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        const uint32_t n = h->A.n;
        if (h->xb.size() < n) { h->xb.alloc(n); h->bb.alloc(n); }
        PRISM_CUDA(cudaMemcpyAsync(h->xb.get(), x, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        h->spmv(h->xb.get(), h->bb.get());
        PRISM_CUDA(cudaMemcpyAsync(y, h->bb.get(), n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        PRISM_CUDA(cudaStreamSynchronize(h->stream));
        return PRISM_OK;
    });
}

// ---- preconditioners --------------------------------------------------------
int32_t prism_set_precond_none(prism_handle h) {
    if (!h) return fail(PRISM_ERR_ARG, "null handle");
    h->P.reset();
    return PRISM_OK;
}

int32_t prism_set_precond_ic(prism_handle h, double threshold, int32_t precision) {
    return set_tri(h, PRISM_PRECOND_IC, threshold, 0, precision);
}

int32_t prism_set_precond_ildlt(prism_handle h, double tol, int32_t precision) {
    return set_tri(h, PRISM_PRECOND_ILDLT, tol, 0, precision);
}

int32_t prism_set_precond_ilut(prism_handle h, uint32_t lfill, double tol, int32_t precision) {
    return set_tri(h, PRISM_PRECOND_ILUT, tol, lfill, precision);
}

int32_t prism_set_precond_factor(prism_handle h, prism_factor f) {
    if (!h || !f) return fail(PRISM_ERR_ARG, "null argument");
    const uint32_t fn = f->f ? f->f->f0.n : (f->amsed->fp32 ? f->amsed->s32->n : f->amsed->s64->n);
    if (fn != h->A.n) return fail(PRISM_ERR_ARG, "factor dimension does not match the operator");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        h->P.reset();
        if (f->f) h->P = std::make_unique<prism::TriangularPrecond>(*h, f->f);
        else h->P = std::make_unique<prism::AmsedPrecond>(*h, f->amsed);
        return PRISM_OK;
    });
}

void prism_amsed_default_opts(prism_amsed_opts* o) {
    if (!o) return;
    prism::AmsedOptions a;
    o->levels = a.levels;
    o->lanczos_steps = a.lanczos_steps;
    o->low_rank = a.low_rank;
    o->eig_bound = a.eig_bound;
    o->lowrank_type = a.lowrank_type;
    o->lanczos_type = a.lanczos_type;
    o->reorder = a.reorder;
    o->factor_tol = a.factor_tol;
    o->minsep = a.minsep;
    o->seed = a.seed;
}

int32_t prism_set_precond_amsed(prism_handle h, const prism_amsed_opts* o, int32_t precision) {
    if (!h || !o) return fail(PRISM_ERR_ARG, "null argument");
    if (!valid_precision(precision)) return fail(PRISM_ERR_ARG, "bad precision");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        h->P.reset();
        int rc = 0;
        std::string err;
        auto a = build_amsed(h->A_host, o, precision, &rc, &err);
        if (rc) return fail(rc, err);
        h->P = std::make_unique<prism::AmsedPrecond>(*h, a);
        return PRISM_OK;
    });
}

void prism_gmslr_default_opts(prism_amsed_opts* o) {
    if (!o) return;
    prism_amsed_default_opts(o);
    o->lanczos_steps = 20;  // GMSLR_MSTEPS
    o->low_rank = 12;       // GMSLR_RANK
    o->factor_tol = 1e-2;   // GMSLR_FACTOR_TOLRANCE (ILUT lfill is GMSLR_LFILL = 20)
    o->lowrank_type = 0;
}

int32_t prism_set_precond_gmslr(prism_handle h, const prism_amsed_opts* o, int32_t precision) {
    if (!h || !o) return fail(PRISM_ERR_ARG, "null argument");
    if (!valid_precision(precision)) return fail(PRISM_ERR_ARG, "bad precision");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        h->P.reset();
        int rc = 0;
        std::string err;
        auto a = build_amsed(h->A_host, o, precision, &rc, &err, 4);
        if (rc) return fail(rc, err);
        h->P = std::make_unique<prism::AmsedPrecond>(*h, a);
        return PRISM_OK;
    });
}

int32_t prism_factor_create_gmslr(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
                                  const prism_amsed_opts* o, int32_t precision, prism_factor* out) {
    if (!out || !o) return fail(PRISM_ERR_ARG, "null argument");
    *out = nullptr;
    if (n == 0 || !rowptr || !col || !val) return fail(PRISM_ERR_ARG, "empty or null CSR");
    if (!valid_precision(precision)) return fail(PRISM_ERR_ARG, "bad precision");
    std::string bad = prism::validate_csr(n, rowptr, col);
    if (!bad.empty()) return fail(PRISM_ERR_BAD_MATRIX, bad);
    return guarded([&]() -> int {
        prism::CsrHost A;
        A.n = n;
        A.rowptr.assign(rowptr, rowptr + n + 1);
        A.col.assign(col, col + rowptr[n]);
        A.val.assign(val, val + rowptr[n]);
        int rc = 0;
        std::string err;
        auto a = build_amsed(A, o, precision, &rc, &err, 4);
        if (rc) return fail(rc, err);
        *out = new prism_factor_s{nullptr, std::move(a)};
        return PRISM_OK;
    });
}

int32_t prism_factor_create_amsed(uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
                                  const prism_amsed_opts* o, int32_t precision, prism_factor* out) {
    if (!out || !o) return fail(PRISM_ERR_ARG, "null argument");
    *out = nullptr;
    if (n == 0 || !rowptr || !col || !val) return fail(PRISM_ERR_ARG, "empty or null CSR");
    if (!valid_precision(precision)) return fail(PRISM_ERR_ARG, "bad precision");
    std::string bad = prism::validate_csr(n, rowptr, col);
    if (!bad.empty()) return fail(PRISM_ERR_BAD_MATRIX, bad);
    return guarded([&]() -> int {
        prism::CsrHost A;
        A.n = n;
        A.rowptr.assign(rowptr, rowptr + n + 1);
        A.col.assign(col, col + rowptr[n]);
        A.val.assign(val, val + rowptr[n]);
        int rc = 0;
        std::string err;
        auto a = build_amsed(A, o, precision, &rc, &err);
        if (rc) return fail(rc, err);
        *out = new prism_factor_s{nullptr, std::move(a)};
        return PRISM_OK;
    });
}

// ---- AMSED structure export (parity checks) -------------------------------------
}  // extern "C"

template <typename F>
static int32_t with_amsed(prism_factor f, F&& fn) {
    if (!f || !f->amsed) return fail(PRISM_ERR_ARG, "not an AMSED factor");
    return guarded([&]() -> int {
        if (f->amsed->fp32) return fn(*f->amsed->s32);
        return fn(*f->amsed->s64);
    });
}

extern "C" {

int32_t prism_amsed_info(prism_factor f, uint32_t* nlev, uint32_t* lev_ptr, uint32_t* ncomps, uint32_t* ranks,
                         uint64_t* mnnz) {
    return with_amsed(f, [&](const auto& S) -> int {
        if (nlev) *nlev = S.nlev;
        if (mnnz) *mnnz = S.mnnz;
        for (uint32_t l = 0; l < S.nlev; ++l) {
            if (ncomps) ncomps[l] = S.levels[l].ncomps;
            if (ranks) ranks[l] = S.levels[l].rank_reported;
        }
        if (lev_ptr) std::memcpy(lev_ptr, S.lev_ptr.data(), S.lev_ptr.size() * sizeof(uint32_t));
        return PRISM_OK;
    });
}

int32_t prism_amsed_perm(prism_factor f, uint32_t* pperm) {
    if (!pperm) return fail(PRISM_ERR_ARG, "null output");
    return with_amsed(f, [&](const auto& S) -> int {
        std::memcpy(pperm, S.pperm.data(), S.pperm.size() * sizeof(uint32_t));
        return PRISM_OK;
    });
}

int32_t prism_amsed_dom_ptr(prism_factor f, int32_t level, uint32_t* dom_ptr) {
    if (!dom_ptr) return fail(PRISM_ERR_ARG, "null output");
    return with_amsed(f, [&](const auto& S) -> int {
        if (level < 0 || (uint32_t)level >= S.nlev) return fail(PRISM_ERR_ARG, "level out of range");
        const auto& d = S.levels[level].dom_ptr;
        std::memcpy(dom_ptr, d.data(), d.size() * sizeof(uint32_t));
        return PRISM_OK;
    });
}

int32_t prism_amsed_block(prism_factor f, int32_t level, int32_t block, uint32_t* n, uint64_t* nnz,
                          uint32_t* rowptr, uint32_t* col, double* val, double* diag) {
    return with_amsed(f, [&](const auto& S) -> int {
        if (level < 0 || (uint32_t)level >= S.nlev) return fail(PRISM_ERR_ARG, "level out of range");
        const auto& L = S.levels[level];
        if (block < 0 || (size_t)block >= L.Lt.size()) return fail(PRISM_ERR_ARG, "block out of range");
        const auto& F = L.Lt[block];
        if (n) *n = F.n;
        if (nnz) *nnz = F.nnz();
        if (rowptr) std::memcpy(rowptr, F.rowptr.data(), F.rowptr.size() * sizeof(uint32_t));
        if (col) std::memcpy(col, F.col.data(), F.col.size() * sizeof(uint32_t));
        if (val)
            for (size_t k = 0; k < F.val.size(); ++k) val[k] = (double)F.val[k];
        if (diag && block < (int32_t)L.D.size() && !L.D[block].empty())
            std::memcpy(diag, L.D[block].data(), L.D[block].size() * sizeof(double));
        return PRISM_OK;
    });
}

int32_t prism_amsed_coupling(prism_factor f, int32_t level, int32_t which, uint32_t* nrows, uint64_t* nnz,
                             uint32_t* rowptr, uint32_t* col, double* val) {
    return with_amsed(f, [&](const auto& S) -> int {
        if (level < 0 || (uint32_t)level + 1 >= S.nlev) return fail(PRISM_ERR_ARG, "level has no coupling block");
        const prism::CsrHost& M = which == 0 ? S.levels[level].E : (which == 1 ? S.levels[level].C : S.levels[level].F);
        if (nrows) *nrows = M.n;
        if (nnz) *nnz = M.nnz();
        if (rowptr) std::memcpy(rowptr, M.rowptr.data(), M.rowptr.size() * sizeof(uint32_t));
        if (col) std::memcpy(col, M.col.data(), M.col.size() * sizeof(uint32_t));
        if (val) std::memcpy(val, M.val.data(), M.val.size() * sizeof(double));
        return PRISM_OK;
    });
}

int32_t prism_gmslr_block(prism_factor f, int32_t level, int32_t block, int32_t which, uint32_t* n, uint64_t* nnz,
                          uint32_t* rowptr, uint32_t* col, double* val, double* dinv) {
    return with_amsed(f, [&](const auto& S) -> int {
        if (level < 0 || (uint32_t)level >= S.nlev) return fail(PRISM_ERR_ARG, "level out of range");
        const auto& L = S.levels[level];
        if (L.U.empty()) return fail(PRISM_ERR_ARG, "not a GMSLR factor");
        if (block < 0 || (size_t)block >= L.U.size()) return fail(PRISM_ERR_ARG, "block out of range");
        const auto& F = which == 0 ? L.Lt[block] : L.U[block];
        if (n) *n = F.n;
        if (nnz) *nnz = F.nnz();
        if (rowptr) std::memcpy(rowptr, F.rowptr.data(), F.rowptr.size() * sizeof(uint32_t));
        if (col) std::memcpy(col, F.col.data(), F.col.size() * sizeof(uint32_t));
        if (val)
            for (size_t k = 0; k < F.val.size(); ++k) val[k] = (double)F.val[k];
        if (dinv)
            for (size_t k = 0; k < L.Dinv[block].size(); ++k) dinv[k] = (double)L.Dinv[block][k];
        return PRISM_OK;
    });
}

int32_t prism_amsed_lowrank(prism_factor f, int32_t level, uint32_t* rank, uint32_t* nrem, double* W, double* H) {
    return with_amsed(f, [&](const auto& S) -> int {
        if (level < 0 || (uint32_t)level >= S.nlev) return fail(PRISM_ERR_ARG, "level out of range");
        const auto& L = S.levels[level];
        if (rank) *rank = L.rank;
        if (nrem) *nrem = S.n - S.lev_ptr[level + 1];
        if (W) std::memcpy(W, L.W.data(), L.W.size() * sizeof(double));
        if (H) std::memcpy(H, L.H.data(), L.H.size() * sizeof(double));
        return PRISM_OK;
    });
}

// ---- host-only factors ------------------------------------------------------------
int32_t prism_factor_create(int32_t kind, uint32_t n, const uint32_t* rowptr, const uint32_t* col, const double* val,
                            double tol, uint32_t lfill, int32_t precision, prism_factor* out) {
    if (!out) return fail(PRISM_ERR_ARG, "null output");
    *out = nullptr;
    if (n == 0 || !rowptr || !col || !val) return fail(PRISM_ERR_ARG, "empty or null CSR");
    if (kind != PRISM_PRECOND_IC && kind != PRISM_PRECOND_ILUT && kind != PRISM_PRECOND_ILDLT)
        return fail(PRISM_ERR_UNSUPPORTED, "kind must be IC, ILUT or ILDLT");
    if (!valid_precision(precision)) return fail(PRISM_ERR_ARG, "bad precision");
    std::string bad = prism::validate_csr(n, rowptr, col);
    if (!bad.empty()) return fail(PRISM_ERR_BAD_MATRIX, bad);
    return guarded([&]() -> int {
        prism::CsrHost A;
        A.n = n;
        A.rowptr.assign(rowptr, rowptr + n + 1);
        A.col.assign(col, col + rowptr[n]);
        A.val.assign(val, val + rowptr[n]);
        auto f = std::make_shared<prism::HostFactor>();
        std::string err;
        int rc = prism::build_triangular(kind, A, tol, lfill, precision != PRISM_FP64, *f, &err);
        if (rc) return fail(rc, err);
        f->apply32 = precision == PRISM_FP32_APPLY;
        *out = new prism_factor_s{std::move(f), nullptr};
        return PRISM_OK;
    });
}

int32_t prism_factor_destroy(prism_factor f) {
    delete f;
    return PRISM_OK;
}

int32_t prism_factor_get(prism_factor f, int32_t which, uint32_t* n, uint64_t* nnz, uint32_t* rowptr, uint32_t* col,
                         double* val, double* diag) {
    if (!f || !f->f) return fail(PRISM_ERR_ARG, "null or non-triangular factor");
    int rc = prism::export_host_factor(*f->f, which, n, nnz, rowptr, col, val, diag);
    if (rc) return fail(rc, "which must be 0 (or 1 for ILUT)");
    return PRISM_OK;
}

int32_t prism_factor_info(prism_factor f, uint64_t* mnnz, uint32_t* lower_levels, uint32_t* upper_levels) {
    if (!f) return fail(PRISM_ERR_ARG, "null factor");
    if (f->amsed) {
        if (mnnz) *mnnz = f->amsed->fp32 ? f->amsed->s32->mnnz : f->amsed->s64->mnnz;
        if (lower_levels) *lower_levels = 0;
        if (upper_levels) *upper_levels = 0;
        return PRISM_OK;
    }
    const prism::HostFactor& F = *f->f;
    if (mnnz) *mnnz = F.mnnz;
    if (lower_levels) *lower_levels = F.fp32 ? F.lower32.num_levels : F.lower64.num_levels;
    if (upper_levels) *upper_levels = F.fp32 ? F.upper32.num_levels : F.upper64.num_levels;
    return PRISM_OK;
}

int32_t prism_precond_nnz(prism_handle h, uint64_t* mnnz) {
    if (!h || !mnnz) return fail(PRISM_ERR_ARG, "null argument");
    if (!h->P) return fail(PRISM_ERR_NOT_READY, "no preconditioner set");
    *mnnz = h->P->mnnz();
    return PRISM_OK;
}

int32_t prism_precond_type(prism_handle h, int32_t* kind) {
    if (!h || !kind) return fail(PRISM_ERR_ARG, "null argument");
    *kind = h->P ? h->P->kind() : PRISM_PRECOND_NONE;
    return PRISM_OK;
}

int32_t prism_precond_factor(prism_handle h, int32_t which, uint32_t* n, uint64_t* nnz, uint32_t* rowptr,
                             uint32_t* col, double* val, double* diag) {
    if (!h) return fail(PRISM_ERR_ARG, "null handle");
    if (!h->P) return fail(PRISM_ERR_NOT_READY, "no preconditioner set");
    int rc = h->P->export_factor(which, n, nnz, rowptr, col, val, diag);
    if (rc) return fail(rc, "factor export not available for this preconditioner/which");
    return PRISM_OK;
}

int32_t prism_precond_levels(prism_handle h, int32_t sweep, uint32_t* num_levels) {
    if (!h || !num_levels) return fail(PRISM_ERR_ARG, "null argument");
    if (!h->P) return fail(PRISM_ERR_NOT_READY, "no preconditioner set");
    *num_levels = h->P->levels(sweep);
    return PRISM_OK;
}

int32_t prism_apply_device(prism_handle h, const double* in_d, double* out_d) {
    if (!h) return fail(PRISM_ERR_ARG, "null handle");
    if (!in_d || !out_d) return fail(PRISM_ERR_ARG, "null vector");
    if (!h->P) return fail(PRISM_ERR_NOT_READY, "no preconditioner set");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        h->P->apply(h->stream, in_d, out_d);
        h->check_status();
        return PRISM_OK;
    });
}

int32_t prism_apply(prism_handle h, const double* in, double* out) {
    if (!h) return fail(PRISM_ERR_ARG, "null handle");
    if (!in || !out) return fail(PRISM_ERR_ARG, "null vector");
    if (!h->P) return fail(PRISM_ERR_NOT_READY, "no preconditioner set");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        const uint32_t n = h->A.n;
        if (h->xb.size() < n) { h->xb.alloc(n); h->bb.alloc(n); }
        PRISM_CUDA(cudaMemcpyAsync(h->bb.get(), in, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        h->P->apply(h->stream, h->bb.get(), h->xb.get());
        PRISM_CUDA(cudaMemcpyAsync(out, h->xb.get(), n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        h->check_status();
        return PRISM_OK;
    });
}

int32_t prism_precond_sweep_device(prism_handle h, int32_t sweep, const double* in_d, double* out_d,
                                   int32_t prepare) {
    if (!h || !in_d || !out_d) return fail(PRISM_ERR_ARG, "null argument");
    if (sweep < 0) return fail(PRISM_ERR_ARG, "sweep must be >= 0");
    if (in_d == out_d) return fail(PRISM_ERR_ARG, "a sweep cannot run in place");
    if (!h->P) return fail(PRISM_ERR_NOT_READY, "no preconditioner set");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        if (prepare < 0 || prepare > 2) return fail(PRISM_ERR_ARG, "prepare must be 0, 1 or 2");
        if (!h->P->run_sweep(h->stream, sweep, in_d, out_d, prepare))
            return fail(PRISM_ERR_ARG, "no such sweep for this preconditioner");
        return PRISM_OK;
    });
}

int32_t prism_precond_sweep_info(prism_handle h, int32_t sweep, uint32_t* n, uint64_t* nnz, uint32_t* value_bytes,
                                 uint32_t* num_levels, uint32_t* kernel) {
    if (!h) return fail(PRISM_ERR_ARG, "null handle");
    if (!h->P) return fail(PRISM_ERR_NOT_READY, "no preconditioner set");
    if (!h->P->sweep_info(sweep, n, nnz, value_bytes, num_levels, kernel))
        return fail(PRISM_ERR_UNSUPPORTED, "preconditioner has no single sweeps");
    return PRISM_OK;
}

// ---- solvers -------------------------------------------------------------------
// xref: device pointer of the reference solution (or null)
static void run_solver(prism::Handle& h, const prism_solve_opts& o, const double* b, double* x,
                       prism_solve_stats* st, const double* xref) {
    if (o.solver == PRISM_SOLVER_FCG || o.solver == PRISM_SOLVER_CG) prism::fcg_solve(h, o, b, x, st);
    else prism::gmres_solve(h, o, b, x, st);
    if (st) st->forward_error = xref ? prism::forward_error(h, x, xref) : -1.0;
}

static int check_opts(prism_handle h, const prism_solve_opts* o) {
    if (!h) return fail(PRISM_ERR_ARG, "null handle");
    if (!o) return fail(PRISM_ERR_ARG, "null options");
    if (!(o->tol > 0.0)) return fail(PRISM_ERR_ARG, "tol must be > 0");
    if (o->solver < PRISM_SOLVER_FCG || o->solver > PRISM_SOLVER_GMRES) return fail(PRISM_ERR_ARG, "unknown solver kind");
    if ((o->solver == PRISM_SOLVER_FGMRES || o->solver == PRISM_SOLVER_GMRES) && o->restart + 2 > prism::Handle::kMaxKrylov)
        return fail(PRISM_ERR_ARG, "restart length above the Krylov workspace limit (1022)");
    return PRISM_OK;
}

int32_t prism_solve_device(prism_handle h, const prism_solve_opts* opts, const double* b_d, double* x_d,
                           prism_solve_stats* stats) {
    int rc = check_opts(h, opts);
    if (rc) return rc;
    if (!b_d || !x_d) return fail(PRISM_ERR_ARG, "null vector");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        run_solver(*h, *opts, b_d, x_d, stats, opts->x_ref);
        return PRISM_OK;
    });
}

int32_t prism_solve(prism_handle h, const prism_solve_opts* opts, const double* b, double* x,
                    prism_solve_stats* stats) {
    int rc = check_opts(h, opts);
    if (rc) return rc;
    if (!b || !x) return fail(PRISM_ERR_ARG, "null vector");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        const uint32_t n = h->A.n;
        if (h->xb.size() < n) { h->xb.alloc(n); h->bb.alloc(n); }
        PRISM_CUDA(cudaMemcpyAsync(h->bb.get(), b, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        PRISM_CUDA(cudaMemcpyAsync(h->xb.get(), x, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        const double* xref = nullptr;
        if (opts->x_ref) {
            if (h->xr.size() < n) h->xr.alloc(n);
            PRISM_CUDA(cudaMemcpyAsync(h->xr.get(), opts->x_ref, n * sizeof(double), cudaMemcpyHostToDevice,
                                       h->stream));
            xref = h->xr.get();
        }
        run_solver(*h, *opts, h->bb.get(), h->xb.get(), stats, xref);
        PRISM_CUDA(cudaMemcpyAsync(x, h->xb.get(), n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        PRISM_CUDA(cudaStreamSynchronize(h->stream));
        return PRISM_OK;
    });
}


int32_t prism_update_values(prism_handle h, const double* val) {
    if (!h) return fail(PRISM_ERR_ARG, "null handle");
    if (!val) return fail(PRISM_ERR_ARG, "null values");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        const size_t nnz = h->A.nnz;
        std::memcpy(h->A_host.val.data(), val, nnz * sizeof(double));
        PRISM_CUDA(cudaMemcpyAsync(h->A.val.get(), val, nnz * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        PRISM_CUDA(cudaStreamSynchronize(h->stream));
        h->symmetric = -1;
        return PRISM_OK;
    });
}

int32_t prism_update_values_device(prism_handle h, const double* val_d) {
    if (!h) return fail(PRISM_ERR_ARG, "null handle");
    if (!val_d) return fail(PRISM_ERR_ARG, "null values");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        const size_t nnz = h->A.nnz;
        PRISM_CUDA(cudaMemcpyAsync(h->A.val.get(), val_d, nnz * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        PRISM_CUDA(cudaMemcpyAsync(h->A_host.val.data(), val_d, nnz * sizeof(double), cudaMemcpyDeviceToHost,
                                   h->stream));
        PRISM_CUDA(cudaStreamSynchronize(h->stream));
        h->symmetric = -1;
        return PRISM_OK;
    });
}

int32_t prism_refactor(prism_handle h) {
    if (!h) return fail(PRISM_ERR_ARG, "null handle");
    if (!h->P) return fail(PRISM_ERR_NOT_READY, "no preconditioner set");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        h->P->refactor();
        return PRISM_OK;
    });
}

static void adjoint(prism::Handle& h, const prism_solve_opts& o, const double* g_d, const double* x_d,
                    double* lambda_d, double* grad_d, prism_solve_stats* st) {
    if (h.symmetric < 0) h.symmetric = prism::csr_symmetric(h.A_host) ? 1 : 0;
    if (!h.symmetric)
        throw prism::Error(PRISM_ERR_UNSUPPORTED, "adjoint solve needs A == A^T (a nonsymmetric A needs a "
                                                  "transposed operator and preconditioner)");
    // A^T = A: lambda = A^{-1} g with the handle's own solver and preconditioner, from zero
    PRISM_CUDA(cudaMemsetAsync(lambda_d, 0, (size_t)h.A.n * sizeof(double), h.stream));
    run_solver(h, o, g_d, lambda_d, st, nullptr);  // no reference solution for lambda
    if (grad_d) prism::launch_adjoint_outer(h, h.stream, lambda_d, x_d, grad_d);
    PRISM_CUDA(cudaStreamSynchronize(h.stream));
}

int32_t prism_adjoint_solve_device(prism_handle h, const prism_solve_opts* opts, const double* g_d, const double* x_d,
                                   double* lambda_d, double* grad_val_d, prism_solve_stats* stats) {
    int rc = check_opts(h, opts);
    if (rc) return rc;
    if (!g_d || !lambda_d) return fail(PRISM_ERR_ARG, "null vector");
    if (grad_val_d && !x_d) return fail(PRISM_ERR_ARG, "the pattern gradient needs x");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        adjoint(*h, *opts, g_d, x_d, lambda_d, grad_val_d, stats);
        return PRISM_OK;
    });
}

int32_t prism_adjoint_solve(prism_handle h, const prism_solve_opts* opts, const double* g, const double* x,
                            double* lambda, double* grad_val, prism_solve_stats* stats) {
    int rc = check_opts(h, opts);
    if (rc) return rc;
    if (!g || !lambda) return fail(PRISM_ERR_ARG, "null vector");
    if (grad_val && !x) return fail(PRISM_ERR_ARG, "the pattern gradient needs x");
    return guarded([&]() -> int {
        DeviceGuard gd(h->info.device);
        const uint32_t n = h->A.n;
        const size_t nnz = h->A.nnz;
        prism::DevBuf<double> gd_(n), xd(n), ld(n), vd(grad_val ? nnz : 1);
        PRISM_CUDA(cudaMemcpyAsync(gd_.get(), g, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        if (x) PRISM_CUDA(cudaMemcpyAsync(xd.get(), x, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        adjoint(*h, *opts, gd_.get(), xd.get(), ld.get(), grad_val ? vd.get() : nullptr, stats);
        PRISM_CUDA(cudaMemcpyAsync(lambda, ld.get(), n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        if (grad_val)
            PRISM_CUDA(cudaMemcpyAsync(grad_val, vd.get(), nnz * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        PRISM_CUDA(cudaStreamSynchronize(h->stream));
        return PRISM_OK;
    });
}

static int check_block(prism_handle h, uint32_t k, uint64_t ld) {
    if (!h) return fail(PRISM_ERR_ARG, "null handle");
    if (k == 0 || k > 64) return fail(PRISM_ERR_ARG, "block of right-hand sides: k must be in 1..64");
    if (k > 1 && ld < h->A.n) return fail(PRISM_ERR_ARG, "leading dimension below n");
    return PRISM_OK;
}

int32_t prism_apply_batched_device(prism_handle h, uint32_t k, const double* in_d, double* out_d, uint64_t ld) {
    int rc = check_block(h, k, ld);
    if (rc) return rc;
    if (!in_d || !out_d) return fail(PRISM_ERR_ARG, "null block");
    if (in_d == out_d) return fail(PRISM_ERR_ARG, "block apply needs distinct input and output");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        prism::batched_apply(*h, k, in_d, out_d, k > 1 ? ld : h->A.n);
        PRISM_CUDA(cudaStreamSynchronize(h->stream));
        return PRISM_OK;
    });
}

static int check_block_solver(const prism_solve_opts* o) {
    if (o->solver != PRISM_SOLVER_FCG && o->solver != PRISM_SOLVER_CG)
        return fail(PRISM_ERR_UNSUPPORTED, "blocks of right-hand sides are solved with FCG / CG");
    return PRISM_OK;
}

int32_t prism_solve_batched_device(prism_handle h, const prism_solve_opts* opts, uint32_t k, const double* B_d,
                                   double* X_d, uint64_t ld, prism_solve_stats* stats) {
    int rc = check_opts(h, opts);
    if (!rc) rc = check_block(h, k, ld);
    if (!rc) rc = check_block_solver(opts);
    if (rc) return rc;
    if (!B_d || !X_d) return fail(PRISM_ERR_ARG, "null block");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        prism::batched_fcg_solve(*h, *opts, k, B_d, X_d, k > 1 ? ld : h->A.n, stats);
        return PRISM_OK;
    });
}

int32_t prism_solve_batched(prism_handle h, const prism_solve_opts* opts, uint32_t k, const double* B, double* X,
                            uint64_t ld, prism_solve_stats* stats) {
    int rc = check_opts(h, opts);
    if (!rc) rc = check_block(h, k, ld);
    if (!rc) rc = check_block_solver(opts);
    if (rc) return rc;
    if (!B || !X) return fail(PRISM_ERR_ARG, "null block");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        const uint32_t n = h->A.n;
        const uint64_t l = k > 1 ? ld : n;
        prism::DevBuf<double> Bd((size_t)n * k), Xd((size_t)n * k);
        // column c of the host block starts at c * l; copy the n used rows of each column
        for (uint32_t c = 0; c < k; ++c) {
            PRISM_CUDA(cudaMemcpyAsync(Bd.get() + (size_t)c * n, B + c * l, n * sizeof(double),
                                       cudaMemcpyHostToDevice, h->stream));
            PRISM_CUDA(cudaMemcpyAsync(Xd.get() + (size_t)c * n, X + c * l, n * sizeof(double),
                                       cudaMemcpyHostToDevice, h->stream));
        }
        prism::batched_fcg_solve(*h, *opts, k, Bd.get(), Xd.get(), n, stats);
        for (uint32_t c = 0; c < k; ++c)
            PRISM_CUDA(cudaMemcpyAsync(X + c * l, Xd.get() + (size_t)c * n, n * sizeof(double),
                                       cudaMemcpyDeviceToHost, h->stream));
        PRISM_CUDA(cudaStreamSynchronize(h->stream));
        return PRISM_OK;
    });
}

int32_t prism_solve_segments_device(prism_handle h, const prism_solve_opts* opts, uint32_t nseg,
                                    const uint32_t* seg_ptr, const double* b_d, double* x_d,
                                    prism_solve_stats* stats) {
    int rc = check_opts(h, opts);
    if (!rc) rc = check_block_solver(opts);
    if (rc) return rc;
    if (!seg_ptr || !b_d || !x_d) return fail(PRISM_ERR_ARG, "null argument");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        prism::segmented_fcg_solve(*h, *opts, nseg, seg_ptr, b_d, x_d, stats);
        return PRISM_OK;
    });
}

int32_t prism_solve_segments(prism_handle h, const prism_solve_opts* opts, uint32_t nseg, const uint32_t* seg_ptr,
                             const double* b, double* x, prism_solve_stats* stats) {
    int rc = check_opts(h, opts);
    if (!rc) rc = check_block_solver(opts);
    if (rc) return rc;
    if (!seg_ptr || !b || !x) return fail(PRISM_ERR_ARG, "null argument");
    return guarded([&]() -> int {
        DeviceGuard g(h->info.device);
        const uint32_t n = h->A.n;
        prism::DevBuf<double> bd(n), xd(n);
        PRISM_CUDA(cudaMemcpyAsync(bd.get(), b, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        PRISM_CUDA(cudaMemcpyAsync(xd.get(), x, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        prism::segmented_fcg_solve(*h, *opts, nseg, seg_ptr, bd.get(), xd.get(), stats);
        PRISM_CUDA(cudaMemcpyAsync(x, xd.get(), n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        PRISM_CUDA(cudaStreamSynchronize(h->stream));
        return PRISM_OK;
    });
}

}  // extern "C"
