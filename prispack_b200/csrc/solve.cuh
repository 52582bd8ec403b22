// Device-resident operator, preconditioners and Krylov solvers behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "../../include/prism_solve.h"
#include "device_common.cuh"
#include "host_setup.hpp"
#include "amsed_setup.hpp"

namespace prism {

// Per-device launch geometry, looked up once per handle.
struct DeviceInfo {
    int device = 0;
    int sms = 148;
    int sweep_blocks_per_sm = 1;   // co-resident k_sweep blocks (cooperative launch bound)
    int max_smem_optin = 0;        // bytes of dynamic shared memory one block may opt into
    int sweep_kernel = 0;          // 0: autotune per sweep, 1: global level order, 2: slab-blocked, 3: streamed rounds
    uint32_t slab_min_rows = 2048; // smallest slab (small systems use fewer CTAs)
    uint32_t slab_max_rows = 1u << 30;  // largest slab (default: what shared memory holds)
    uint32_t stream_min_rows = 1024;    // smallest streamed slab (small systems use fewer CTAs)
    int stream_pair = 1;           // where asked: 0 never paired, 1 the tuner decides, 2 paired (pair_sweep)
};

// Reduction scratch shared by all kernels of one stream (they run serially).
struct Reducer {
    DevBuf<double> partial;     // [kMaxGrid * 2]
    DevBuf<unsigned> ticket;    // [1]
    DevBuf<double> scalars;     // [kNumScalars]
    static constexpr int kMaxGrid = 4096;
    ReduceSlot slot(int scalar) const { return ReduceSlot{partial.get(), ticket.get(), scalars.get() + scalar}; }
};

// Scalar slots.
// Sweep operation codes shared with the kernels.

enum Scalar : int {
    SC_BB = 0, SC_RES = 1,   // written together by k_residual: Σ b², Σ (b - y)²
    SC_RR = 2,
    SC_WV = 3,
    SC_DV = 4, SC_DR = 5,    // written together by k_spmv<.,.,2>: Σ v·d, Σ d·r
    SC_TMP = 6, SC_TMP2 = 7,
    SC_DR2 = 8,
    kNumScalars = 16
};

struct DeviceCsr {
    uint32_t n = 0;
    uint64_t nnz = 0;
    DevBuf<uint32_t> rowptr, col;
    DevBuf<double> val;
};

// Device layouts of a triangular sweep.
enum SweepLayout : int { LAYOUT_LEVEL = 0, LAYOUT_SLAB = 1, LAYOUT_STREAM = 2 };

// One triangular sweep resident on the device (see build_sweep for the layout).
// The host part of a streamed upload (pairing, layout, launch shape; no CUDA calls), which
// DevSweep::commit_stream uploads.  ok false: the sweep does not fit the streamed layout.
struct StreamPlan {
    bool ok = false, paired = false, fp32 = false, a32 = false;
    StreamLayout L;
    PairMap pm;
    uint32_t n = 0, num_levels = 0;
    int op = 0;
    uint32_t ctas = 0, ctas_req = 0, slot_bytes = 0, cap = 0, ring = 0, smem = 0;
    uint64_t nnz = 0;
};
template <typename Low>
StreamPlan plan_stream(const Sweep<Low>& sweep, const DeviceInfo& info, bool acc32, bool pair);

struct DevSweep {
    uint32_t n = 0, num_levels = 0;
    int op = SWEEP_NONE;
    bool fp32 = false;
    bool acc32 = false;            // streamed layout: single-precision arithmetic (float values only)
    int layout = LAYOUT_LEVEL;
    // LAYOUT_SLAB (k_sweep_slab): num_ctas > 0
    uint32_t num_ctas = 0, rows_per_cta = 0, smem_rows = 0;
    DevBuf<uint32_t> order, rowptr, col, cta_pos;
    DevBuf<double> val64, diag;
    DevBuf<float> val32;
    // LAYOUT_STREAM (k_sweep_stream): round records, see StreamLayout
    uint32_t str_ctas = 0, str_ring = 0, str_meta_slots = 0, str_slots = 0, str_rounds = 0, str_smem = 0;
    uint64_t str_nnz = 0;
    DevBuf<unsigned char> str_blob;
    DevBuf<uint32_t> str_meta, str_cta_round, str_slab_start, str_in_slot;
    DevBuf<uint32_t> str_halo_ptr, str_halo_row, str_halo_sw;
    uint32_t str_ctas_req = 0, str_slot_bytes = 0;  // what the layout was built with (for its export)
    uint32_t str_round_cap = 0;                     // ... and its record cap (0: none)
    // LAYOUT_STREAM built from the paired sweep (pair_sweep): the right-hand side map the prep
    // applies before the kernel
    bool paired = false;
    DevBuf<uint32_t> pair_ptr, pair_dep;
    DevBuf<double> pair_coef;
    // Uploads the sweep in the given layout; false (nothing uploaded) when the
    // layout does not fit the sweep (stream layout only).  pair: the streamed layout
    // of the paired sweep (half the wavefronts; other layouts ignore it).
    template <typename Low>
    bool upload(const Sweep<Low>& s, const DeviceInfo& info, int layout, cudaStream_t st, bool pair = false);
    void commit_stream(StreamPlan&& plan, cudaStream_t st);
    // the stream layout marks its own output pending; the others need launch_fill first
    bool self_filling() const { return layout == LAYOUT_STREAM; }
    uint64_t entries() const { return layout == LAYOUT_STREAM ? str_nnz : (fp32 ? val32.size() : val64.size()); }
    void release();                // frees the arrays; n = 0 afterwards
    // the summation order of the streamed layout this sweep was uploaded with (s = the same
    // host sweep); false for the other layouts
    template <typename Low>
    bool stream_order(const Sweep<Low>& s, StreamOrder& o) const;
    float tuned_ms = 0.f;          // time of the chosen kernel at setup (0: not tuned)
};

class Precond {
  public:
    Precond();
    virtual ~Precond() = default;
    // distinct for every preconditioner object of the process (never reused), so that work
    // captured from one (a GMRES cycle graph) is never replayed against another
    const uint64_t uid;
    virtual int kind() const = 0;
    virtual uint64_t mnnz() const = 0;
    // out = M^{-1} in; in != out not required.
    virtual void apply(cudaStream_t st, const double* in, double* out) = 0;
    virtual uint32_t levels(int sweep) const { (void)sweep; return 0; }
    // OUT = M^{-1} IN for k <= 64 interleaved columns (X[row * k + c]); in != out.
    virtual void apply_batched(cudaStream_t st, uint32_t k, const double* in, double* out) {
        (void)st; (void)k; (void)in; (void)out;
        throw Error(PRISM_ERR_UNSUPPORTED, "this preconditioner has no block apply");
    }
    // one sweep alone (diagnostics / kernel timing); returns false if not a sweep-based preconditioner
    virtual bool run_sweep(cudaStream_t st, int sweep, const double* in, double* out, int prepare) {
        (void)st; (void)sweep; (void)in; (void)out; (void)prepare;
        return false;
    }
    virtual bool sweep_info(int sweep, uint32_t* n, uint64_t* nnz, uint32_t* vbytes, uint32_t* levels,
                            uint32_t* kernel) const {
        (void)sweep; (void)n; (void)nnz; (void)vbytes; (void)levels; (void)kernel;
        return false;
    }
    // summation order of a streamed sweep (see StreamOrder); false when the sweep runs another kernel
    virtual bool sweep_order(int sweep, StreamOrder& o) const {
        (void)sweep; (void)o;
        return false;
    }
    // numeric refactorisation for the operator's current values on the factor's own pattern
    virtual void refactor() { throw Error(PRISM_ERR_UNSUPPORTED, "this preconditioner has no device refactorisation"); }
    // factor export (parity checks)
    virtual int export_factor(int which, uint32_t* n, uint64_t* nnz, uint32_t* rowptr, uint32_t* col, double* val,
                              double* diag) const {
        (void)which; (void)n; (void)nnz; (void)rowptr; (void)col; (void)val; (void)diag;
        return 9;
    }
};

struct Handle;
struct RefactorState;              // device refactorisation of an IC / ILDLT factor (refactor.cu)
void refactor_release(RefactorState* r);

// IC / ILDLT / ILUT: two sweeps on the device (ILDLT's D^{-1} is folded into
// its upper sweep).  Built from a host factor, which it keeps for export.
class TriangularPrecond : public Precond {
  public:
    TriangularPrecond(Handle& h, std::shared_ptr<const HostFactor> f);
    int kind() const override { return f_->kind; }
    uint64_t mnnz() const override { return f_->mnnz; }
    void apply(cudaStream_t st, const double* in, double* out) override;
    void apply_batched(cudaStream_t st, uint32_t k, const double* in, double* out) override;
    uint32_t levels(int sweep) const override { return sweep == 0 ? lower_.num_levels : upper_.num_levels; }
    int export_factor(int which, uint32_t* n, uint64_t* nnz, uint32_t* rowptr, uint32_t* col, double* val,
                      double* diag) const override;
    bool run_sweep(cudaStream_t st, int sweep, const double* in, double* out, int prepare) override;
    bool sweep_info(int sweep, uint32_t* n, uint64_t* nnz, uint32_t* vbytes, uint32_t* levels,
                    uint32_t* kernel) const override;
    bool sweep_order(int sweep, StreamOrder& o) const override;
    // IC / ILDLT: the factor's values recomputed on the device for the operator's current
    // values (same pattern, the host factorisation's operation order), then written into
    // every device layout of the two sweeps
    void refactor() override;

  private:
    int export_refactored(int which, uint32_t* n, uint64_t* nnz, uint32_t* rowptr, uint32_t* col, double* val,
                          double* diag) const;
    void refresh_level_copy(DevSweep& d, bool lower);
    Handle& h_;
    std::shared_ptr<const HostFactor> f_;
    DevSweep lower_, upper_;
    DevSweep lower_lv_, upper_lv_;   // level-order copies for the block sweeps when the tuner chose slabs
    DevBuf<double> tmp_, tmpk_;
    std::unique_ptr<RefactorState, void (*)(RefactorState*)> rf_{nullptr, refactor_release};
};

// Factor export shared by the device preconditioner and the host-only factor object.
int export_host_factor(const HostFactor& f, int which, uint32_t* n, uint64_t* nnz, uint32_t* rowptr, uint32_t* col,
                       double* val, double* diag);

// Host-built AMSED/MSLR setup, shared by any number of device handles.
struct HostAmsed {
    bool fp32 = false;
    bool apply32 = false;  // single-precision arithmetic in the streamed sweeps
    AmsedOptions opt;
    std::shared_ptr<AmsedSetup<float>> s32;
    std::shared_ptr<AmsedSetup<double>> s64;
};

// AMSED/MSLR apply on the device (amsed.cu).
class AmsedPrecond : public Precond {
  public:
    AmsedPrecond(Handle& h, std::shared_ptr<const HostAmsed> a);
    int kind() const override { return gmslr_ ? PRISM_PRECOND_GMSLR : PRISM_PRECOND_AMSED; }
    uint64_t mnnz() const override;
    void apply(cudaStream_t st, const double* in, double* out) override;
    // k <= 64 interleaved columns: block sweeps per level, k-column couplings, and the
    // low-rank correction as two matrix products (BF16 tensor cores with FP32 factor
    // values, FP64 otherwise); see amsed_block.cuh
    void apply_batched(cudaStream_t st, uint32_t k, const double* in, double* out) override;
    uint32_t levels(int sweep) const override;
    // sweeps are numbered 2*level + (0: lower, 1: upper) over the HID levels
    bool run_sweep(cudaStream_t st, int sweep, const double* in, double* out, int prepare) override;
    bool sweep_info(int sweep, uint32_t* n, uint64_t* nnz, uint32_t* vbytes, uint32_t* levels,
                    uint32_t* kernel) const override;
    bool sweep_order(int sweep, StreamOrder& o) const override;

  private:
    struct Level {
        uint32_t nb = 0, nfac = 0, nrem = 0, rank = 0;
        DevSweep lower, upper;
        DeviceCsr E, Et;   // Et: the downward coupling, E^T (AMSED) or F (GMSLR)
        DevBuf<double> W, H, xc, tmp, tmp2, t;
    };
    template <typename Low>
    void build(const AmsedSetup<Low>& S);
    // the block-diagonal lower / upper sweeps of level l, as build() uploads them
    template <typename Low>
    void level_sweeps(const AmsedSetup<Low>& S, uint32_t l, Sweep<Low>& lo, Sweep<Low>& up) const;
    void block_solve(cudaStream_t st, int level, const double* in, double* out);
    void c_solve(cudaStream_t st, int level, double* x);
    // block apply (built on first use for a given k)
    struct BlockLevel {
        DevSweep lower, upper;            // level-order copies of the level's sweeps
        uint32_t rpad = 0, ldw = 0;       // rank rounded up to 16, rows rounded up to 16
        DevBuf<uint16_t> Wc, Wr;          // BF16 W: column-major rpad x ldw, row-major ldw x rpad
        DevBuf<float> H32;                // [rpad], zero padded
        DevBuf<double> xc, tmp, tmp2;     // nrem x k, nb x k, nb x k
    };
    void prepare_block(uint32_t k);
    void block_solve_k(cudaStream_t st, int level, uint32_t k, const double* in, double* out);
    void c_solve_k(cudaStream_t st, int level, uint32_t k, double* x);
    void lowrank_k(cudaStream_t st, int level, uint32_t k, const double* xc, double* y);
    std::vector<BlockLevel> blv_;
    uint32_t bk_ = 0;                     // columns the block workspace holds
    bool tensor_lowrank_ = false;         // BF16 tensor-core low-rank products (FP32 factor values)
    DevBuf<double> Xk_, sweep_tmpk_, lr_t64_, lr_part64_;
    DevBuf<float> lr_t32_, lr_part32_;
    DevBuf<unsigned> lr_ticket_;
    Handle& h_;
    std::shared_ptr<const HostAmsed> a_;
    bool gmslr_ = false;
    uint32_t n_ = 0, nlev_ = 0;
    std::vector<uint32_t> lev_ptr_;
    DevBuf<uint32_t> pperm_;
    DevBuf<double> X_, sweep_tmp_, partial_;
    std::vector<Level> lv_;
};

struct BatchWork;                  // block-of-RHS workspace (batched.cu)
void batch_release(BatchWork* w);
struct SegWork;                    // batch-of-systems workspace (segments.cu)
void seg_release(SegWork* w);
struct GmresWork;                  // device GMRES scalars and scratch (gmres.cu)
void gmres_release(GmresWork* w);

struct Handle {
    DeviceInfo info;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    CsrHost A_host;
    DeviceCsr A;
    std::unique_ptr<Precond> P;
    Reducer red;
    DevBuf<int> status;            // device status word of the bounded waits
    DevBuf<double> r, w, d, v, y;  // Krylov workspace (n each)
    DevBuf<double> xb, bb, xr;     // host-pointer API staging (xr: reference solution)
    DevBuf<double> V, Z;           // GMRES bases (n x (m+1), column-major)
    double* pinned = nullptr;      // host mirror of scalars (pinned), kScalarCapacity entries
    static constexpr uint32_t kMaxKrylov = 1024;  // restart length limit
    static constexpr uint32_t kScalarCapacity = kNumScalars + kMaxKrylov + 2;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::unique_ptr<BatchWork, void (*)(BatchWork*)> batch{nullptr, batch_release};
    std::unique_ptr<SegWork, void (*)(SegWork*)> seg{nullptr, seg_release};
    std::unique_ptr<GmresWork, void (*)(GmresWork*)> gmres{nullptr, gmres_release};
    int symmetric = -1;            // A == A^T exactly: -1 not yet checked, 0 no, 1 yes

    ~Handle();
    void spmv(const double* x, double* y, int ndot = 0, const double* z = nullptr, const double* q = nullptr,
              int scalar = 0);
    // the shape of A's SpMV kernel (index into the shape table in solve.cu), chosen at
    // creation by timing each shape (tune_spmv) unless PRISM_SPMV_SHAPE names one
    int spmv_shape = 0;
    void tune_spmv();
    void spmv_shape_of(int* lanes_per_row, int* rows_per_pass) const;
    void check_status();           // synchronises; throws on a raised device status
    void ensure_workspace();
};

// ---- launch helpers shared by the preconditioners --------------------------
int vec_grid(const Handle& h, uint32_t n);
// marks n doubles pending (the sweeps' readiness encoding)
void launch_fill(cudaStream_t st, const Handle& h, uint32_t n, double* p);
// One sweep: out = T^{-1} in.  Layouts other than LAYOUT_STREAM need `out`
// marked pending (launch_fill) first; the stream layout does that itself.
void launch_sweep(const Handle& h, cudaStream_t st, const DevSweep& s, const double* in, double* out);
// The two halves of a sweep: marking `out` pending (and, for the stream
// layout, staging `in` into the round records), then the sweep kernel.
void launch_sweep_prepare(const Handle& h, cudaStream_t st, const DevSweep& s, const double* in, double* out);
void launch_sweep_kernel(const Handle& h, cudaStream_t st, const DevSweep& s, const double* in, double* out);
// y = M x (sub = 0) or y -= M x (sub = 1) for a CSR with nrows rows
void launch_spmv(const Handle& h, cudaStream_t st, uint32_t nrows, const uint32_t* rowptr, const uint32_t* col,
                 const double* val, const double* x, double* y, int sub);
// uploads a sweep, choosing its kernel by timing the layouts (see solve.cu);
// acc32 (float values only): single-precision arithmetic, streamed layout only;
// pair: the paired streamed layout (pair_sweep) is one more candidate
template <typename Low>
void tune_sweep(Handle& h, DevSweep& d, const Sweep<Low>& s, bool acc32 = false, bool pair = false);

// grad[k] = -lambda[row(k)] * x[col(k)] over A's stored entries
void launch_adjoint_outer(const Handle& h, cudaStream_t st, const double* lambda, const double* x, double* grad);

// Runs the streamed sweep kernel alone on `device` for sweep s laid out in at most num_ctas
// slabs (the layout's own boundaries), single-precision arithmetic when acc32 (float values);
// host input and output.  The summation order is stream_layout's with the same slabs.
template <typename Low>
void stream_sweep_run(int device, const Sweep<Low>& s, bool acc32, uint32_t num_ctas, const double* in, double* out);
// slabs the streamed layout of an n-row sweep gets when at most num_ctas are wanted
uint32_t stream_slab_count(uint32_t n, uint32_t num_ctas, uint32_t min_rows);

// The AMSED block low-rank correction alone (amsed.cu): Y += W (H o (W^T X)), W column-major
// nrem x rank, X and Y interleaved nrem x k (k <= 64); BF16 tensor cores when tensor, else FP64.
void lowrank_block_run(int device, uint32_t nrem, uint32_t rank, uint32_t k, const double* W, const double* H,
                       const double* X, double* Y, bool tensor);

// Runs the bounded-wait self test (see solve.cu); returns the device status the wait raised.
int selftest_wait_timeout(int device, unsigned long long wait_ns, int* device_status);

// Queries SM count and the co-resident capacity of the sweep kernel.
void init_device_info(DeviceInfo& info, int device);

void fcg_solve(Handle& h, const prism_solve_opts& o, const double* b, double* x, prism_solve_stats* st);
// ||x - xref||_2 / ||xref||_2 (device vectors of the handle's size; synchronises)
double forward_error(Handle& h, const double* x, const double* xref);
void gmres_solve(Handle& h, const prism_solve_opts& o, const double* b, double* x, prism_solve_stats* st);
// blocks of k <= 64 right-hand sides, column-major with leading dimension ld (batched.cu)
void batched_apply(Handle& h, uint32_t k, const double* in_d, double* out_d, uint64_t ld);
void batched_fcg_solve(Handle& h, const prism_solve_opts& o, uint32_t k, const double* B_d, double* X_d, uint64_t ld,
                       prism_solve_stats* st);
// independent systems on the diagonal blocks [seg_ptr[s], seg_ptr[s+1]) of the handle's matrix (segments.cu)
void segmented_fcg_solve(Handle& h, const prism_solve_opts& o, uint32_t nseg, const uint32_t* seg_ptr,
                         const double* b, double* x, prism_solve_stats* st);

}  // namespace prism
