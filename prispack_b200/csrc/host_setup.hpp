// Host-side setup of the solve phase: model problems, incomplete
// factorisations and the integer level schedules of the triangular sweeps.
//
// The factorisations follow the reference's serial algorithms operation by
// operation (same traversal order, same rounding points, same drop tests), so
// that for the same CSR input they produce the same factor arrays bit for bit
// as HOST::IncompleteCholesky / IncompleteLDLT / IncompleteLU::setup().
// This file must be compiled without FMA contraction (-ffp-contract=off).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace prism {

struct CsrHost {
    uint32_t n = 0;                 // square: n rows, n columns
    std::vector<uint32_t> rowptr;   // n + 1
    std::vector<uint32_t> col;      // nnz
    std::vector<double> val;        // nnz
    uint64_t nnz() const { return rowptr.empty() ? 0 : rowptr[n]; }
};

template <typename V>
struct CsrT {
    uint32_t n = 0;
    std::vector<uint32_t> rowptr;
    std::vector<uint32_t> col;
    std::vector<V> val;
    uint64_t nnz() const { return rowptr.empty() ? 0 : rowptr[n]; }
};

enum SetupStatus : int {
    SETUP_OK = 0,
    SETUP_NOT_SPD = 4,
    SETUP_ZERO_PIVOT = 3,
    SETUP_BAD_INPUT = 1,
};

// ---- model problems --------------------------------------------------------
// generateLaplacianCOO + transCOO2CSR (source/MatrixClass/ModelProblem.cpp:68-133,
// include/MatrixClass/MatrixTools.h:16-62): 5-point (any dim == 1) or 7-point
// stencil, off-diagonals -1 -/+ alpha, diagonal (4 or 6) - shift, rows sorted.
bool laplacian_dims(int32_t nx, int32_t ny, int32_t nz, uint32_t* n, uint32_t* nnz);
void laplacian_fill(int32_t nx, int32_t ny, int32_t nz, double ax, double ay, double az, double shift,
                    uint32_t* rowptr, uint32_t* col, double* val);

// Structural validation of a caller CSR: monotone offsets, columns < n and
// strictly increasing inside a row.  Returns an empty string when valid.
std::string validate_csr(uint32_t n, const uint32_t* rowptr, const uint32_t* col);
// true when A equals its transpose exactly (pattern and values); rows sorted
bool csr_symmetric(const CsrHost& A);

// ---- incomplete factorisations ---------------------------------------------
// IncompleteCholesky<Low,double>::setup (source/Preconditioner/IncompleteCholesky.cpp:96-246):
// left-looking threshold Cholesky; Lt holds L^T by rows, diagonal first.
template <typename Low>
int ict_factor(const CsrHost& A, double threshold, CsrT<Low>& Lt, std::string* err);

// IncompleteLDLT<Low,double>::setup (source/Preconditioner/IncompleteLDLT.cpp:39-186):
// unit L^T by rows without the diagonal; D (double) separately.
template <typename Low>
int ildlt_factor(const CsrHost& A, double tol, CsrT<Low>& Lt, std::vector<double>& D, std::string* err);

// IncompleteLU<Low,double>::setup (source/Preconditioner/IncompleteLU.cpp:38-266):
// Saad's ILUT(lfill, tol); L unit strictly lower, U strictly upper (columns in
// qsplit order, not sorted), Dinv = 1 / pivot in Low precision.
template <typename Low>
int ilut_factor(const CsrHost& A, uint32_t lfill, double tol, CsrT<Low>& L, CsrT<Low>& U,
                std::vector<Low>& Dinv, std::string* err);

// ---- triangular sweeps in gather form ------------------------------------------
// Every preconditioner sweep is rewritten as
//     out[r] = post( pre(in[r]) - sum_k val[k] * out[col[k]] )
// over rows r in dependency order.  `Sweep` holds it with rows renumbered into
// level order (positions), which is the layout the device kernels read.
enum SweepOp : int {
    SWEEP_DIV = 0,      // out = (in - s) / diag           IC lower/upper
    SWEEP_MUL = 1,      // out = (in - s) * diag           ILUT upper (Dinv)
    SWEEP_NONE = 2,     // out = in - s                    unit lower (ILDLT, ILUT)
    SWEEP_PREDIV = 3    // out = in / diag - s             ILDLT upper after D^{-1}
};

template <typename Low>
struct Sweep {
    uint32_t n = 0;
    int op = SWEEP_NONE;
    bool lower = true;                 // dependencies point to smaller rows
    uint32_t num_levels = 0;
    std::vector<uint32_t> level_ptr;   // num_levels + 1, positions
    std::vector<uint32_t> order;       // position -> row
    std::vector<uint32_t> rowptr;      // by position
    std::vector<uint32_t> col;         // dependency rows (original numbering)
    std::vector<Low> val;
    std::vector<double> diag;          // by position (unused for SWEEP_NONE)
    std::vector<uint32_t> level;       // by row: wavefront index
};

// Slab layout of a sweep for the blocked device kernel: CTA b owns the
// contiguous rows [b*rows_per_cta, (b+1)*rows_per_cta) and visits them in
// (level, row) order.  Positions are renumbered so that CTA b's rows occupy
// positions [cta_pos[b], cta_pos[b+1]); rowptr/col/val/diag/order follow.
template <typename Low>
void slab_layout(const Sweep<Low>& s, uint32_t num_ctas, uint32_t rows_per_cta, std::vector<uint32_t>& cta_pos,
                 Sweep<Low>& out);

// Streamed round layout of a sweep (k_sweep_stream).
//
// The rows are cut into slabs of contiguous rows, one per CTA; each slab's
// positions, in (level, row) order, are cut greedily into rounds of at most
// kRoundRows consecutive positions none of which depends on another row of
// the same round, so a CTA can compute a round's rows all at once, one thread
// per row.  Every value a round reads lives in a shared-memory value slot:
// a row of the slab gets a slot when it has readers in the slab (its result
// is written there), a row of another slab (a "halo" row) gets one for the
// rounds that read it (a prefetcher copies it there from global memory).
// Slots are reused once their value's last reader has run; for halo values
// the prefetcher first waits until that round is done (xwait).  Slot 0 holds
// 0.0 and pads short rows.  Each round is one 16-byte aligned record, with
// m = nr rounded up to a multiple of 8 and L = the round's longest row:
//
//   f64 in[m]        right-hand side of each row (written per call)
//   f64 diag[m]      (1 / diag for the dividing operations)
//   u16 lrow[m]      row - first row of the slab
//   u16 oslot[m]     value slot of the row's result (0xFFFF: no reader in the slab)
//   entries          entry k of row j at e = k*m + j: the value slot of the dependency
//                    (0: padding) and its coefficient (0: padding).  Float values:
//                    {u32 slot, f32 value} at ent + 8e, one load.  Double values:
//                    u16 slot at ent + 2e and f64 value at val + 8e (val = ent + 2Lm).
//   u32 xrow[X]      halo rows whose values this round copies in ...
//   u16 xslot[X]     ... into these slots ...
//   u16 xwait[X]     ... once this many rounds of the slab are done
//
// (the halo sections padded to 16 bytes).  meta[r] = {offset / 16, bytes,
// nr | L << 16, X}; the rounds of CTA b are [cta_round[b], cta_round[b+1]);
// in_slot[row] indexes the row's `in` entry in the blob (in doubles).
#ifdef __CUDACC__
#define PRISM_HD __host__ __device__
#else
#define PRISM_HD
#endif
constexpr uint32_t kRoundRows = 128;
constexpr uint32_t kNoSlot = 0xFFFFu;
struct RoundRec {
    uint32_t m, in, diag, lrow, oslot, ent, val, xrow, xslot, xwait, bytes;
};
PRISM_HD inline uint32_t pad16(uint32_t b) { return (b + 15u) & ~15u; }
PRISM_HD inline RoundRec round_rec(uint32_t nr, uint32_t L, uint32_t X, uint32_t vb) {
    RoundRec r;
    r.m = (nr + 7u) & ~7u;
    r.in = 0;
    r.diag = 8u * r.m;
    r.lrow = 16u * r.m;
    r.oslot = 18u * r.m;
    r.ent = 20u * r.m;
    if (vb == 4) {  // {u32 slot, f32 value} pairs
        r.val = r.ent + 4u;
        r.xrow = r.ent + 8u * L * r.m;
    } else {        // u16 slots, then f64 values
        r.val = r.ent + 2u * L * r.m;
        r.xrow = r.val + 8u * L * r.m;
    }
    r.xslot = r.xrow + pad16(4u * X);
    r.xwait = r.xslot + pad16(2u * X);
    r.bytes = r.xwait + pad16(2u * X);
    return r;
}
struct StreamLayout {
    uint32_t num_ctas = 0, num_rounds = 0, max_round_bytes = 0, max_rounds_per_cta = 0;
    uint32_t slots = 0;                // value slots of the CTA that needs most
    std::vector<uint32_t> slab_start, cta_pos, cta_round, meta, in_slot;
    std::vector<uint8_t> blob;
};
// Slab boundaries for num_ctas CTAs (num_ctas + 1 entries, empty slabs
// dropped): rows are first split where no dependency crosses (independent
// diagonal blocks, such as the subdomains of an AMSED level, never share a
// slab), CTAs are given to those segments in proportion to their rows, and
// each segment is split evenly.
template <typename Low>
std::vector<uint32_t> slab_ranges(const Sweep<Low>& s, uint32_t num_ctas);
// Builds the records for slabs [start[b], start[b+1]).  For the dividing
// operations (SWEEP_DIV, SWEEP_PREDIV) the record holds 1 / diag and the
// kernel multiplies.  Returns false (and why) when the sweep does not fit the
// record format or needs more than max_slots value slots in one slab.
template <typename Low>
bool stream_layout(const Sweep<Low>& s, const std::vector<uint32_t>& start, uint32_t max_slots, StreamLayout& out,
                   std::string* why);
// Replays k_sweep_stream on the host: stages `in` as the prep kernel does,
// runs each slab's rounds in order (a round only once the halo rows it copies
// in are finished), checks every offset, that each slot read holds the value
// of the dependency it stands for, that no slot is overwritten before its last
// reader ran and that no prefetch waits on its own or a later round, and
// solves the sweep.  Returns an empty string, or what is wrong with the layout.
template <typename Low>
std::string stream_layout_replay(const Sweep<Low>& s, const StreamLayout& L, const double* in, double* out);

// Builds a sweep from a gather-form CSR (row r lists its dependencies and
// coefficients, in the order the reference accumulates them) plus optional
// per-row diagonal.  Computes the exact integer level schedule:
// level(r) = 1 + max level(dep), and orders positions by (level, row).
template <typename Low>
void build_sweep(uint32_t n, const std::vector<uint32_t>& rowptr, const std::vector<uint32_t>& col,
                 const std::vector<Low>& val, const std::vector<double>* diag, int op, bool lower,
                 Sweep<Low>& out);

// Transpose of a CSR (pattern + values), keeping, inside every output row, the
// increasing order of source rows.  Used to turn the reference's column
// (scatter) solves over L^T into row (gather) solves over L.
template <typename V>
void transpose_csr(uint32_t n, const std::vector<uint32_t>& rowptr, const std::vector<uint32_t>& col,
                   const std::vector<V>& val, std::vector<uint32_t>& trp, std::vector<uint32_t>& tcol,
                   std::vector<V>& tval);

// A complete triangular preconditioner built on the host: the stored factors
// in the reference's layout (widened to double, for export) and the two
// device-layout sweeps.  kind: 1 IC, 2 ILUT, 3 ILDLT (prism_precond_kind).
struct HostFactor {
    int kind = 0;
    bool fp32 = false;
    bool apply32 = false;  // single-precision arithmetic in the streamed sweeps
    uint64_t mnnz = 0;             // getPreconditionNonZeroCount()
    CsrT<double> f0, f1;           // IC/ILDLT: L^T; ILUT: L, U
    std::vector<double> diag;      // ILDLT: D; ILUT: Dinv
    Sweep<double> lower64, upper64;
    Sweep<float> lower32, upper32;
};

// The two device sweeps of an IC factor (L^T with diagonal first) and of an
// ILDLT factor (unit L^T without diagonal, pivots D).
template <typename Low>
void ic_sweeps(const CsrT<Low>& Lt, Sweep<Low>& lo, Sweep<Low>& up);
template <typename Low>
void ildlt_sweeps(const CsrT<Low>& Lt, const std::vector<double>& D, Sweep<Low>& lo, Sweep<Low>& up);

// The two device sweeps of an ILUT factor (unit L, U with inverse pivots).
template <typename Low>
void ilut_sweeps(const CsrT<Low>& L, const CsrT<Low>& U, const std::vector<Low>& Dinv, Sweep<Low>& lo, Sweep<Low>& up);

int build_triangular(int kind, const CsrHost& A, double tol, uint32_t lfill, bool fp32, HostFactor& out,
                     std::string* err);

}  // namespace prism
