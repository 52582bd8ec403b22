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
#include <memory>
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

// ---- Matrix Market files (mtx.cpp) -----------------------------------------
// A sparse "coordinate" file as HOST::ReadMtxTools::loadMatrix reads it
// (source/utils/TestTools/ReadMtxTools.cpp): real values (complex files: part
// 0 the real part, part 1 the imaginary part, each with its own pattern),
// near-zero entries dropped, symmetric / skew-symmetric files expanded, rows
// ordered by column.  base: index base of the file (1 for Matrix Market).
int read_mtx(const std::string& path, uint32_t base, int part, uint32_t& rows, uint32_t& cols,
             std::vector<uint32_t>& rowptr, std::vector<uint32_t>& col, std::vector<double>& val, std::string* err);
// A dense "array" file (a right-hand side block): rows x cols values, column-major.
int read_mtx_dense(const std::string& path, uint32_t& rows, uint32_t& cols, std::vector<double>& values,
                   std::string* err);

// Structural validation of a caller CSR: monotone offsets, columns < n and
// strictly increasing inside a row.  Returns an empty string when valid.
std::string validate_csr(uint32_t n, const uint32_t* rowptr, const uint32_t* col);
// true when A equals its transpose exactly (pattern and values); rows sorted
bool csr_symmetric(const CsrHost& A);

// ---- incomplete factorisations ---------------------------------------------
// The operation order of one left-looking factorisation on its own pattern, recorded
// while it runs, so that the factor values can be computed again for new matrix values
// on the same pattern (device numeric refactorisation) with every floating-point
// operation in the same order.  Column j: its accumulator starts from the matrix
// entries a_pos[a_ptr[j] .. a_ptr[j+1]) (positions in A's value array, row j with
// column >= j, in stored order), then subtracts, for each finished column k listed in
// up_k[up_ptr[j] .. up_ptr[j+1]) in that order, L_ik * L_jk (* D_k) over the entries of
// column k from position up_start (L_jk) to its end.
struct RefactorPlan {
    uint32_t n = 0;
    bool ldlt = false;
    std::vector<uint32_t> a_ptr, a_pos;
    std::vector<uint32_t> up_ptr, up_k, up_start;
    uint32_t max_col = 0;  // longest column of the factor, diagonal included
};

// IncompleteCholesky<Low,double>::setup (source/Preconditioner/IncompleteCholesky.cpp:96-246):
// left-looking threshold Cholesky; Lt holds L^T by rows, diagonal first.
template <typename Low>
int ict_factor(const CsrHost& A, double threshold, CsrT<Low>& Lt, std::string* err, RefactorPlan* plan = nullptr);

// IncompleteLDLT<Low,double>::setup (source/Preconditioner/IncompleteLDLT.cpp:39-186):
// unit L^T by rows without the diagonal; D (double) separately.
template <typename Low>
int ildlt_factor(const CsrHost& A, double tol, CsrT<Low>& Lt, std::vector<double>& D, std::string* err,
                 RefactorPlan* plan = nullptr);

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
// per row.  Every value a round reads lives in a shared-memory value slot
// (slot_bytes each: 4 for single-precision arithmetic, else 8): a row of the
// slab gets a slot when it has readers in the slab (its result is written
// there), a row of another slab (a "halo" row) gets one for the rounds that
// read it (a prefetcher copies it there from global memory).  Slots are
// reused once their value's last reader has run.  The first NZ slots (32 for
// 4-byte slots, 16 for 8-byte ones: one per shared-memory bank) hold 0.0 and
// pad short rows.
//
// The dependencies of a row of round r split in two: "late" ones, rows of the
// slab computed in the kStreamLate rounds before r, and "early" ones,
// everything else (rows of earlier rounds and halo rows).  The kernel sums a
// round's early entries while the rounds before it are still being computed,
// so only the late ones (about a quarter of a row's entries on 3D stencils)
// sit on the chain of rounds.  Inside
// each group of rows that one shared-memory wavefront serves (32 rows for
// 4-byte slots, 16 for 8-byte ones) the entries of every row are ordered so
// that, position by position, the rows read slots of distinct banks where the
// pattern allows it (a greedy edge colouring, most constrained row first).
//
// Each round is one 16-byte aligned record; m = rows rounded up to 8,
// Eg / Kg = groups of four early / late entries (the round's longest row, at
// least stream_early_groups / 1):
//
//   fld  [m] x 16 B  4-byte slots: {f32 in, f32 diag, u32 lo, 0};
//                    8-byte slots: {f64 in, f64 diag}
//   lo   [m] x 4 B   8-byte slots only: row - first row of the slab (low 16
//                    bits) | value slot of the row's result << 16 (0xFFFF: no
//                    reader in the slab)
//   es   [Eg][m] x 8 B       early slots, 4 x u16 per row and group
//   ec   [Eg][m] x 4*vb B    their coefficients (vb = bytes of a factor value)
//   ls   [Kg][m] x 8 B       late slots
//   lc   [Kg][m] x 4*vb B    their coefficients
//
// diag holds 1 / diag for the dividing operations.  The sum of row j is
//   P = (c0 + c1) + (c2 + c3),  c_i = fma chains over early positions 4g + i,
//   s = P, then s = fma(coef, x, s) over the late positions in order,
// padding included (slot of value 0.0, coefficient 0), in the slot type's
// arithmetic.  meta[r] = {offset / 16, bytes, nr | Eg << 8 | Kg << 16 |
// has_halo << 24, 0}; the rounds of CTA b are [cta_round[b], cta_round[b+1]);
// round g's halo copies are [halo_ptr[g], halo_ptr[g+1]) of halo_row /
// halo_sw (slot | rounds of the slab to finish first << 16); in_slot[row]
// indexes the row's `in` field in the blob in units of slot_bytes.
#ifdef __CUDACC__
#define PRISM_HD __host__ __device__
#else
#define PRISM_HD
#endif
constexpr uint32_t kRoundRows = 128;
// A dependency of a row of round r is "late" when it is a row of the slab computed in one of
// the kStreamLate rounds before r; every other dependency (rounds <= r - kStreamLate - 1,
// halo rows) is "early" and is summed before round r starts.
constexpr uint32_t kStreamLate = 3;
constexpr uint32_t kNoSlot = 0xFFFFu;
struct RoundRec {
    uint32_t m, fld, lo, es, ec, ls, lc, bytes;
};
PRISM_HD inline uint32_t pad16(uint32_t b) { return (b + 15u) & ~15u; }
// vb: bytes of a factor value (coefficient), ab: bytes of a value slot
PRISM_HD inline RoundRec round_rec(uint32_t nr, uint32_t Eg, uint32_t Kg, uint32_t vb, uint32_t ab) {
    RoundRec r;
    r.m = (nr + 7u) & ~7u;
    r.fld = 0;
    uint32_t o = 16u * r.m;
    r.lo = o;
    if (ab == 8) o += pad16(4u * r.m);
    r.es = o;
    o += 8u * Eg * r.m;
    r.ec = o;
    o += 4u * vb * Eg * r.m;
    r.ls = o;
    o += 8u * Kg * r.m;
    r.lc = o;
    o += 4u * vb * Kg * r.m;
    r.bytes = o;
    return r;
}
PRISM_HD inline uint32_t zero_slots(uint32_t slot_bytes) { return slot_bytes == 4 ? 32u : 16u; }
// Early entry groups the kernel holds in registers: every round is padded to at least this
// many (and to at least one late group), so that the kernel loads a fixed count with
// straight-line code; rows with more entries continue from the record.
PRISM_HD constexpr uint32_t stream_early_groups(uint32_t slot_bytes) { return slot_bytes == 4 ? 7u : 5u; }
struct StreamLayout {
    uint32_t num_ctas = 0, num_rounds = 0, max_round_bytes = 0, max_rounds_per_cta = 0;
    uint32_t slots = 0;                // value slots of the CTA that needs most (zero slots included)
    uint32_t slot_bytes = 8;
    std::vector<uint32_t> slab_start, cta_pos, cta_round, meta, in_slot;
    std::vector<uint32_t> halo_ptr, halo_row, halo_sw;
    std::vector<uint8_t> blob;
};
// The order in which the kernel sums each row (for the oracle): per row of
// the sweep (its own numbering), the early positions then the late ones, each
// a dependency row (0xFFFFFFFF for padding) and its coefficient.
struct StreamOrder {
    std::vector<uint32_t> eptr, edep, kptr, kdep;  // eptr / kptr: n + 1
    std::vector<double> ecoef, kcoef;
    std::vector<double> diag;                      // per row: the sweep's diagonal (as given, not inverted)
    int op = 0;                                    // SweepOp
    bool lower = true;
    // a paired sweep's right-hand side map (see PairMap), empty otherwise
    std::vector<uint32_t> mptr, mdep;
    std::vector<double> mcoef;
};
// Slab boundaries for num_ctas CTAs (num_ctas + 1 entries, empty slabs
// dropped): rows are first split where no dependency crosses (independent
// diagonal blocks, such as the subdomains of an AMSED level, never share a
// slab), CTAs are given to those segments in proportion to their rows, and
// each segment is split evenly.
template <typename Low>
std::vector<uint32_t> slab_ranges(const Sweep<Low>& s, uint32_t num_ctas);
// Builds the records for slabs [start[b], start[b+1]) with slot_bytes-wide
// value slots.  For the dividing operations (SWEEP_DIV, SWEEP_PREDIV) the
// record holds 1 / diag and the kernel multiplies.  Returns false (and why)
// when the sweep does not fit the record format or needs more than max_slots
// value slots in one slab.  `order`, when given, receives the summation order.
// `coef_map`, when given, receives one pair per coefficient written from the sweep:
// (position in the blob in units of the factor value, index of the sweep entry).
// `max_round_bytes` (0: none) ends a round early where its record, with the row
// about to join, could grow beyond that many bytes (rows of many entries).
template <typename Low>
bool stream_layout(const Sweep<Low>& s, const std::vector<uint32_t>& start, uint32_t max_slots, uint32_t slot_bytes,
                   StreamLayout& out, std::string* why, StreamOrder* order = nullptr,
                   std::vector<uint32_t>* coef_map = nullptr, uint32_t max_round_bytes = 0);
// Replays k_sweep_stream on the host, in its arithmetic (float for 4-byte
// slots): stages `in` as the prep kernel does and runs each slab's rounds in
// the kernel's pipeline order -- round r's late entries and round r + 1's
// early ones are read while round r is computed -- with every halo copy made
// as early as its wait allows and every read checked after the writes that
// may race with it.  Checks every offset, that each slot read holds the value
// of the dependency it stands for and that no prefetch waits on its own or a
// later round, and solves the sweep.  Returns an empty string, or what is
// wrong with the layout.
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

// Wavefront pairing: the same triangular solve in half as many wavefronts.  A
// row k on an odd level 2R+1 depends on rows i of level 2R; substituting
// x_i = g_i (b_i - sum_j l_ij x_j) (g_i = 1 / d_i for SWEEP_DIV, d_i for
// SWEEP_MUL, 1 for SWEEP_NONE; for SWEEP_PREDIV x_i = g_i b_i - sum_j l_ij x_j,
// g_i = 1 / d_i) leaves k depending on levels <= 2R-1 only, so that the paired
// sweep's level of every row is half its old one:
//   x_k = op_k(b'_k, sum_j c_kj x_j),  c_kj = l_kj - sum_i l_ki f_i l_ij,
//   b'_k = b_k - sum_i m_ki b_i,
// with f_i = g_i and m_ki = l_ki g_i (DIV, MUL, NONE), or f_i = 1 and
// m_ki = l_ki g_i / g_k (PREDIV).  c is computed in double and stored in the
// sweep's value type; m (double) is applied to the right-hand side before the
// sweep (the streamed kernel's prep): per row r, in stored order,
//   v = b_r;  v = fma(-m, b_dep, v) over [ptr[r], ptr[r+1]).
struct PairMap {
    std::vector<uint32_t> ptr, dep;  // by row (n + 1 / entries)
    std::vector<double> coef;
};
template <typename Low>
void pair_sweep(const Sweep<Low>& s, Sweep<Low>& out, PairMap& m);

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
    std::shared_ptr<const RefactorPlan> plan;  // IC / ILDLT: the factorisation's operation order
};
// The two sweeps of an IC / ILDLT factor's pattern whose values are the indices of the
// factor entries they come from (entries of f0, as doubles); diag holds, per position,
// the index of the diagonal entry (IC) or the row (ILDLT: an index into D).
void factor_index_sweeps(const HostFactor& f, Sweep<double>& lo, Sweep<double>& up);

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
