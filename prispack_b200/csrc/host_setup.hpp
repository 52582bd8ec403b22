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
