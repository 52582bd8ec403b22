// Host setup of the AMSED / MSLR multilevel Schur-complement low-rank
// preconditioner (source/Preconditioner/AMSEDPrecondition.cpp of the
// reference): HID ordering, level structure, per-block incomplete factors,
// and the low-rank correction W H W^T from a generalized Lanczos process.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "host_setup.hpp"

namespace prism {

struct AmsedOptions {
    int32_t family = 5;              // 5: AMSED (ILDLT blocks, ICT last level, Lanczos correction)
                                     // 4: GMSLR (ILUT(20, tol) blocks and last level, F = A(C, B) coupling)
    int32_t levels = 3;              // m_nlev_setup
    int32_t lanczos_steps = 30;      // m_lanczosSteps (AMSED_MSTEPS)
    int32_t low_rank = 16;           // m_lowRankSize (AMSED_RANK); caps the MSLR (basic) rank
    double eig_bound = 0.8;          // m_eigValCorrectBound (AMSED_EIGVAL_CORRECTION)
    int32_t lowrank_type = 1;        // 0: AMSEDBasic (MSLR), 1: AMSEDEigenvalueDeflation
    int32_t lanczos_type = 0;        // 0: UseClassicLanczos (1: restart Lanczos, not provided)
    int32_t reorder = 2;             // 0: MatrixReorderNo, 2: MatrixReorderRCM (1: AMD, not provided)
    double factor_tol = 1e-3;        // AMSED_FACTOR_TOLRANCE
    uint32_t minsep = 3;             // AMSED_MINSEP
    uint64_t seed = 20241116;        // start vector of the Lanczos process
};

// One level of the hierarchy (LevelStructure, include/Preconditioner/AMSEDPrecondition.h:75-85).
template <typename Low>
struct AmsedLevel {
    uint32_t ncomps = 0;
    std::vector<uint32_t> dom_ptr;          // global (permuted) row offsets of the domains, ncomps + 1
    std::vector<CsrHost> B;                 // diagonal blocks, local numbering
    std::vector<CsrT<Low>> Lt;              // per block: ILDLT unit L^T (last level: IC L^T incl. diagonal);
                                            // GMSLR: ILUT L
    std::vector<std::vector<double>> D;     // per block: ILDLT pivots (empty on the last level)
    std::vector<CsrT<Low>> U;               // GMSLR: per block ILUT U
    std::vector<std::vector<Low>> Dinv;     // GMSLR: per block ILUT inverse pivots
    CsrHost E;                              // coupling rows of this level's B x columns of its C block
    CsrHost F;                              // GMSLR: C rows x B columns (GMSLRDPrecondition.cpp:239)
    CsrHost C;                              // the level's C block (for the Lanczos process)
    uint32_t rank = 0;                      // columns of W used by the apply
    uint32_t rank_reported = 0;             // rank the reference reports (GMSLR: W is identically zero)
    std::vector<double> H;                  // rank
    std::vector<double> W;                  // n_remain x rank, column-major
};

template <typename Low>
struct AmsedSetup {
    uint32_t n = 0;
    uint32_t nlev = 0;                      // m_nlev_used
    std::vector<uint32_t> pperm;            // new index -> original index
    std::vector<uint32_t> lev_ptr;          // nlev + 1
    std::vector<AmsedLevel<Low>> levels;
    uint64_t mnnz = 0, incomp_nnz = 0, lowrank_nnz = 0;
    std::vector<int32_t> lanczos_steps_done;  // per level
};

template <typename Low>
int amsed_setup(const CsrHost& A, const AmsedOptions& opt, AmsedSetup<Low>& S, std::string* err);

// Host restatements used by the setup itself (the Lanczos process applies the
// partial preconditioner): x[off : off + size of level's B] <- B_level^{-1} (...)
// and the recursive C_level^{-1} (AMSEDPrecondition.cpp:1494-1754).
template <typename Low>
void amsed_block_solve_host(const AmsedSetup<Low>& S, int level, double* x);
template <typename Low>
void amsed_c_solve_host(const AmsedSetup<Low>& S, int level, double* x, uint32_t len);

// Vendored genrcm (external_packages/RCM/lib/rcm.cpp: genrcm/root_find/rcm/degree/level_set)
// restated: perm[new] = old for the CSR graph including its diagonal.
void rcm_order(uint32_t n, const uint32_t* rowptr, const uint32_t* col, uint32_t* perm);

}  // namespace prism
