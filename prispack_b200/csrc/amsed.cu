// AMSED / MSLR preconditioner apply on the device:
// AMSEDPrecondition::MInvSolve (source/Preconditioner/AMSEDPrecondition.cpp:1976-2087)
// and levelCInvRecursiveSolve (:1494-1587).
//
// Per level the diagonal blocks of all subdomains form one block-diagonal
// factor, so a level's block solve is one lower and one upper sync-free sweep
// over every subdomain at once (the reference runs them as OpenMP tasks,
// :1690-1754).  E^T is stored explicitly so that x2 -= E^T x1 is a gather
// (the reference scatters, CSRMatrix.h:453-486).  The low-rank term
// W (H o (W^T x)) is a multi-dot plus a rank-r update.  The permutation of
// the right-hand side (prepareRightHand / recoverRightHand) brackets the
// recursion.  All scratch is allocated once, at construction.
#include <algorithm>
#include <cstring>

#include "amsed_block.cuh"
#include "amsed_setup.hpp"
#include "kernels.cuh"
#include "solve.cuh"

namespace prism {

namespace {
// CSR transpose for a rectangular nrows x ncols matrix (column order inside
// each output row = increasing source row, i.e. the reference's scatter order)
void transpose_rect(const CsrHost& M, uint32_t ncols, std::vector<uint32_t>& trp, std::vector<uint32_t>& tcol,
                    std::vector<double>& tval) {
    const uint64_t nnz = M.nnz();
    trp.assign((size_t)ncols + 1, 0);
    tcol.resize(nnz);
    tval.resize(nnz);
    for (uint64_t k = 0; k < nnz; ++k) trp[M.col[k] + 1]++;
    for (uint32_t c = 0; c < ncols; ++c) trp[c + 1] += trp[c];
    std::vector<uint32_t> fill(trp.begin(), trp.end() - 1);
    for (uint32_t r = 0; r < M.n; ++r)
        for (uint32_t k = M.rowptr[r]; k < M.rowptr[r + 1]; ++k) {
            const uint32_t c = M.col[k];
            tcol[fill[c]] = r;
            tval[fill[c]] = M.val[k];
            fill[c]++;
        }
}

void upload_csr(DeviceCsr& d, uint32_t nrows, const std::vector<uint32_t>& rp, const std::vector<uint32_t>& ci,
                const std::vector<double>& v, cudaStream_t st) {
    d.n = nrows;
    d.nnz = rp.empty() ? 0 : rp[nrows];
    d.rowptr.upload(rp.data(), rp.size(), st);
    d.col.upload(ci.data(), ci.size(), st);
    d.val.upload(v.data(), v.size(), st);
    if (d.col.size() == 0) d.col.alloc(1);
    if (d.val.size() == 0) d.val.alloc(1);
}
}  // namespace

template <typename Low>
void AmsedPrecond::level_sweeps(const AmsedSetup<Low>& S, uint32_t l, Sweep<Low>& lo, Sweep<Low>& up) const {
    const AmsedLevel<Low>& L = S.levels[l];
    const uint32_t nb = S.lev_ptr[l + 1] - S.lev_ptr[l];
    const uint32_t nfac = l + 1 == nlev_ ? L.B[0].n : nb;  // rows with a factor
    if (gmslr_) {
        // ILUT blocks on every level (the last level: block 0 only, GMSLRDPrecondition.cpp:664-688)
        const uint32_t nblk = l + 1 == nlev_ ? 1 : L.ncomps;
        CsrT<Low> Lc, Uc;
        std::vector<Low> Dc;
        Lc.n = Uc.n = nfac;
        Lc.rowptr.assign((size_t)nfac + 1, 0);
        Uc.rowptr.assign((size_t)nfac + 1, 0);
        for (uint32_t b = 0; b < nblk; ++b) {
            const uint32_t off = L.dom_ptr[b] - L.dom_ptr[0];
            const CsrT<Low>& fl = L.Lt[b];
            const CsrT<Low>& fu = L.U[b];
            for (uint32_t i = 0; i < fl.n; ++i) {
                for (uint32_t k = fl.rowptr[i]; k < fl.rowptr[i + 1]; ++k) {
                    Lc.col.push_back(fl.col[k] + off);
                    Lc.val.push_back(fl.val[k]);
                }
                Lc.rowptr[off + i + 1] = (uint32_t)Lc.col.size();
                for (uint32_t k = fu.rowptr[i]; k < fu.rowptr[i + 1]; ++k) {
                    Uc.col.push_back(fu.col[k] + off);
                    Uc.val.push_back(fu.val[k]);
                }
                Uc.rowptr[off + i + 1] = (uint32_t)Uc.col.size();
            }
            Dc.insert(Dc.end(), L.Dinv[b].begin(), L.Dinv[b].end());
        }
        ilut_sweeps<Low>(Lc, Uc, Dc, lo, up);
    } else if (l + 1 == nlev_) {
        // last level: IC of block 0 (the reference factors and applies only B_mat[0], :694-716, :1504-1508)
        ic_sweeps<Low>(L.Lt[0], lo, up);
    } else {
        // block-diagonal ILDLT of all subdomains of the level
        CsrT<Low> Lt;
        std::vector<double> Dg;
        Lt.n = nb;
        Lt.rowptr.assign((size_t)nb + 1, 0);
        for (uint32_t b = 0; b < L.ncomps; ++b) {
            const uint32_t off = L.dom_ptr[b] - L.dom_ptr[0];
            const CsrT<Low>& f = L.Lt[b];
            for (uint32_t i = 0; i < f.n; ++i) {
                for (uint32_t k = f.rowptr[i]; k < f.rowptr[i + 1]; ++k) {
                    Lt.col.push_back(f.col[k] + off);
                    Lt.val.push_back(f.val[k]);
                }
                Lt.rowptr[off + i + 1] = (uint32_t)Lt.col.size();
            }
            Dg.insert(Dg.end(), L.D[b].begin(), L.D[b].end());
        }
        ildlt_sweeps<Low>(Lt, Dg, lo, up);
    }
}

AmsedPrecond::AmsedPrecond(Handle& h, std::shared_ptr<const HostAmsed> a) : h_(h), a_(std::move(a)) {
    gmslr_ = a_->opt.family == 4;
    if (a_->fp32) build(*a_->s32);
    else build(*a_->s64);
}

uint64_t AmsedPrecond::mnnz() const { return a_->fp32 ? a_->s32->mnnz : a_->s64->mnnz; }

template <typename Low>
void AmsedPrecond::build(const AmsedSetup<Low>& S) {
    cudaStream_t st = h_.stream;
    n_ = S.n;
    nlev_ = S.nlev;
    lev_ptr_ = S.lev_ptr;
    pperm_.upload(S.pperm.data(), S.pperm.size(), st);
    X_.alloc(n_);
    sweep_tmp_.alloc(n_);
    lv_.clear();
    lv_.resize(nlev_);
    uint32_t max_rank = 0;
    for (uint32_t l = 0; l < nlev_; ++l) {
        const AmsedLevel<Low>& L = S.levels[l];
        Level& D = lv_[l];
        D.nb = S.lev_ptr[l + 1] - S.lev_ptr[l];
        D.nrem = S.n - S.lev_ptr[l + 1];
        Sweep<Low> lo, up;
        level_sweeps<Low>(S, l, lo, up);
        D.nfac = l + 1 == nlev_ ? L.B[0].n : D.nb;  // the last level factors block 0 only
        // the streamed kernel may run the level's sweeps paired (half the wavefronts)
        tune_sweep<Low>(h_, D.lower, lo, a_->apply32, true);
        tune_sweep<Low>(h_, D.upper, up, a_->apply32, true);
        if (l + 1 < nlev_) {
            upload_csr(D.E, L.E.n, L.E.rowptr, L.E.col, L.E.val, st);
            if (gmslr_) {
                // x2 -= F x1 with F = A(C rows, B cols) (GMSLRDPrecondition.cpp:1080)
                upload_csr(D.Et, D.nrem, L.F.rowptr, L.F.col, L.F.val, st);
            } else {
                // x2 -= E^T x1 (AMSEDPrecondition.cpp:1535-1540), E^T explicit
                std::vector<uint32_t> trp, tcol;
                std::vector<double> tval;
                transpose_rect(L.E, D.nrem, trp, tcol, tval);
                upload_csr(D.Et, D.nrem, trp, tcol, tval, st);
            }
            D.rank = L.rank;
            if (D.rank > (uint32_t)kMaxRank)
                throw Error(PRISM_ERR_UNSUPPORTED, "low-rank correction above " + std::to_string(kMaxRank) + " columns");
            if (D.rank) {
                D.W.upload(L.W.data(), L.W.size(), st);
                D.H.upload(L.H.data(), L.H.size(), st);
                D.t.alloc(D.rank);
            }
            D.xc.alloc(std::max<uint32_t>(D.nrem, 1));
            D.tmp.alloc(std::max<uint32_t>(D.nb, 1));
            D.tmp2.alloc(std::max<uint32_t>(D.nb, 1));
            max_rank = std::max(max_rank, D.rank);
        }
    }
    partial_.alloc((size_t)std::max<uint32_t>(max_rank, 1) * (size_t)h_.info.sms * 4);
    PRISM_CUDA(cudaStreamSynchronize(st));
}

// out = B_level^{-1} in over the level's rows (in == out allowed)
void AmsedPrecond::block_solve(cudaStream_t st, int level, const double* in, double* out) {
    Level& L = lv_[level];
    if (L.nfac < L.nb && in != out)  // rows without a factor (last level beyond block 0) pass through
        PRISM_CUDA(cudaMemcpyAsync(out + L.nfac, in + L.nfac, (L.nb - L.nfac) * sizeof(double),
                                   cudaMemcpyDeviceToDevice, st));
    if (!L.lower.self_filling()) launch_fill(st, h_, L.nfac, sweep_tmp_.get());
    if (in != out && !L.upper.self_filling()) launch_fill(st, h_, L.nfac, out);
    launch_sweep(h_, st, L.lower, in, sweep_tmp_.get());
    if (in == out && !L.upper.self_filling()) launch_fill(st, h_, L.nfac, out);
    launch_sweep(h_, st, L.upper, sweep_tmp_.get(), out);
}

// levelCInvRecursiveSolve(level, x): x is the C block of `level` (global rows lev_ptr[level+1]..n)
void AmsedPrecond::c_solve(cudaStream_t st, int level, double* x) {
    const int next = level + 1;
    if (level == (int)nlev_ - 2) {
        block_solve(st, next, x, x);
        return;
    }
    Level& L = lv_[next];
    const int vg = vec_grid(h_, std::max(L.nb, L.nrem));
    // x1 = B^{-1} x1
    block_solve(st, next, x, x);
    // x2 -= E^T x1
    launch_spmv(h_, st, L.nrem, L.Et.rowptr.get(), L.Et.col.get(), L.Et.val.get(), x, x + L.nb, 1);
    // xc = x2 ; x2 = C^{-1} x2
    PRISM_CUDA(cudaMemcpyAsync(L.xc.get(), x + L.nb, L.nrem * sizeof(double), cudaMemcpyDeviceToDevice, st));
    c_solve(st, next, x + L.nb);
    // x2 += W (H o (W^T xc))
    if (L.rank) {
        const int g = vec_grid(h_, L.nrem);
        k_lowrank_dots<<<g, kBlock, 0, st>>>(L.nrem, L.rank, L.W.get(), L.xc.get(), partial_.get());
        PRISM_LAUNCHED();
        k_lowrank_finish<<<1, 128, 0, st>>>((uint32_t)g, L.rank, partial_.get(), L.H.get(), L.t.get());
        PRISM_LAUNCHED();
        k_lowrank_add<<<g, kBlock, 0, st>>>(L.nrem, L.rank, L.W.get(), L.t.get(), x + L.nb);
        PRISM_LAUNCHED();
    }
    // x1 -= B^{-1} (E x2)
    launch_spmv(h_, st, L.nb, L.E.rowptr.get(), L.E.col.get(), L.E.val.get(), x + L.nb, L.tmp.get(), 0);
    block_solve(st, next, L.tmp.get(), L.tmp2.get());
    k_sub<<<vg, kBlock, 0, st>>>(L.nb, L.tmp2.get(), x);
    PRISM_LAUNCHED();
}

void AmsedPrecond::apply(cudaStream_t st, const double* in, double* out) {
    const int vg = vec_grid(h_, n_);
    k_permute<<<vg, kBlock, 0, st>>>(n_, pperm_.get(), in, X_.get(), 0);
    PRISM_LAUNCHED();
    if (nlev_ == 1) block_solve(st, 0, X_.get(), X_.get());
    else c_solve(st, -1, X_.get());
    k_permute<<<vg, kBlock, 0, st>>>(n_, pperm_.get(), X_.get(), out, 1);
    PRISM_LAUNCHED();
}

// ============================================================================
// Block apply: k <= 64 interleaved columns (X[row * k + c])
// ============================================================================
void launch_bt_fill(cudaStream_t st, const Handle& h, uint64_t count, double* p);
void launch_bt_sweep(const Handle& h, cudaStream_t st, const DevSweep& s, uint32_t k, const double* in, double* out);

namespace {
// float -> BF16, round to nearest even (NaN kept quiet)
uint16_t bf16_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7F800000u) == 0x7F800000u && (u & 0x007FFFFFu)) return (uint16_t)((u >> 16) | 0x40u);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

int bk_grid(const Handle& h, uint64_t items, uint32_t per_block) {
    uint64_t want = (items + per_block - 1) / per_block;
    const uint64_t cap = (uint64_t)h.info.sms * 4;
    if (want < 1) want = 1;
    return (int)(want < cap ? want : cap);
}
}  // namespace

void AmsedPrecond::prepare_block(uint32_t k) {
    if (bk_ >= k && !blv_.empty()) return;
    cudaStream_t st = h_.stream;
    tensor_lowrank_ = a_->fp32;
    const bool first = blv_.empty();
    if (first) blv_.resize(nlev_);
    size_t part64 = 1, part32 = 1, t64 = 1, t32 = 1;
    uint32_t max_nfac = 1;
    for (uint32_t l = 0; l < nlev_; ++l) {
        Level& L = lv_[l];
        BlockLevel& B = blv_[l];
        if (first) {
            // level-order copies of the sweeps (the block sweep kernel's layout)
            if (a_->fp32) {
                Sweep<float> lo, up;
                level_sweeps<float>(*a_->s32, l, lo, up);
                B.lower.upload(lo, h_.info, LAYOUT_LEVEL, st);
                B.upper.upload(up, h_.info, LAYOUT_LEVEL, st);
            } else {
                Sweep<double> lo, up;
                level_sweeps<double>(*a_->s64, l, lo, up);
                B.lower.upload(lo, h_.info, LAYOUT_LEVEL, st);
                B.upper.upload(up, h_.info, LAYOUT_LEVEL, st);
            }
            if (L.rank && tensor_lowrank_) {
                const std::vector<double>& W = a_->fp32 ? a_->s32->levels[l].W : a_->s64->levels[l].W;
                const std::vector<double>& Hh = a_->fp32 ? a_->s32->levels[l].H : a_->s64->levels[l].H;
                B.rpad = (L.rank + 15) / 16 * 16;
                B.ldw = (L.nrem + 15) / 16 * 16;
                std::vector<uint16_t> wc((size_t)B.rpad * B.ldw, 0), wr((size_t)B.ldw * B.rpad, 0);
                for (uint32_t q = 0; q < L.rank; ++q)
                    for (uint32_t i = 0; i < L.nrem; ++i) {
                        const uint16_t v = bf16_bits((float)W[(size_t)q * L.nrem + i]);
                        wc[(size_t)q * B.ldw + i] = v;
                        wr[(size_t)i * B.rpad + q] = v;
                    }
                std::vector<float> h32(B.rpad, 0.f);
                for (uint32_t q = 0; q < L.rank; ++q) h32[q] = (float)Hh[q];
                B.Wc.upload(wc.data(), wc.size(), st);
                B.Wr.upload(wr.data(), wr.size(), st);
                B.H32.upload(h32.data(), h32.size(), st);
            }
        }
        max_nfac = std::max(max_nfac, L.nfac);
        if (l + 1 < nlev_) {
            B.xc.alloc(std::max<size_t>((size_t)L.nrem * k, 1));
            B.tmp.alloc(std::max<size_t>((size_t)L.nb * k, 1));
            B.tmp2.alloc(std::max<size_t>((size_t)L.nb * k, 1));
            if (L.rank) {
                part64 = std::max(part64, (size_t)bk_grid(h_, L.nrem, 64) * L.rank * kLrMaxK);
                t64 = std::max(t64, (size_t)L.rank * kLrMaxK);
                if (tensor_lowrank_) {
                    part32 = std::max(part32, (size_t)bk_grid(h_, B.ldw / 16, kBlock / 32) * B.rpad * kLrMaxK);
                    t32 = std::max(t32, (size_t)B.rpad * kLrMaxK);
                }
            }
        }
    }
    Xk_.alloc((size_t)n_ * k);
    sweep_tmpk_.alloc((size_t)max_nfac * k);
    lr_part64_.alloc(part64);
    lr_t64_.alloc(t64);
    lr_part32_.alloc(part32);
    lr_t32_.alloc(t32);
    if (lr_ticket_.size() == 0) {
        lr_ticket_.alloc(1);
        PRISM_CUDA(cudaMemsetAsync(lr_ticket_.get(), 0, sizeof(unsigned), st));
    }
    bk_ = k;
    PRISM_CUDA(cudaStreamSynchronize(st));
}

// out = B_level^{-1} in over the level's rows, k columns (in == out allowed)
void AmsedPrecond::block_solve_k(cudaStream_t st, int level, uint32_t k, const double* in, double* out) {
    Level& L = lv_[level];
    BlockLevel& B = blv_[level];
    if (L.nfac < L.nb && in != out)
        PRISM_CUDA(cudaMemcpyAsync(out + (size_t)L.nfac * k, in + (size_t)L.nfac * k,
                                   (size_t)(L.nb - L.nfac) * k * sizeof(double), cudaMemcpyDeviceToDevice, st));
    const uint64_t cnt = (uint64_t)L.nfac * k;
    launch_bt_fill(st, h_, cnt, sweep_tmpk_.get());
    if (in != out) launch_bt_fill(st, h_, cnt, out);
    launch_bt_sweep(h_, st, B.lower, k, in, sweep_tmpk_.get());
    if (in == out) launch_bt_fill(st, h_, cnt, out);
    launch_bt_sweep(h_, st, B.upper, k, sweep_tmpk_.get(), out);
}

// x2 += W (H o (W^T xc)) on k columns
void AmsedPrecond::lowrank_k(cudaStream_t st, int level, uint32_t k, const double* xc, double* y) {
    Level& L = lv_[level];
    BlockLevel& B = blv_[level];
    if (tensor_lowrank_) {
        const int g = bk_grid(h_, B.ldw / 16, kBlock / 32);
        k_lr_dots_tc<<<g, kBlock, 0, st>>>(L.nrem, B.ldw, k, B.rpad, reinterpret_cast<const __nv_bfloat16*>(B.Wc.get()),
                                           B.H32.get(), xc, lr_part32_.get(), lr_ticket_.get(), lr_t32_.get());
        PRISM_LAUNCHED();
        const size_t smem = (size_t)(B.rpad / 2) * kLrMaxK * sizeof(uint32_t);
        k_lr_add_tc<<<g, kBlock, smem, st>>>(L.nrem, B.ldw, k, B.rpad, reinterpret_cast<const __nv_bfloat16*>(B.Wr.get()),
                                             lr_t32_.get(), y);
        PRISM_LAUNCHED();
    } else {
        const int g = bk_grid(h_, L.nrem, 64);
        k_lr_dots_f64<<<g, kBlock, 0, st>>>(L.nrem, k, L.rank, L.W.get(), L.H.get(), xc, lr_part64_.get(),
                                            lr_ticket_.get(), lr_t64_.get());
        PRISM_LAUNCHED();
        k_lr_add_f64<<<bk_grid(h_, (uint64_t)L.nrem * k, kBlock), kBlock, 0, st>>>(L.nrem, k, L.rank, L.W.get(),
                                                                                   lr_t64_.get(), y);
        PRISM_LAUNCHED();
    }
}

// levelCInvRecursiveSolve(level, x) on k columns; x is the C block of `level`
void AmsedPrecond::c_solve_k(cudaStream_t st, int level, uint32_t k, double* x) {
    const int next = level + 1;
    if (level == (int)nlev_ - 2) {
        block_solve_k(st, next, k, x, x);
        return;
    }
    Level& L = lv_[next];
    BlockLevel& B = blv_[next];
    double* x2 = x + (size_t)L.nb * k;
    // x1 = B^{-1} x1
    block_solve_k(st, next, k, x, x);
    // x2 -= E^T x1
    k_bk_csr<1><<<bk_grid(h_, L.nrem, kBlock / 32), kBlock, 0, st>>>(L.nrem, k, L.Et.rowptr.get(), L.Et.col.get(),
                                                                      L.Et.val.get(), x, x2);
    PRISM_LAUNCHED();
    // xc = x2 ; x2 = C^{-1} x2
    PRISM_CUDA(cudaMemcpyAsync(B.xc.get(), x2, (size_t)L.nrem * k * sizeof(double), cudaMemcpyDeviceToDevice, st));
    c_solve_k(st, next, k, x2);
    // x2 += W (H o (W^T xc))
    if (L.rank) lowrank_k(st, next, k, B.xc.get(), x2);
    // x1 -= B^{-1} (E x2)
    k_bk_csr<0><<<bk_grid(h_, L.nb, kBlock / 32), kBlock, 0, st>>>(L.nb, k, L.E.rowptr.get(), L.E.col.get(),
                                                                    L.E.val.get(), x2, B.tmp.get());
    PRISM_LAUNCHED();
    block_solve_k(st, next, k, B.tmp.get(), B.tmp2.get());
    k_bk_sub<<<bk_grid(h_, (uint64_t)L.nb * k, kBlock), kBlock, 0, st>>>((uint64_t)L.nb * k, B.tmp2.get(), x);
    PRISM_LAUNCHED();
}

void AmsedPrecond::apply_batched(cudaStream_t st, uint32_t k, const double* in, double* out) {
    if (k == 0 || k > (uint32_t)kLrMaxK) throw Error(PRISM_ERR_ARG, "a block holds 1 to 64 columns");
    prepare_block(k);
    const int g = bk_grid(h_, (uint64_t)n_ * k, kBlock);
    k_bk_permute<<<g, kBlock, 0, st>>>(n_, k, pperm_.get(), in, Xk_.get(), 0);
    PRISM_LAUNCHED();
    if (nlev_ == 1) block_solve_k(st, 0, k, Xk_.get(), Xk_.get());
    else c_solve_k(st, -1, k, Xk_.get());
    k_bk_permute<<<g, kBlock, 0, st>>>(n_, k, pperm_.get(), Xk_.get(), out, 1);
    PRISM_LAUNCHED();
}

// The block low-rank correction alone on `device` (host arrays): Y += W (H o (W^T X)).
void lowrank_block_run(int device, uint32_t nrem, uint32_t rank, uint32_t k, const double* W, const double* H,
                       const double* X, double* Y, bool tensor) {
    DeviceInfo info;
    init_device_info(info, device);
    cudaStream_t st;
    PRISM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{st};
    const size_t nk = (size_t)nrem * k;
    DevBuf<double> dX, dY;
    dX.upload(X, nk, st);
    dY.upload(Y, nk, st);
    DevBuf<unsigned> ticket(1);
    PRISM_CUDA(cudaMemsetAsync(ticket.get(), 0, sizeof(unsigned), st));
    auto grid = [&](uint64_t items, uint32_t per) {
        uint64_t want = (items + per - 1) / per;
        const uint64_t cap = (uint64_t)info.sms * 4;
        return (int)std::max<uint64_t>(1, std::min(want, cap));
    };
    if (tensor) {
        const uint32_t rpad = (rank + 15) / 16 * 16, ldw = (nrem + 15) / 16 * 16;
        std::vector<uint16_t> wc((size_t)rpad * ldw, 0), wr((size_t)ldw * rpad, 0);
        for (uint32_t q = 0; q < rank; ++q)
            for (uint32_t i = 0; i < nrem; ++i) {
                const uint16_t v = bf16_bits((float)W[(size_t)q * nrem + i]);
                wc[(size_t)q * ldw + i] = v;
                wr[(size_t)i * rpad + q] = v;
            }
        std::vector<float> h32(rpad, 0.f);
        for (uint32_t q = 0; q < rank; ++q) h32[q] = (float)H[q];
        DevBuf<uint16_t> dWc, dWr;
        DevBuf<float> dH, dT((size_t)rpad * kLrMaxK);
        dWc.upload(wc.data(), wc.size(), st);
        dWr.upload(wr.data(), wr.size(), st);
        dH.upload(h32.data(), h32.size(), st);
        const int g = grid(ldw / 16, kBlock / 32);
        DevBuf<float> part((size_t)g * rpad * kLrMaxK);
        k_lr_dots_tc<<<g, kBlock, 0, st>>>(nrem, ldw, k, rpad, reinterpret_cast<const __nv_bfloat16*>(dWc.get()),
                                           dH.get(), dX.get(), part.get(), ticket.get(), dT.get());
        PRISM_LAUNCHED();
        k_lr_add_tc<<<g, kBlock, (size_t)(rpad / 2) * kLrMaxK * sizeof(uint32_t), st>>>(
            nrem, ldw, k, rpad, reinterpret_cast<const __nv_bfloat16*>(dWr.get()), dT.get(), dY.get());
        PRISM_LAUNCHED();
        PRISM_CUDA(cudaMemcpyAsync(Y, dY.get(), nk * sizeof(double), cudaMemcpyDeviceToHost, st));
        PRISM_CUDA(cudaStreamSynchronize(st));
    } else {
        DevBuf<double> dW, dH, dT((size_t)rank * kLrMaxK);
        dW.upload(W, (size_t)rank * nrem, st);
        dH.upload(H, rank, st);
        const int g = grid(nrem, 64);
        DevBuf<double> part((size_t)g * rank * kLrMaxK);
        k_lr_dots_f64<<<g, kBlock, 0, st>>>(nrem, k, rank, dW.get(), dH.get(), dX.get(), part.get(), ticket.get(),
                                            dT.get());
        PRISM_LAUNCHED();
        k_lr_add_f64<<<grid(nk, kBlock), kBlock, 0, st>>>(nrem, k, rank, dW.get(), dT.get(), dY.get());
        PRISM_LAUNCHED();
        PRISM_CUDA(cudaMemcpyAsync(Y, dY.get(), nk * sizeof(double), cudaMemcpyDeviceToHost, st));
        PRISM_CUDA(cudaStreamSynchronize(st));
    }
}

uint32_t AmsedPrecond::levels(int sweep) const {
    uint32_t m = 0;
    for (const Level& L : lv_) m = std::max(m, sweep == 0 ? L.lower.num_levels : L.upper.num_levels);
    return m;
}

bool AmsedPrecond::run_sweep(cudaStream_t st, int sweep, const double* in, double* out, int prepare) {
    if (sweep < 0 || sweep >= (int)(2 * nlev_)) return false;
    const Level& L = lv_[sweep / 2];
    const DevSweep& s = (sweep & 1) ? L.upper : L.lower;
    if (prepare != 0) launch_sweep_prepare(h_, st, s, in, out);
    if (prepare != 2) launch_sweep_kernel(h_, st, s, in, out);
    return true;
}

bool AmsedPrecond::sweep_info(int sweep, uint32_t* n, uint64_t* nnz, uint32_t* vbytes, uint32_t* levels,
                              uint32_t* kernel) const {
    if (sweep < 0 || sweep >= (int)(2 * nlev_)) return false;
    const Level& L = lv_[sweep / 2];
    const DevSweep& s = (sweep & 1) ? L.upper : L.lower;
    if (n) *n = s.n;
    if (nnz) *nnz = s.entries();
    if (vbytes) *vbytes = s.fp32 ? 4 : 8;
    if (levels) *levels = s.num_levels;
    if (kernel) *kernel = s.layout == LAYOUT_STREAM ? 3 : (s.layout == LAYOUT_SLAB ? 2 : 1);
    return true;
}

bool AmsedPrecond::sweep_order(int sweep, StreamOrder& o) const {
    if (sweep < 0 || sweep >= (int)(2 * nlev_)) return false;
    const Level& L = lv_[sweep / 2];
    const DevSweep& d = (sweep & 1) ? L.upper : L.lower;
    if (d.layout != LAYOUT_STREAM) return false;
    if (a_->fp32) {
        Sweep<float> lo, up;
        level_sweeps<float>(*a_->s32, (uint32_t)sweep / 2, lo, up);
        return d.stream_order<float>((sweep & 1) ? up : lo, o);
    }
    Sweep<double> lo, up;
    level_sweeps<double>(*a_->s64, (uint32_t)sweep / 2, lo, up);
    return d.stream_order<double>((sweep & 1) ? up : lo, o);
}

template void AmsedPrecond::build<double>(const AmsedSetup<double>&);
template void AmsedPrecond::build<float>(const AmsedSetup<float>&);

}  // namespace prism
