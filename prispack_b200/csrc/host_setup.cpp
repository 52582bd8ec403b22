// Host-side setup: model problems, bit-exact incomplete factorisations and the
// exact integer level schedules used by the device sweeps.
#include "host_setup.hpp"

#include <algorithm>
#include <cmath>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <thread>
#include <type_traits>

namespace prism {

// ============================================================================
// Model problems
// ============================================================================
bool laplacian_dims(int32_t nx, int32_t ny, int32_t nz, uint32_t* n, uint32_t* nnz) {
    if (nx <= 0 || ny <= 0 || nz <= 0) return false;
    uint64_t N = (uint64_t)nx * ny * nz;
    if (N >= 0xFFFFFFFFull) return false;
    // every row has a diagonal plus one entry per existing neighbour
    uint64_t off = 2ull * ((uint64_t)(nx - 1) * ny * nz + (uint64_t)nx * (ny - 1) * nz + (uint64_t)nx * ny * (nz - 1));
    uint64_t total = N + off;
    if (total >= 0xFFFFFFFFull) return false;
    *n = (uint32_t)N;
    *nnz = (uint32_t)total;
    return true;
}

void laplacian_fill(int32_t nx, int32_t ny, int32_t nz, double ax, double ay, double az, double shift,
                    uint32_t* rowptr, uint32_t* col, double* val) {
    // Coefficients as generateLaplacianCOO computes them (ModelProblem.cpp:76-93):
    // a problem is "2D" as soon as one dimension is 1.
    int ones = (nx == 1) + (ny == 1) + (nz == 1);
    const double v = -1.0;
    const double vxp = v - ax, vxn = v + ax, vyp = v - ay, vyn = v + ay, vzp = v - az, vzn = v + az;
    double vd = ones > 0 ? 4.0 : 6.0;
    vd -= shift;
    const int64_t nxy = (int64_t)nx * ny;
    const int64_t N = nxy * nz;
    uint32_t pos = 0;
    rowptr[0] = 0;
    for (int64_t ii = 0; ii < N; ++ii) {
        const int64_t k = ii / nxy;
        const int64_t i = (ii - k * nxy) / nx;
        const int64_t j = ii - k * nxy - i * nx;
        // collect (column, value) then order by column, as transCOO2CSR's per-row sort does
        int64_t c[7];
        double w[7];
        int m = 0;
        if (k > 0) { c[m] = ii - nxy; w[m++] = vzn; }
        if (k < nz - 1) { c[m] = ii + nxy; w[m++] = vzp; }
        if (i > 0) { c[m] = ii - nx; w[m++] = vyn; }
        if (i < ny - 1) { c[m] = ii + nx; w[m++] = vyp; }
        if (j > 0) { c[m] = ii - 1; w[m++] = vxn; }
        if (j < nx - 1) { c[m] = ii + 1; w[m++] = vxp; }
        c[m] = ii;
        w[m++] = vd;
        for (int a = 1; a < m; ++a) {  // insertion sort, stable
            int64_t kc = c[a];
            double kv = w[a];
            int b = a - 1;
            while (b >= 0 && c[b] > kc) { c[b + 1] = c[b]; w[b + 1] = w[b]; --b; }
            c[b + 1] = kc;
            w[b + 1] = kv;
        }
        for (int a = 0; a < m; ++a) { col[pos] = (uint32_t)c[a]; val[pos] = w[a]; ++pos; }
        rowptr[ii + 1] = pos;
    }
}

std::string validate_csr(uint32_t n, const uint32_t* rowptr, const uint32_t* col) {
    if (rowptr[0] != 0) return "rowptr[0] must be 0";
    for (uint32_t i = 0; i < n; ++i) {
        if (rowptr[i + 1] < rowptr[i]) return "row offsets must be non-decreasing (row " + std::to_string(i) + ")";
        for (uint32_t k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            if (col[k] >= n) return "column index out of range in row " + std::to_string(i);
            if (k > rowptr[i] && col[k] <= col[k - 1])
                return "columns must be strictly increasing inside row " + std::to_string(i);
        }
    }
    return std::string();
}

bool csr_symmetric(const CsrHost& A) {
    for (uint32_t i = 0; i < A.n; ++i) {
        for (uint32_t k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k) {
            const uint32_t j = A.col[k];
            if (j <= i) continue;
            const uint32_t* b = A.col.data() + A.rowptr[j];
            const uint32_t* e = A.col.data() + A.rowptr[j + 1];
            const uint32_t* f = std::lower_bound(b, e, i);
            if (f == e || *f != i || A.val[f - A.col.data()] != A.val[k]) return false;
        }
    }
    return true;
}

// ============================================================================
// Threshold incomplete Cholesky (left-looking, column linked lists)
// ============================================================================
namespace {
constexpr uint32_t kNone = 0xFFFFFFFFu;

// Shared driver of the two left-looking threshold factorisations.  The
// reference keeps, for every finished column k, a cursor (`next`) to its next
// unconsumed entry and threads k into the list of the row that entry lives in
// (`link` doubles as list head for rows not yet reached and as list link for
// finished columns; lists are LIFO).  Column j gathers its updates by walking
// the list of row j.  `ldlt` selects the IncompleteLDLT variant (no sqrt,
// pivot kept in D, unit L^T stored without its diagonal).
template <typename Low, bool ldlt>
int left_looking(const CsrHost& A, double thr, CsrT<Low>& Lt, std::vector<double>* D, std::string* err,
                 RefactorPlan* plan) {
    const uint32_t n = A.n;
    std::vector<uint8_t> used(n, 0);
    std::vector<uint32_t> touched(n);
    std::vector<double> acc(n, 0.0);
    std::vector<uint32_t> link(n, kNone);
    std::vector<uint32_t> next(n, 0);
    Lt.n = n;
    Lt.rowptr.assign((size_t)n + 1, 0);
    Lt.col.clear();
    Lt.val.clear();
    Lt.col.reserve(A.nnz() * 4);
    Lt.val.reserve(A.nnz() * 4);
    if (ldlt) D->assign(n, 0.0);
    if (plan) {
        *plan = RefactorPlan();
        plan->n = n;
        plan->ldlt = ldlt;
        plan->a_ptr.assign(1, 0);
        plan->up_ptr.assign(1, 0);
    }

    for (uint32_t j = 0; j < n; ++j) {
        uint32_t cnt = 0;
        double colThr = 0.0;
        // lower part of column j of A (row j, symmetric storage)
        for (uint32_t p = A.rowptr[j]; p < A.rowptr[j + 1]; ++p) {
            const uint32_t i = A.col[p];
            const double a = A.val[p];
            if (i >= j) {
                if (plan) plan->a_pos.push_back(p);
                colThr += std::fabs(a);
                if (!used[i]) { acc[i] = 0.0; used[i] = 1; touched[cnt++] = i; }
                acc[i] += a;
            }
        }
        colThr *= thr;
        // updates from every finished column k with a non-zero in row j
        uint32_t k = link[j];
        while (k != kNone) {
            uint32_t start = next[k];
            if (plan) {
                plan->up_k.push_back(k);
                plan->up_start.push_back(start);
            }
            const double Ljk = (double)Lt.val[start];
            const double dk = ldlt ? (*D)[k] : 0.0;
            const uint32_t stop = Lt.rowptr[k + 1];
            for (uint32_t p = start; p < stop; ++p) {
                const uint32_t i = Lt.col[p];
                const double Lik = (double)Lt.val[p];
                if (!used[i]) { used[i] = 1; acc[i] = 0.0; touched[cnt++] = i; }
                if (ldlt) acc[i] -= Lik * Ljk * dk;
                else acc[i] -= Lik * Ljk;
            }
            ++start;
            const uint32_t knext = link[k];
            if (start < stop) {
                next[k] = start;
                const uint32_t i = Lt.col[start];
                link[k] = link[i];
                link[i] = k;
            }
            k = knext;
        }
        double piv = acc[j];
        if (ldlt) {
            if (std::fabs(piv) < 1e-15) {
                if (err) *err = "ILDLT: zero diagonal encountered! Zero diagonal row index is: " + std::to_string(j);
                return SETUP_ZERO_PIVOT;
            }
            (*D)[j] = piv;
            next[j] = (uint32_t)Lt.col.size();
        } else {
            if (piv <= 0.0) {
                if (err) *err = "The original matrix is not positive definite! (column " + std::to_string(j) + ")";
                return SETUP_NOT_SPD;
            }
            piv = std::sqrt(piv);
            acc[j] = piv;
            Lt.val.push_back((Low)piv);
            Lt.col.push_back(j);
            next[j] = (uint32_t)Lt.col.size();
        }
        std::sort(touched.begin(), touched.begin() + cnt);
        bool first = true;
        for (uint32_t q = 0; q < cnt; ++q) {
            const uint32_t i = touched[q];
            if (i != j) {
                double Lij = acc[i];
                if (std::fabs(Lij) >= colThr) {
                    if (first) {
                        first = false;
                        link[j] = link[i];
                        link[i] = j;
                    }
                    Lij = Lij / piv;
                    Lt.val.push_back((Low)Lij);
                    Lt.col.push_back(i);
                }
            }
            used[i] = 0;
        }
        Lt.rowptr[j + 1] = (uint32_t)Lt.col.size();
        if (plan) {
            plan->a_ptr.push_back((uint32_t)plan->a_pos.size());
            plan->up_ptr.push_back((uint32_t)plan->up_k.size());
            plan->max_col = std::max<uint32_t>(plan->max_col, Lt.rowptr[j + 1] - Lt.rowptr[j] + (ldlt ? 1u : 0u));
        }
    }
    return SETUP_OK;
}

// Selection of the Ncut largest |a| to the front (SPARSKIT qsplit, as used by
// include/VectorClass/VectorTools.h:160-203); it also reorders the rest, and
// the reference calls it even when nothing is dropped, so its exact swap
// sequence fixes the column order of every ILUT row.
template <typename T>
void qsplit_select(T* a, int32_t* ind, int32_t n, int32_t ncut_count) {
    const int32_t ncut = ncut_count - 1;
    int32_t first = 0, last = n - 1;
    if (ncut < first || ncut > last) return;
    int32_t mid;
    do {
        mid = first;
        const double key = std::fabs((double)a[mid]);
        for (int32_t j = first + 1; j <= last; ++j) {
            if (std::fabs((double)a[j]) > key) {
                ++mid;
                const double tmp = (double)a[mid];
                const int32_t itmp = ind[mid];
                a[mid] = a[j];
                ind[mid] = ind[j];
                a[j] = (T)tmp;
                ind[j] = itmp;
            }
        }
        const double tmp = (double)a[mid];
        a[mid] = a[first];
        a[first] = (T)tmp;
        const int32_t itmp = ind[mid];
        ind[mid] = ind[first];
        ind[first] = itmp;
        if (mid == ncut) break;
        if (mid > ncut) last = mid - 1;
        else first = mid + 1;
    } while (mid != ncut);
}
}  // namespace

template <typename Low>
int ict_factor(const CsrHost& A, double threshold, CsrT<Low>& Lt, std::string* err, RefactorPlan* plan) {
    return left_looking<Low, false>(A, threshold, Lt, nullptr, err, plan);
}

template <typename Low>
int ildlt_factor(const CsrHost& A, double tol, CsrT<Low>& Lt, std::vector<double>& D, std::string* err,
                 RefactorPlan* plan) {
    return left_looking<Low, true>(A, tol, Lt, &D, err, plan);
}

template <typename Low>
int ilut_factor(const CsrHost& A, uint32_t lfill, double tol, CsrT<Low>& L, CsrT<Low>& U, std::vector<Low>& Dinv,
                std::string* err) {
    const int32_t n = (int32_t)A.n;
    L.n = U.n = A.n;
    L.rowptr.assign((size_t)n + 1, 0);
    U.rowptr.assign((size_t)n + 1, 0);
    L.col.clear(); L.val.clear(); U.col.clear(); U.val.clear();
    Dinv.assign(n, (Low)0);
    std::vector<int32_t> iw(n, -1), jbuf(n);
    std::vector<Low> wn(n), w(n);
    for (int32_t i = 0; i < n; ++i) {
        const uint32_t begin = A.rowptr[i], end = A.rowptr[i + 1];
        const uint32_t nzcount = end - begin;
        double tnorm = 0.0;
        for (uint32_t p = begin; p < end; ++p) tnorm += std::fabs(A.val[p]);
        if (tnorm < 1e-15) {
            if (err) *err = "ILUT: zero row encountered! (row " + std::to_string(i) + ")";
            return SETUP_ZERO_PIVOT;
        }
        tnorm /= (double)nzcount;
        const double tolnorm = tol * tnorm;
        // split row i of A into the work row: L part at [0, lenl), diagonal at i, U part at (i, i+lenu]
        int32_t lenu = 0, lenl = 0;
        jbuf[i] = i;
        w[i] = (Low)0;
        iw[i] = i;
        for (uint32_t p = begin; p < end; ++p) {
            const int32_t c = (int32_t)A.col[p];
            const Low t = (Low)A.val[p];
            if (c < i) {
                iw[c] = lenl; jbuf[lenl] = c; w[lenl] = t; ++lenl;
            } else if (c == i) {
                w[i] = t;
            } else {
                ++lenu;
                const int32_t jpos = i + lenu;
                iw[c] = jpos; jbuf[jpos] = c; w[jpos] = t;
            }
        }
        // eliminate the L part in increasing column order (selection of the smallest remaining column)
        for (int32_t jj = 0; jj < lenl; ++jj) {
            int32_t jrow = jbuf[jj];
            int32_t jpos = jj;
            for (int32_t q = jj + 1; q < lenl; ++q)
                if (jbuf[q] < jrow) { jrow = jbuf[q]; jpos = q; }
            if (jpos != jj) {
                const int32_t c = jbuf[jj];
                jbuf[jj] = jbuf[jpos];
                jbuf[jpos] = c;
                iw[jrow] = jj;
                iw[c] = jpos;
                const Low t = w[jj];
                w[jj] = w[jpos];
                w[jpos] = t;
            }
            const Low fact = w[jj] * Dinv[jrow];
            w[jj] = fact;
            iw[jrow] = -1;
            for (uint32_t q = U.rowptr[jrow]; q < U.rowptr[jrow + 1]; ++q) {
                const int32_t c = (int32_t)U.col[q];
                const int32_t cpos = iw[c];
                const Low lxu = -fact * U.val[q];
                if (std::fabs((double)lxu) < tolnorm && cpos == -1) continue;
                if (c < i) {
                    if (cpos == -1) {
                        jbuf[lenl] = c; iw[c] = lenl; w[lenl] = lxu; ++lenl;
                    } else {
                        w[cpos] += lxu;
                    }
                } else {
                    if (cpos == -1 && std::fabs((double)lxu) > tolnorm) {
                        ++lenu;
                        const int32_t upos = i + lenu;
                        jbuf[upos] = c; iw[c] = upos; w[upos] = lxu;
                    } else if (cpos != -1) {
                        // (|lxu| == tolnorm exactly with no slot: the reference indexes w[-1]; skipped here)
                        w[cpos] += lxu;
                    }
                }
            }
        }
        iw[i] = -1;
        for (int32_t q = 0; q < lenu; ++q) iw[jbuf[i + q + 1]] = -1;
        if (std::fabs((double)w[i]) < 1e-15) {
            if (err) *err = "ILUT: zero diagonal encountered! Zero diagonal row index is: " + std::to_string(i);
            return SETUP_ZERO_PIVOT;
        }
        Dinv[i] = (Low)1 / w[i];
        // keep the lfill largest of the L part
        int32_t len = lenl < (int32_t)lfill ? lenl : (int32_t)lfill;
        for (int32_t q = 0; q < lenl; ++q) { wn[q] = (Low)std::fabs((double)w[q]); iw[q] = q; }
        qsplit_select(wn.data(), iw.data(), lenl, len);
        for (int32_t q = 0; q < len; ++q) {
            const int32_t jpos = iw[q];
            L.col.push_back((uint32_t)jbuf[jpos]);
            L.val.push_back(w[jpos]);
        }
        L.rowptr[i + 1] = (uint32_t)L.col.size();
        for (int32_t q = 0; q < lenl; ++q) iw[q] = -1;
        // keep the lfill largest of the U part
        len = lenu < (int32_t)lfill ? lenu : (int32_t)lfill;
        for (int32_t q = 0; q < lenu; ++q) { wn[q] = (Low)std::fabs((double)w[i + q + 1]); iw[q] = i + q + 1; }
        qsplit_select(wn.data(), iw.data(), lenu, len);
        for (int32_t q = 0; q < len; ++q) {
            const int32_t jpos = iw[q];
            U.col.push_back((uint32_t)jbuf[jpos]);
            U.val.push_back(w[jpos]);
        }
        U.rowptr[i + 1] = (uint32_t)U.col.size();
        for (int32_t q = 0; q < lenu; ++q) iw[q] = -1;
    }
    return SETUP_OK;
}

// ============================================================================
// Sweeps and level schedules
// ============================================================================
template <typename V>
void transpose_csr(uint32_t n, const std::vector<uint32_t>& rowptr, const std::vector<uint32_t>& col,
                   const std::vector<V>& val, std::vector<uint32_t>& trp, std::vector<uint32_t>& tcol,
                   std::vector<V>& tval) {
    const uint64_t nnz = rowptr[n];
    trp.assign((size_t)n + 1, 0);
    tcol.resize(nnz);
    tval.resize(nnz);
    for (uint64_t k = 0; k < nnz; ++k) trp[col[k] + 1]++;
    for (uint32_t i = 0; i < n; ++i) trp[i + 1] += trp[i];
    std::vector<uint32_t> fill(trp.begin(), trp.end() - 1);
    for (uint32_t r = 0; r < n; ++r)
        for (uint32_t k = rowptr[r]; k < rowptr[r + 1]; ++k) {
            const uint32_t c = col[k];
            tcol[fill[c]] = r;
            tval[fill[c]] = val[k];
            fill[c]++;
        }
}

template <typename Low>
void build_sweep(uint32_t n, const std::vector<uint32_t>& rowptr, const std::vector<uint32_t>& col,
                 const std::vector<Low>& val, const std::vector<double>* diag, int op, bool lower,
                 Sweep<Low>& out) {
    std::vector<uint32_t> level(n, 0);
    uint32_t maxLevel = 0;
    if (lower) {
        for (uint32_t r = 0; r < n; ++r) {
            uint32_t l = 0;
            for (uint32_t k = rowptr[r]; k < rowptr[r + 1]; ++k) l = std::max(l, level[col[k]] + 1);
            level[r] = l;
            maxLevel = std::max(maxLevel, l);
        }
    } else {
        for (uint32_t r = n; r-- > 0;) {
            uint32_t l = 0;
            for (uint32_t k = rowptr[r]; k < rowptr[r + 1]; ++k) l = std::max(l, level[col[k]] + 1);
            level[r] = l;
            maxLevel = std::max(maxLevel, l);
        }
    }
    out.n = n;
    out.op = op;
    out.lower = lower;
    out.num_levels = n ? maxLevel + 1 : 0;
    out.level_ptr.assign((size_t)out.num_levels + 1, 0);
    for (uint32_t r = 0; r < n; ++r) out.level_ptr[level[r] + 1]++;
    for (uint32_t l = 0; l < out.num_levels; ++l) out.level_ptr[l + 1] += out.level_ptr[l];
    out.order.resize(n);
    {
        std::vector<uint32_t> fill(out.level_ptr.begin(), out.level_ptr.end() - 1);
        for (uint32_t r = 0; r < n; ++r) out.order[fill[level[r]]++] = r;
    }
    out.level = level;
    out.rowptr.assign((size_t)n + 1, 0);
    for (uint32_t p = 0; p < n; ++p) {
        const uint32_t r = out.order[p];
        out.rowptr[p + 1] = out.rowptr[p] + (rowptr[r + 1] - rowptr[r]);
    }
    out.col.resize(out.rowptr[n]);
    out.val.resize(out.rowptr[n]);
    out.diag.assign(n, 1.0);
    for (uint32_t p = 0; p < n; ++p) {
        const uint32_t r = out.order[p];
        std::copy(col.begin() + rowptr[r], col.begin() + rowptr[r + 1], out.col.begin() + out.rowptr[p]);
        std::copy(val.begin() + rowptr[r], val.begin() + rowptr[r + 1], out.val.begin() + out.rowptr[p]);
        if (diag) out.diag[p] = (*diag)[r];
    }
}

template <typename Low>
void pair_sweep(const Sweep<Low>& s, Sweep<Low>& out, PairMap& m) {
    const uint32_t n = s.n;
    std::vector<uint32_t> pos(n);  // row -> position
    for (uint32_t p = 0; p < n; ++p) pos[s.order[p]] = p;
    auto g_of = [&](uint32_t row) -> double {
        const double d = s.diag[pos[row]];
        switch (s.op) {
            case SWEEP_DIV:
            case SWEEP_PREDIV: return 1.0 / d;
            case SWEEP_MUL: return d;
            default: return 1.0;
        }
    };
    std::vector<double> diag(n, 1.0);
    // Rows are independent: contiguous chunks of rows on host threads, each with its own
    // scratch, concatenated in row order (the result does not depend on the threads).
    struct Chunk {
        std::vector<uint32_t> len, mlen, ci, dep;
        std::vector<Low> cv;
        std::vector<double> coef;
    };
    unsigned hc = std::max(1u, std::thread::hardware_concurrency());
    if (const char* e = std::getenv("PRISM_LAYOUT_THREADS")) hc = (unsigned)std::max(1, std::atoi(e));
    const uint32_t T = n < 65536 ? 1u : std::min<uint32_t>(std::min(hc, 16u), n);
    std::vector<Chunk> parts(T);
    auto work = [&](uint32_t t) {
        Chunk& c = parts[t];
        const uint32_t r0 = (uint32_t)((uint64_t)n * t / T), r1 = (uint32_t)((uint64_t)n * (t + 1) / T);
        std::vector<int32_t> slot(n, -1);  // dependency row -> index in the row being built
        std::vector<uint32_t> deps, idx;
        std::vector<double> acc;
        for (uint32_t r = r0; r < r1; ++r) {
            const uint32_t p = pos[r], lk = s.level[r];
            diag[r] = s.diag[p];
            deps.clear();
            acc.clear();
            auto add = [&](uint32_t j, double v) {
                if (slot[j] < 0) {
                    slot[j] = (int32_t)deps.size();
                    deps.push_back(j);
                    acc.push_back(v);
                } else {
                    acc[(size_t)slot[j]] = acc[(size_t)slot[j]] + v;
                }
            };
            const bool odd = (lk & 1u) != 0;
            uint32_t mcount = 0;
            // the row's own entries that stay, in stored order
            for (uint32_t k = s.rowptr[p]; k < s.rowptr[p + 1]; ++k) {
                const uint32_t j = s.col[k];
                if (!(odd && s.level[j] + 1 == lk)) add(j, (double)s.val[k]);
            }
            if (odd) {
                const double gk = g_of(r);
                for (uint32_t k = s.rowptr[p]; k < s.rowptr[p + 1]; ++k) {
                    const uint32_t i = s.col[k];
                    if (s.level[i] + 1 != lk) continue;
                    const double lki = (double)s.val[k], gi = g_of(i);
                    const double f = lki * (s.op == SWEEP_PREDIV ? 1.0 : gi);
                    const uint32_t pi = pos[i];
                    for (uint32_t q = s.rowptr[pi]; q < s.rowptr[pi + 1]; ++q) add(s.col[q], -(f * (double)s.val[q]));
                    c.dep.push_back(i);
                    c.coef.push_back(s.op == SWEEP_PREDIV ? lki * gi / gk : lki * gi);
                    ++mcount;
                }
            }
            c.mlen.push_back(mcount);
            // the row's entries, dependencies in increasing order
            idx.resize(deps.size());
            std::iota(idx.begin(), idx.end(), 0u);
            std::sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) { return deps[x] < deps[y]; });
            for (uint32_t t2 : idx) {
                c.ci.push_back(deps[t2]);
                c.cv.push_back((Low)acc[t2]);
            }
            c.len.push_back((uint32_t)deps.size());
            for (uint32_t j : deps) slot[j] = -1;
        }
    };
    if (T == 1) {
        work(0);
    } else {
        std::vector<std::thread> pool;
        for (uint32_t t = 0; t < T; ++t) pool.emplace_back(work, t);
        for (auto& th : pool) th.join();
    }
    std::vector<uint32_t> rp((size_t)n + 1, 0), ci;
    std::vector<Low> cv;
    m.ptr.assign((size_t)n + 1, 0);
    m.dep.clear();
    m.coef.clear();
    uint32_t r = 0;
    for (uint32_t t = 0; t < T; ++t) {
        Chunk& c = parts[t];
        for (size_t u = 0; u < c.len.size(); ++u, ++r) {
            rp[r + 1] = rp[r] + c.len[u];
            m.ptr[r + 1] = m.ptr[r] + c.mlen[u];
        }
        ci.insert(ci.end(), c.ci.begin(), c.ci.end());
        cv.insert(cv.end(), c.cv.begin(), c.cv.end());
        m.dep.insert(m.dep.end(), c.dep.begin(), c.dep.end());
        m.coef.insert(m.coef.end(), c.coef.begin(), c.coef.end());
        Chunk().ci.swap(c.ci);  // release as we go
        Chunk().cv.swap(c.cv);
    }
    build_sweep<Low>(n, rp, ci, cv, &diag, s.op, s.lower, out);
}

template <typename Low>
void slab_layout_ranges(const Sweep<Low>& s, const std::vector<uint32_t>& start, std::vector<uint32_t>& cta_pos,
                        Sweep<Low>& out) {
    const uint32_t n = s.n;
    const uint32_t num_ctas = (uint32_t)start.size() - 1;
    std::vector<uint32_t> owner(n);
    for (uint32_t b = 0; b < num_ctas; ++b)
        for (uint32_t r = start[b]; r < start[b + 1]; ++r) owner[r] = b;
    cta_pos.assign((size_t)num_ctas + 1, 0);
    for (uint32_t r = 0; r < n; ++r) cta_pos[owner[r] + 1]++;
    for (uint32_t b = 0; b < num_ctas; ++b) cta_pos[b + 1] += cta_pos[b];
    // the global (level, row) order, bucketed by owning CTA, stays (level, row) ordered per CTA
    std::vector<uint32_t> fill(cta_pos.begin(), cta_pos.end() - 1);
    std::vector<uint32_t> newpos_of_old(n);
    for (uint32_t p = 0; p < n; ++p) newpos_of_old[p] = fill[owner[s.order[p]]]++;
    out.n = n;
    out.op = s.op;
    out.lower = s.lower;
    out.num_levels = s.num_levels;
    out.level_ptr = s.level_ptr;
    out.level = s.level;
    out.order.resize(n);
    out.diag.resize(n);
    out.rowptr.assign((size_t)n + 1, 0);
    std::vector<uint32_t> old_of_new(n);
    for (uint32_t p = 0; p < n; ++p) old_of_new[newpos_of_old[p]] = p;
    for (uint32_t q = 0; q < n; ++q) {
        const uint32_t p = old_of_new[q];
        out.order[q] = s.order[p];
        out.diag[q] = s.diag[p];
        out.rowptr[q + 1] = out.rowptr[q] + (s.rowptr[p + 1] - s.rowptr[p]);
    }
    out.col.resize(s.col.size());
    out.val.resize(s.val.size());
    for (uint32_t q = 0; q < n; ++q) {
        const uint32_t p = old_of_new[q];
        std::copy(s.col.begin() + s.rowptr[p], s.col.begin() + s.rowptr[p + 1], out.col.begin() + out.rowptr[q]);
        std::copy(s.val.begin() + s.rowptr[p], s.val.begin() + s.rowptr[p + 1], out.val.begin() + out.rowptr[q]);
    }
}

template <typename Low>
void slab_layout(const Sweep<Low>& s, uint32_t num_ctas, uint32_t rows_per_cta, std::vector<uint32_t>& cta_pos,
                 Sweep<Low>& out) {
    std::vector<uint32_t> start((size_t)num_ctas + 1);
    for (uint32_t b = 0; b <= num_ctas; ++b) start[b] = (uint32_t)std::min<uint64_t>((uint64_t)b * rows_per_cta, s.n);
    start[num_ctas] = s.n;
    slab_layout_ranges<Low>(s, start, cta_pos, out);
}

template <typename Low>
std::vector<uint32_t> slab_ranges(const Sweep<Low>& s, uint32_t num_ctas) {
    const uint32_t n = s.n;
    // cut points: row boundaries that no dependency crosses (independent blocks of a
    // block-diagonal factor, e.g. the subdomains of an AMSED level)
    std::vector<uint32_t> reach(n);  // per row: farthest dependency (lowest for a lower sweep)
    for (uint32_t p = 0; p < n; ++p) {
        const uint32_t r = s.order[p];
        uint32_t m = r;
        for (uint32_t k = s.rowptr[p]; k < s.rowptr[p + 1]; ++k)
            m = s.lower ? std::min(m, s.col[k]) : std::max(m, s.col[k]);
        reach[r] = m;
    }
    std::vector<uint32_t> cuts{0};
    if (s.lower) {
        std::vector<uint32_t> suf((size_t)n + 1, n);
        for (uint32_t r = n; r-- > 0;) suf[r] = std::min(suf[r + 1], reach[r]);
        for (uint32_t b = 1; b < n; ++b)
            if (suf[b] >= b) cuts.push_back(b);
    } else {
        uint32_t pre = 0;
        for (uint32_t b = 1; b < n; ++b) {
            pre = std::max(pre, reach[b - 1]);
            if (pre < b) cuts.push_back(b);
        }
    }
    cuts.push_back(n);
    // segments of at least half a slab; smaller pieces join their neighbour
    const uint64_t target = ((uint64_t)n + num_ctas - 1) / num_ctas;
    std::vector<uint32_t> seg{0};
    for (size_t i = 1; i + 1 < cuts.size(); ++i)
        if (cuts[i] - seg.back() >= target / 2 && n - cuts[i] >= target / 2) seg.push_back(cuts[i]);
    seg.push_back(n);
    // CTAs per segment in proportion to its rows (at least one each), then even splits
    const uint32_t nseg = (uint32_t)seg.size() - 1;
    std::vector<uint32_t> k(nseg, 1);
    uint32_t used = nseg;
    while (used < num_ctas) {
        uint32_t best = 0;
        double worst = -1.0;
        for (uint32_t i = 0; i < nseg; ++i) {
            const double per = (double)(seg[i + 1] - seg[i]) / k[i];
            if (per > worst) {
                worst = per;
                best = i;
            }
        }
        ++k[best];
        ++used;
    }
    std::vector<uint32_t> start{0};
    for (uint32_t i = 0; i < nseg; ++i) {
        const uint64_t len = seg[i + 1] - seg[i];
        for (uint32_t j = 1; j <= k[i]; ++j) start.push_back(seg[i] + (uint32_t)(len * j / k[i]));
    }
    std::vector<uint32_t> out{0};  // empty slabs dropped
    for (size_t i = 1; i < start.size(); ++i)
        if (start[i] > out.back()) out.push_back(start[i]);
    return out;
}

// ============================================================================
// Triangular preconditioners in device layout
// ============================================================================
namespace {
template <typename Low>
void widen_csr(const CsrT<Low>& in, CsrT<double>& out) {
    out.n = in.n;
    out.rowptr = in.rowptr;
    out.col = in.col;
    out.val.assign(in.val.begin(), in.val.end());
}

}  // namespace

template <typename Low>
void ic_sweeps(const CsrT<Low>& Lt, Sweep<Low>& lo, Sweep<Low>& up) {
    // IC: L^T rows hold the diagonal first.  Lower sweep = gather over L
    // (transpose of the strictly upper part), upper sweep = gather over L^T.
    const uint32_t n = Lt.n;
    std::vector<uint32_t> urp(n + 1, 0), ucol;
    std::vector<Low> uval;
    std::vector<double> dg(n);
    ucol.reserve(Lt.nnz());
    uval.reserve(Lt.nnz());
    for (uint32_t i = 0; i < n; ++i) {
        dg[i] = (double)Lt.val[Lt.rowptr[i]];
        for (uint32_t k = Lt.rowptr[i] + 1; k < Lt.rowptr[i + 1]; ++k) {
            ucol.push_back(Lt.col[k]);
            uval.push_back(Lt.val[k]);
        }
        urp[i + 1] = (uint32_t)ucol.size();
    }
    std::vector<uint32_t> lrp, lcol;
    std::vector<Low> lval;
    transpose_csr<Low>(n, urp, ucol, uval, lrp, lcol, lval);
    build_sweep<Low>(n, lrp, lcol, lval, &dg, SWEEP_DIV, true, lo);
    build_sweep<Low>(n, urp, ucol, uval, &dg, SWEEP_DIV, false, up);
}

template <typename Low>
void ildlt_sweeps(const CsrT<Low>& Lt, const std::vector<double>& D, Sweep<Low>& lo, Sweep<Low>& up) {
    // ILDLT: unit L^T without diagonal, D separate; D^{-1} folded into the upper sweep.
    const uint32_t n = Lt.n;
    std::vector<uint32_t> lrp, lcol;
    std::vector<Low> lval;
    transpose_csr<Low>(n, Lt.rowptr, Lt.col, Lt.val, lrp, lcol, lval);
    build_sweep<Low>(n, lrp, lcol, lval, nullptr, SWEEP_NONE, true, lo);
    build_sweep<Low>(n, Lt.rowptr, Lt.col, Lt.val, &D, SWEEP_PREDIV, false, up);
}
template <typename Low>
void ilut_sweeps(const CsrT<Low>& L, const CsrT<Low>& U, const std::vector<Low>& Dinv, Sweep<Low>& lo, Sweep<Low>& up) {
    std::vector<double> dd(Dinv.begin(), Dinv.end());
    build_sweep<Low>(L.n, L.rowptr, L.col, L.val, nullptr, SWEEP_NONE, true, lo);
    build_sweep<Low>(U.n, U.rowptr, U.col, U.val, &dd, SWEEP_MUL, false, up);
}
template void ilut_sweeps<double>(const CsrT<double>&, const CsrT<double>&, const std::vector<double>&,
                                  Sweep<double>&, Sweep<double>&);
template void ilut_sweeps<float>(const CsrT<float>&, const CsrT<float>&, const std::vector<float>&, Sweep<float>&,
                                 Sweep<float>&);
template void ic_sweeps<double>(const CsrT<double>&, Sweep<double>&, Sweep<double>&);
template void ic_sweeps<float>(const CsrT<float>&, Sweep<float>&, Sweep<float>&);
template void ildlt_sweeps<double>(const CsrT<double>&, const std::vector<double>&, Sweep<double>&, Sweep<double>&);
template void ildlt_sweeps<float>(const CsrT<float>&, const std::vector<double>&, Sweep<float>&, Sweep<float>&);

void factor_index_sweeps(const HostFactor& f, Sweep<double>& lo, Sweep<double>& up) {
    CsrT<double> Lt;
    Lt.n = f.f0.n;
    Lt.rowptr = f.f0.rowptr;
    Lt.col = f.f0.col;
    Lt.val.resize(f.f0.col.size());
    for (size_t e = 0; e < Lt.val.size(); ++e) Lt.val[e] = (double)e;
    if (f.kind == 1) {
        ic_sweeps<double>(Lt, lo, up);
    } else {
        std::vector<double> rows(Lt.n);
        for (uint32_t r = 0; r < Lt.n; ++r) rows[r] = (double)r;
        ildlt_sweeps<double>(Lt, rows, lo, up);
    }
}

namespace {
template <typename Low>
int build_tri_t(int kind, const CsrHost& A, double tol, uint32_t lfill, HostFactor& F, Sweep<Low>& lo,
                Sweep<Low>& up, std::string* err) {
    const uint32_t n = A.n;
    if (kind == 1) {
        // IC: L^T rows hold the diagonal first.  Lower sweep = gather over L
        // (transpose of the strictly upper part), upper sweep = gather over L^T.
        CsrT<Low> Lt;
        auto plan = std::make_shared<RefactorPlan>();
        int rc = ict_factor<Low>(A, tol, Lt, err, plan.get());
        if (rc) return rc;
        F.plan = plan;
        ic_sweeps<Low>(Lt, lo, up);
        F.mnnz = Lt.nnz() * 2 + n;  // IncompleteCholesky.cpp:245
        widen_csr(Lt, F.f0);
        return 0;
    }
    if (kind == 3) {
        // ILDLT: unit L^T without diagonal, D separate; D^{-1} folded into the upper sweep.
        CsrT<Low> Lt;
        std::vector<double> D;
        auto plan = std::make_shared<RefactorPlan>();
        int rc = ildlt_factor<Low>(A, tol, Lt, D, err, plan.get());
        if (rc) return rc;
        F.plan = plan;
        ildlt_sweeps<Low>(Lt, D, lo, up);
        F.mnnz = Lt.nnz() * 2 + n;  // IncompleteLDLT.cpp:185
        widen_csr(Lt, F.f0);
        F.diag = D;
        return 0;
    }
    if (kind == 2) {
        CsrT<Low> L, U;
        std::vector<Low> Dinv;
        int rc = ilut_factor<Low>(A, lfill, tol, L, U, Dinv, err);
        if (rc) return rc;
        std::vector<double> dd(Dinv.begin(), Dinv.end());
        ilut_sweeps<Low>(L, U, Dinv, lo, up);
        F.mnnz = L.nnz() + U.nnz() + n;  // IncompleteLU.cpp:264
        widen_csr(L, F.f0);
        widen_csr(U, F.f1);
        F.diag = dd;
        return 0;
    }
    if (err) *err = "unknown triangular preconditioner kind " + std::to_string(kind);
    return SETUP_BAD_INPUT;
}
}  // namespace

int build_triangular(int kind, const CsrHost& A, double tol, uint32_t lfill, bool fp32, HostFactor& out,
                     std::string* err) {
    out = HostFactor();
    out.kind = kind;
    out.fp32 = fp32;
    if (fp32) return build_tri_t<float>(kind, A, tol, lfill, out, out.lower32, out.upper32, err);
    return build_tri_t<double>(kind, A, tol, lfill, out, out.lower64, out.upper64, err);
}

namespace {
// Positions for the entries of a group of rows that one shared-memory wavefront serves.
// rows[i] lists (slot, source index) pairs; every row gets exactly P positions (entries
// plus padding).  Position by position the rows take entries whose slots fall in banks no
// other row uses there (the same slot twice is a broadcast, not a conflict); a row whose
// remaining entries just fill its remaining positions must take one even if its bank is
// taken.  Padding reads the zero slot of a bank left free (slot b holds 0.0 and sits in
// bank b).  out[i][u] = index into rows[i] or -(1 + zero slot).
void bank_order(const std::vector<std::vector<std::pair<uint32_t, uint32_t>>>& rows, uint32_t P, uint32_t nb,
                std::vector<std::vector<int64_t>>& out) {
    const size_t G = rows.size();
    out.assign(G, std::vector<int64_t>(P, 0));
    std::vector<std::vector<uint8_t>> taken(G);
    std::vector<uint32_t> left(G);
    for (size_t i = 0; i < G; ++i) {
        taken[i].assign(rows[i].size(), 0);
        left[i] = (uint32_t)rows[i].size();
    }
    std::vector<size_t> idx(G);
    std::vector<int64_t> bank_slot(nb);
    std::vector<uint8_t> padded(G);
    for (uint32_t u = 0; u < P; ++u) {
        std::fill(bank_slot.begin(), bank_slot.end(), -1);
        std::iota(idx.begin(), idx.end(), 0);
        // most constrained rows first: least slack between positions left and entries left
        std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return left[a] > left[b]; });
        for (size_t t = 0; t < G; ++t) {
            const size_t i = idx[t];
            padded[i] = 0;
            if (left[i] == 0) {
                padded[i] = 1;
                continue;
            }
            const bool must = left[i] >= P - u;
            int64_t pick = -1;
            for (size_t e = 0; e < rows[i].size() && pick < 0; ++e) {
                if (taken[i][e]) continue;
                const uint32_t sl = rows[i][e].first, b = sl % nb;
                if (bank_slot[b] < 0 || bank_slot[b] == (int64_t)sl) pick = (int64_t)e;
            }
            if (pick < 0 && must)
                for (size_t e = 0; e < rows[i].size(); ++e)
                    if (!taken[i][e]) {
                        pick = (int64_t)e;
                        break;
                    }
            if (pick < 0) {
                padded[i] = 1;
                continue;
            }
            taken[i][(size_t)pick] = 1;
            --left[i];
            const uint32_t sl = rows[i][(size_t)pick].first;
            if (bank_slot[sl % nb] < 0) bank_slot[sl % nb] = sl;
            out[i][u] = pick;
        }
        for (size_t i = 0; i < G; ++i) {
            if (!padded[i]) continue;
            uint32_t b = 0;
            while (b < nb && bank_slot[b] >= 0 && bank_slot[b] != (int64_t)b) ++b;
            if (b == nb) b = 0;  // every bank taken: the zero slot of bank 0 (a conflict at worst)
            if (bank_slot[b] < 0) bank_slot[b] = b;
            out[i][u] = -1 - (int64_t)b;
        }
    }
}
}  // namespace

template <typename Low>
bool stream_layout(const Sweep<Low>& s, const std::vector<uint32_t>& start, uint32_t max_slots, uint32_t slot_bytes,
                   StreamLayout& out, std::string* why, StreamOrder* order, std::vector<uint32_t>* coef_map,
                   uint32_t max_round_bytes) {
    auto fail = [&](const std::string& m) {
        if (why) *why = m;
        return false;
    };
    const uint32_t n = s.n;
    if (n == 0 || start.size() < 2) return fail("empty sweep");
    if (slot_bytes != 4 && slot_bytes != 8) return fail("slot width");
    const uint32_t num_ctas = (uint32_t)start.size() - 1;
    if (start[0] != 0 || start[num_ctas] != n) return fail("slabs do not cover the rows");
    for (uint32_t b = 0; b < num_ctas; ++b) {
        if (start[b + 1] <= start[b]) return fail("a slab without rows");
        if (start[b + 1] - start[b] > 0xFFFFu) return fail("slab larger than 65535 rows");
    }
    if (max_slots > kNoSlot) max_slots = kNoSlot;
    const uint32_t NZ = zero_slots(slot_bytes);
    if (max_slots <= NZ) return fail("no room for value slots");
    Sweep<Low> sl;
    std::vector<uint32_t> cpos;
    slab_layout_ranges<Low>(s, start, cpos, sl);
    // coef_map: which entry of s each entry of the slab-ordered copy is
    std::vector<uint32_t> sweep_entry;
    if (coef_map) {
        coef_map->clear();
        Sweep<double> si;
        si.n = s.n;
        si.op = s.op;
        si.lower = s.lower;
        si.num_levels = s.num_levels;
        si.level_ptr = s.level_ptr;
        si.order = s.order;
        si.rowptr = s.rowptr;
        si.col = s.col;
        si.diag = s.diag;
        si.level = s.level;
        si.val.resize(s.val.size());
        for (size_t e = 0; e < si.val.size(); ++e) si.val[e] = (double)e;
        Sweep<double> sli;
        std::vector<uint32_t> cp2;
        slab_layout_ranges<double>(si, start, cp2, sli);
        sweep_entry.resize(sli.val.size());
        for (size_t e = 0; e < sli.val.size(); ++e) sweep_entry[e] = (uint32_t)sli.val[e];
    }
    const uint32_t vb = (uint32_t)sizeof(Low);
    const bool recip = s.op == SWEEP_DIV || s.op == SWEEP_PREDIV;
    out = StreamLayout();
    out.num_ctas = num_ctas;
    out.slot_bytes = slot_bytes;
    out.slab_start = start;
    out.cta_pos = cpos;
    out.cta_round.assign((size_t)num_ctas + 1, 0);
    out.in_slot.assign(n, 0);
    out.halo_ptr.assign(1, 0);
    if (order) {
        order->eptr.assign((size_t)n + 1, 0);
        order->kptr.assign((size_t)n + 1, 0);
        order->diag.assign(n, 1.0);
        for (uint32_t p = 0; p < n; ++p) order->diag[s.order[p]] = s.diag[p];
        order->op = s.op;
        order->lower = s.lower;
    }
    // per row: its (early, late) summation order, filled round by round, gathered at the end
    std::vector<std::vector<std::pair<uint32_t, double>>> ord_e, ord_k;
    if (order) {
        ord_e.resize(n);
        ord_k.resize(n);
    }

    struct Round {
        uint32_t p0, p1;
        std::vector<uint32_t> xrow, xslot, xwait;
    };
    constexpr uint32_t kNone = 0xFFFFFFFFu;
    std::vector<uint32_t> round_of(n, kNone);  // by row: its round in its slab (each slab reads its own rows only)
    // Per-thread scratch: rows a slab reads include other slabs' (halo) rows, so what a slab
    // records about a row lives in its thread's arrays, tagged with the slab.
    struct Scratch {
        std::vector<uint32_t> seen;      // by row: slab that last read it ...
        std::vector<int64_t> last_use;   // ... and the last round of that slab reading it
        std::vector<uint32_t> slot_of;   // by row: its value slot in the slab being laid out
        std::vector<uint32_t> slot_in;   // by row: slab that slot_of refers to
    };
    // What one slab contributes, with blob positions relative to its own records; the slabs
    // are then concatenated in order, so the layout does not depend on the threads.
    struct SlabOut {
        std::string err;
        std::vector<uint8_t> blob;
        std::vector<uint32_t> meta, halo_row, halo_sw, halo_cnt, cmap;
        uint32_t rounds = 0, slots = 0, max_round_bytes = 0;
    };
    std::vector<SlabOut> parts(num_ctas);
    const uint32_t G = slot_bytes == 4 ? 32u : 16u;  // rows one wavefront serves
    auto lay_slab = [&](uint32_t b, Scratch& sc, SlabOut& so) -> bool {
        auto fail = [&](const std::string& m) {
            so.err = m;
            return false;
        };
        std::vector<uint32_t>& seen = sc.seen;
        std::vector<int64_t>& last_use = sc.last_use;
        std::vector<uint32_t>& slot_of = sc.slot_of;
        std::vector<uint32_t>& slot_in = sc.slot_in;
        const uint32_t rb = start[b], re = start[b + 1];
        const uint32_t P0 = cpos[b], P1 = cpos[b + 1];
        std::vector<Round> R;
        // 1. rounds: consecutive positions, at most kRoundRows, no dependency inside a round.
        // With a record cap, each row's early and late entries are counted as step 4 will
        // (late: slab rows of the kStreamLate rounds before) and the record's size
        // (round_rec) is checked before the row joins.
        const uint32_t vbytes = (uint32_t)sizeof(Low);
        for (uint32_t p = P0; p < P1;) {
            Round rd;
            rd.p0 = p;
            const uint32_t id = (uint32_t)R.size();
            uint32_t maxE = 0, maxK = 0;
            while (p < P1 && p - rd.p0 < kRoundRows) {
                bool clash = false;
                uint32_t e = 0, kk = 0;
                for (uint32_t k = sl.rowptr[p]; k < sl.rowptr[p + 1] && !clash; ++k) {
                    const uint32_t d = sl.col[k];
                    const bool in_slab = d >= rb && d < re;
                    clash = in_slab && round_of[d] == id;
                    if (in_slab && round_of[d] < id && round_of[d] + kStreamLate >= id) ++kk;
                    else ++e;
                }
                if (clash) break;
                const uint32_t E2 = std::max(maxE, e), K2 = std::max(maxK, kk);
                if (max_round_bytes && p > rd.p0) {
                    const uint32_t Eg = std::max((E2 + 3) / 4, stream_early_groups(slot_bytes));
                    const uint32_t Kg = std::max<uint32_t>((K2 + 3) / 4, 1);
                    if (round_rec(p - rd.p0 + 1, Eg, Kg, vbytes, slot_bytes).bytes > max_round_bytes) break;
                }
                maxE = E2;
                maxK = K2;
                round_of[sl.order[p]] = id;
                ++p;
            }
            rd.p1 = p;
            R.push_back(std::move(rd));
        }
        if (R.size() >= 0xFFFFu) return fail("more than 65534 rounds in a slab");
        // 2. last reading round of every value the slab reads (its own rows and halo rows)
        for (uint32_t r = 0; r < R.size(); ++r)
            for (uint32_t p = R[r].p0; p < R[r].p1; ++p)
                for (uint32_t k = sl.rowptr[p]; k < sl.rowptr[p + 1]; ++k) {
                    const uint32_t d = sl.col[k];
                    if (seen[d] != b) {
                        seen[d] = b;
                        last_use[d] = -1;
                    }
                    last_use[d] = std::max<int64_t>(last_use[d], r);
                }
        // 3. slots: a value occupies its slot from the round that writes it (its own round for a
        // slab row, its first reading round for a halo row) through its last reading round.
        // Round r's early entries are read once rounds <= r - kStreamLate - 1 are done and before
        // round r starts, its late ones while round r is computed, so its values are free once
        // round r is done.  A row result of round r may take a slot whose last reader is round
        // r - 1 or earlier.  A halo value read first in round r is copied in once rounds
        // <= r - kStreamLate - 1 are done at the latest: its slot's last reader must be round
        // r - kStreamLate - 1 or earlier.  Oldest released slot first.
        std::vector<uint32_t> free_q;
        size_t free_head = 0;
        std::vector<int64_t> slot_last(NZ, INT64_MAX);  // slots 0 .. NZ-1 hold 0.0
        std::vector<std::vector<uint32_t>> release(R.size());
        auto take = [&](int64_t last, uint32_t& slot, uint32_t& wait, int64_t free_by) -> bool {
            if (free_head < free_q.size() && slot_last[free_q[free_head]] <= free_by) {
                slot = free_q[free_head++];
            } else {
                if (slot_last.size() >= max_slots) return false;
                slot = (uint32_t)slot_last.size();
                slot_last.push_back(-1);
            }
            wait = (uint32_t)(slot_last[slot] + 1);  // rounds to finish before the slot is overwritten
            slot_last[slot] = last;
            release[(size_t)last].push_back(slot);
            return true;
        };
        for (uint32_t r = 0; r < R.size(); ++r) {
            if (r > 0)
                for (uint32_t q : release[r - 1]) free_q.push_back(q);
            for (uint32_t p = R[r].p0; p < R[r].p1; ++p)
                for (uint32_t k = sl.rowptr[p]; k < sl.rowptr[p + 1]; ++k) {
                    const uint32_t d = sl.col[k];
                    if ((d >= rb && d < re) || slot_in[d] == b) continue;
                    uint32_t slot, wait;
                    if (!take(last_use[d], slot, wait, (int64_t)r - kStreamLate - 1))
                        return fail("more value slots than shared memory holds");
                    if (r >= kStreamLate ? wait > r - kStreamLate : wait > 0)
                        return fail("a prefetch would wait on a later round");
                    slot_of[d] = slot;
                    slot_in[d] = b;
                    R[r].xrow.push_back(d);
                    R[r].xslot.push_back(slot);
                    R[r].xwait.push_back(wait);
                }
            for (uint32_t p = R[r].p0; p < R[r].p1; ++p) {
                const uint32_t row = sl.order[p];
                if (seen[row] == b && last_use[row] > (int64_t)r) {
                    uint32_t slot, wait;
                    if (!take(last_use[row], slot, wait, (int64_t)r - 1))
                        return fail("more value slots than shared memory holds");
                    if (wait > r) return fail("a slot reused inside its round");
                    slot_of[row] = slot;
                    slot_in[row] = b;
                }
            }
        }
        so.slots = (uint32_t)slot_last.size();
        so.rounds = (uint32_t)R.size();
        // 4. records of this slab's rounds
        for (uint32_t r = 0; r < R.size(); ++r) {
            const Round& rd = R[r];
            const uint32_t nr = rd.p1 - rd.p0;
            // early / late entries of each row: (slot, index of the entry in the sweep)
            std::vector<std::vector<std::pair<uint32_t, uint32_t>>> ear(nr), lat(nr);
            uint32_t E = 0, K = 0;
            for (uint32_t p = rd.p0; p < rd.p1; ++p) {
                const uint32_t j = p - rd.p0;
                for (uint32_t k = sl.rowptr[p]; k < sl.rowptr[p + 1]; ++k) {
                    const uint32_t d = sl.col[k];
                    if (slot_in[d] != b || slot_of[d] < NZ || slot_of[d] == kNoSlot)
                        return fail("a dependency without a value slot");
                    const bool late = d >= rb && d < re && round_of[d] < r && round_of[d] + kStreamLate >= r;
                    (late ? lat : ear)[j].emplace_back(slot_of[d], k);
                }
                E = std::max<uint32_t>(E, (uint32_t)ear[j].size());
                K = std::max<uint32_t>(K, (uint32_t)lat[j].size());
            }
            const uint32_t Eg = std::max((E + 3) / 4, stream_early_groups(slot_bytes));
            const uint32_t Kg = std::max<uint32_t>((K + 3) / 4, 1);
            if (Eg > 255 || Kg > 255) return fail("a row with more than 1020 entries");
            const RoundRec rec = round_rec(nr, Eg, Kg, vb, slot_bytes);
            const uint64_t off = so.blob.size();  // relative to the slab's records until assembled
            so.blob.resize(off + rec.bytes, 0);
            uint8_t* base = so.blob.data() + off;
            for (uint32_t p = rd.p0; p < rd.p1; ++p) {
                const uint32_t j = p - rd.p0, row = sl.order[p];
                const uint32_t os = seen[row] == b && slot_in[row] == b && last_use[row] > (int64_t)r ? slot_of[row]
                                                                                                      : kNoSlot;
                const uint32_t lo = (row - rb) | (os << 16);
                const double dg = recip ? 1.0 / sl.diag[p] : sl.diag[p];  // divisions become products
                uint8_t* f = base + rec.fld + 16u * j;
                if (slot_bytes == 4) {
                    const float dgf = (float)dg;
                    std::memcpy(f + 4, &dgf, 4);
                    std::memcpy(f + 8, &lo, 4);
                    out.in_slot[row] = (uint32_t)((off + rec.fld + 16u * j) / 4);
                } else {
                    std::memcpy(f + 8, &dg, 8);
                    std::memcpy(base + rec.lo + 4u * j, &lo, 4);
                    out.in_slot[row] = (uint32_t)((off + rec.fld + 16u * j) / 8);
                }
            }
            // entry order, one wavefront's rows at a time
            auto place = [&](std::vector<std::vector<std::pair<uint32_t, uint32_t>>>& ent, uint32_t groups,
                             uint32_t sec_s, uint32_t sec_c, std::vector<std::vector<std::pair<uint32_t, double>>>* ord) {
                const uint32_t Pn = 4 * groups;
                if (!Pn) return;
                for (uint32_t g0 = 0; g0 < nr; g0 += G) {
                    const uint32_t g1 = std::min(nr, g0 + G);
                    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> rows(ent.begin() + g0, ent.begin() + g1);
                    std::vector<std::vector<int64_t>> pos;
                    bank_order(rows, Pn, NZ, pos);
                    for (uint32_t j = g0; j < g1; ++j) {
                        const uint32_t row = sl.order[rd.p0 + j];
                        for (uint32_t u = 0; u < Pn; ++u) {
                            const int64_t e = pos[j - g0][u];
                            uint16_t slot;
                            Low coef;
                            uint32_t dep = kNone;
                            if (e >= 0) {
                                const auto& pr = rows[j - g0][(size_t)e];
                                slot = (uint16_t)pr.first;
                                coef = sl.val[pr.second];
                                dep = sl.col[pr.second];
                                if (coef_map) {
                                    const uint64_t at = off + sec_c + 4u * vb * ((size_t)(u / 4) * rec.m + j) + vb * (u % 4);
                                    so.cmap.push_back((uint32_t)(at / vb));
                                    so.cmap.push_back(sweep_entry[pr.second]);
                                }
                            } else {
                                slot = (uint16_t)(-1 - e);
                                coef = (Low)0;
                            }
                            const uint32_t gi = u / 4, ci = u % 4;
                            std::memcpy(base + sec_s + 8u * ((size_t)gi * rec.m + j) + 2u * ci, &slot, 2);
                            std::memcpy(base + sec_c + 4u * vb * ((size_t)gi * rec.m + j) + vb * ci, &coef, vb);
                            if (ord) (*ord)[row].emplace_back(dep, (double)coef);
                        }
                    }
                }
            };
            place(ear, Eg, rec.es, rec.ec, order ? &ord_e : nullptr);
            place(lat, Kg, rec.ls, rec.lc, order ? &ord_k : nullptr);
            const uint32_t X = (uint32_t)rd.xrow.size();
            for (uint32_t x = 0; x < X; ++x) {
                so.halo_row.push_back(rd.xrow[x]);
                so.halo_sw.push_back(rd.xslot[x] | (rd.xwait[x] << 16));
            }
            so.halo_cnt.push_back(X);
            so.meta.push_back((uint32_t)(off / 16));
            so.meta.push_back(rec.bytes);
            so.meta.push_back(nr | (Eg << 8) | (Kg << 16) | ((X > 0 ? 1u : 0u) << 24));
            so.meta.push_back(0);
            so.max_round_bytes = std::max(so.max_round_bytes, rec.bytes);
        }
        return true;
    };
    // the slabs on a few host threads, each with its own scratch
    {
        unsigned hc = std::max(1u, std::thread::hardware_concurrency());
        if (const char* e = std::getenv("PRISM_LAYOUT_THREADS")) hc = (unsigned)std::max(1, std::atoi(e));
        const unsigned T = num_ctas < 8 ? 1u : std::min<unsigned>(std::min(hc, 16u), num_ctas);
        std::atomic<uint32_t> next{0};
        auto worker = [&]() {
            Scratch sc;
            sc.seen.assign(n, kNone);
            sc.last_use.assign(n, -1);
            sc.slot_of.assign(n, kNoSlot);
            sc.slot_in.assign(n, kNone);
            for (uint32_t b = next++; b < num_ctas; b = next++) lay_slab(b, sc, parts[b]);
        };
        if (T == 1) {
            worker();
        } else {
            std::vector<std::thread> pool;
            for (unsigned t = 0; t < T; ++t) pool.emplace_back(worker);
            for (auto& th : pool) th.join();
        }
    }
    // assembly, slab by slab
    for (uint32_t b = 0; b < num_ctas; ++b) {
        SlabOut& so = parts[b];
        if (!so.err.empty()) return fail(so.err);
        const uint64_t base = out.blob.size();
        if ((base + so.blob.size()) / 16 > 0xFFFFFFFFull || (base + so.blob.size()) / slot_bytes > 0xFFFFFFFFull)
            return fail("round records beyond the addressable blob");
        out.blob.insert(out.blob.end(), so.blob.begin(), so.blob.end());
        for (size_t t = 0; t < so.meta.size(); t += 4) {
            out.meta.push_back(so.meta[t] + (uint32_t)(base / 16));
            out.meta.push_back(so.meta[t + 1]);
            out.meta.push_back(so.meta[t + 2]);
            out.meta.push_back(so.meta[t + 3]);
        }
        size_t h = 0;
        for (uint32_t c : so.halo_cnt) {
            for (uint32_t x = 0; x < c; ++x, ++h) {
                out.halo_row.push_back(so.halo_row[h]);
                out.halo_sw.push_back(so.halo_sw[h]);
            }
            out.halo_ptr.push_back((uint32_t)out.halo_row.size());
        }
        for (uint32_t row = start[b]; row < start[b + 1]; ++row) out.in_slot[row] += (uint32_t)(base / slot_bytes);
        if (coef_map)
            for (size_t t = 0; t < so.cmap.size(); t += 2) {
                coef_map->push_back(so.cmap[t] + (uint32_t)(base / vb));
                coef_map->push_back(so.cmap[t + 1]);
            }
        out.slots = std::max(out.slots, so.slots);
        out.cta_round[b + 1] = out.cta_round[b] + so.rounds;
        out.max_rounds_per_cta = std::max(out.max_rounds_per_cta, so.rounds);
        out.max_round_bytes = std::max(out.max_round_bytes, so.max_round_bytes);
        SlabOut().blob.swap(so.blob);  // release the slab's copy
    }
    out.num_rounds = out.cta_round[num_ctas];
    if (order) {
        for (uint32_t r = 0; r < n; ++r) {
            order->eptr[r + 1] = order->eptr[r] + (uint32_t)ord_e[r].size();
            order->kptr[r + 1] = order->kptr[r] + (uint32_t)ord_k[r].size();
        }
        order->edep.reserve(order->eptr[n]);
        order->ecoef.reserve(order->eptr[n]);
        order->kdep.reserve(order->kptr[n]);
        order->kcoef.reserve(order->kptr[n]);
        for (uint32_t r = 0; r < n; ++r) {
            for (const auto& e : ord_e[r]) {
                order->edep.push_back(e.first);
                order->ecoef.push_back(e.second);
            }
            for (const auto& e : ord_k[r]) {
                order->kdep.push_back(e.first);
                order->kcoef.push_back(e.second);
            }
        }
    }
    return true;
}

namespace {
template <typename A>
struct Arith;
template <>
struct Arith<float> {
    static float fma(float a, float b, float c) { return std::fmaf(a, b, c); }
};
template <>
struct Arith<double> {
    static double fma(double a, double b, double c) { return std::fma(a, b, c); }
};

// One row's sum and result in the kernel's arithmetic (Acc: float or double; -ffp-contract=off
// keeps every other operation a separate rounding).
template <typename Acc>
Acc row_result(int op, Acc vin, Acc dg, const Acc* ex, const Acc* ec, uint32_t ne, const Acc* kx, const Acc* kc,
               uint32_t nk) {
    Acc c[4] = {(Acc)0, (Acc)0, (Acc)0, (Acc)0};
    for (uint32_t u = 0; u < ne; ++u) c[u & 3] = Arith<Acc>::fma(ec[u], ex[u], c[u & 3]);
    Acc s = (c[0] + c[1]) + (c[2] + c[3]);
    for (uint32_t k = 0; k < nk; ++k) s = Arith<Acc>::fma(kc[k], kx[k], s);
    if (op == SWEEP_DIV || op == SWEEP_MUL) return (vin - s) * dg;
    if (op == SWEEP_NONE) return vin - s;
    return vin * dg - s;
}

template <typename Low, typename Acc>
std::string replay_impl(const Sweep<Low>& s, const StreamLayout& L, const double* in, double* out) {
    const uint32_t n = s.n;
    const uint32_t vb = (uint32_t)sizeof(Low), ab = (uint32_t)sizeof(Acc);
    const uint32_t NZ = zero_slots(ab);
    const bool recip = s.op == SWEEP_DIV || s.op == SWEEP_PREDIV;
    std::vector<uint8_t> blob = L.blob;
    if (L.in_slot.size() != n) return "in_slot size";
    for (uint32_t r = 0; r < n; ++r) {
        if ((uint64_t)L.in_slot[r] * ab + ab > blob.size()) return "in_slot beyond the blob";
        const Acc v = (Acc)in[r];
        std::memcpy(blob.data() + (uint64_t)L.in_slot[r] * ab, &v, ab);
    }
    if (L.halo_ptr.size() != (size_t)L.num_rounds + 1 || L.halo_ptr.back() != L.halo_row.size() ||
        L.halo_sw.size() != L.halo_row.size())
        return "halo list sizes";
    std::vector<uint32_t> pos_of(n);
    for (uint32_t p = 0; p < n; ++p) pos_of[s.order[p]] = p;
    std::vector<uint8_t> done(n, 0);
    std::vector<Acc> val(n, (Acc)0);   // finished results in the kernel's type
    std::vector<uint32_t> rnd(n, 0);   // round of its slab in which a row was computed
    struct Cta {
        uint32_t next = 0;             // next round to compute
        uint32_t copied = 0;           // halo copies made (in order)
        std::vector<Acc> xs;
        std::vector<int64_t> owner;    // row whose value the slot holds (-1: none, -2: zero)
    };
    std::vector<Cta> ctas(L.num_ctas);
    for (Cta& c : ctas) {
        c.xs.assign(L.slots, (Acc)0);
        c.owner.assign(L.slots, -1);
        for (uint32_t z = 0; z < NZ && z < L.slots; ++z) c.owner[z] = -2;
    }
    struct View {
        uint32_t nr = 0, Eg = 0, Kg = 0, halo = 0;
        RoundRec rec{};
        const uint8_t* base = nullptr;
    };
    auto view = [&](uint32_t gr, View& v) -> std::string {
        const uint64_t off = (uint64_t)L.meta[(size_t)gr * 4] * 16;
        const uint32_t bytes = L.meta[(size_t)gr * 4 + 1], shape = L.meta[(size_t)gr * 4 + 2];
        v.nr = shape & 0xFFu;
        v.Eg = (shape >> 8) & 0xFFu;
        v.Kg = (shape >> 16) & 0xFFu;
        v.halo = shape >> 24;
        v.rec = round_rec(v.nr, v.Eg, v.Kg, vb, ab);
        if (off % 16 || v.rec.bytes != bytes || off + bytes > blob.size() || bytes > L.max_round_bytes)
            return "round record outside the blob";
        if (v.nr == 0 || v.nr > kRoundRows) return "round size";
        if ((v.halo != 0) != (L.halo_ptr[gr + 1] > L.halo_ptr[gr])) return "halo flag";
        v.base = blob.data() + off;
        return std::string();
    };
    auto rd16 = [](const uint8_t* p) { uint16_t v; std::memcpy(&v, p, 2); return v; };
    auto rd32 = [](const uint8_t* p) { uint32_t v; std::memcpy(&v, p, 4); return v; };
    // entries of row j of a round in one section pair: slots and coefficients by position
    auto entries = [&](const View& v, uint32_t j, uint32_t groups, uint32_t ss, uint32_t sc, std::vector<uint32_t>& sl,
                       std::vector<Acc>& cf) {
        sl.clear();
        cf.clear();
        for (uint32_t u = 0; u < 4 * groups; ++u) {
            const size_t e = (size_t)(u / 4) * v.rec.m + j;
            sl.push_back(rd16(v.base + ss + 8 * e + 2 * (u % 4)));
            Low c;
            std::memcpy(&c, v.base + sc + 4 * vb * e + vb * (u % 4), vb);
            cf.push_back((Acc)c);
        }
    };
    uint32_t finished = 0;
    const uint32_t total = L.num_rounds;
    std::vector<uint32_t> sl;
    std::vector<Acc> cf;
    while (finished < total) {
        bool progress = false;
        for (uint32_t b = 0; b < L.num_ctas; ++b) {
            Cta& c = ctas[b];
            const uint32_t rb = L.slab_start[b];
            if (rb >= n) return "a slab beyond the rows";
            const uint32_t owned = L.slab_start[b + 1] - rb;
            const uint32_t g0 = L.cta_round[b], R = L.cta_round[b + 1] - g0;
            // halo copies as early as their waits allow (rounds of this slab done >= wait and
            // the halo row finished), in order
            const uint32_t hbeg = L.halo_ptr[g0], hend = L.halo_ptr[g0 + R];
            while (hbeg + c.copied < hend) {
                const uint32_t x = hbeg + c.copied, row = L.halo_row[x];
                const uint32_t slot = L.halo_sw[x] & 0xFFFFu, wait = L.halo_sw[x] >> 16;
                if (row >= n) return "halo row out of range";
                if (row >= rb && row < rb + owned) return "halo row inside the slab";
                if (slot < NZ || slot >= L.slots) return "halo slot out of range";
                if (c.next < wait || !done[row]) break;
                c.xs[slot] = val[row];
                c.owner[slot] = row;
                ++c.copied;
                progress = true;
            }
            while (c.next < R) {
                const uint32_t r = c.next, gr = g0 + r;
                View v;
                std::string e = view(gr, v);
                if (!e.empty()) return e;
                // round r needs its own halo (its early entries are read once rounds
                // <= r - kStreamLate - 1 are done)
                if (hbeg + c.copied < L.halo_ptr[gr + 1]) break;  // an upstream slab first
                for (uint32_t x = L.halo_ptr[gr]; x < L.halo_ptr[gr + 1]; ++x) {
                    const uint32_t wait = L.halo_sw[x] >> 16;
                    if (r >= kStreamLate ? wait > r - kStreamLate : wait > 0)
                        return "a prefetch waits on its own or a later round";
                }
                // reads of round r (early ones before round r starts, late ones while round r
                // is computed), checked against the slot owners
                std::vector<Acc> res(v.nr);
                std::vector<uint32_t> rows(v.nr);
                std::vector<std::vector<uint32_t>> read_slots(v.nr);
                std::vector<std::vector<int64_t>> read_owner(v.nr);
                for (uint32_t j = 0; j < v.nr; ++j) {
                    const uint8_t* f = v.base + v.rec.fld + 16 * j;
                    const uint32_t lo = ab == 4 ? rd32(f + 8) : rd32(v.base + v.rec.lo + 4 * j);
                    const uint32_t lrow = lo & 0xFFFFu;
                    if (lrow >= owned) return "row outside its slab";
                    const uint32_t row = rb + lrow;
                    rows[j] = row;
                    if (done[row]) return "row visited twice";
                    const uint32_t p = pos_of[row];
                    Acc vin, dg;
                    std::memcpy(&vin, f, ab);
                    std::memcpy(&dg, f + ab, ab);
                    if (dg != (Acc)(recip ? 1.0 / s.diag[p] : s.diag[p])) return "diagonal";
                    // the row's dependencies, each to be found exactly once among its entries
                    std::vector<uint32_t> deps(s.col.begin() + s.rowptr[p], s.col.begin() + s.rowptr[p + 1]);
                    std::vector<Low> cvals(s.val.begin() + s.rowptr[p], s.val.begin() + s.rowptr[p + 1]);
                    std::vector<uint8_t> used(deps.size(), 0);
                    std::vector<Acc> ex, ec, kx, kc;
                    for (int part = 0; part < 2; ++part) {
                        const bool late = part == 1;
                        entries(v, j, late ? v.Kg : v.Eg, late ? v.rec.ls : v.rec.es, late ? v.rec.lc : v.rec.ec,
                                sl, cf);
                        for (size_t u = 0; u < sl.size(); ++u) {
                            const uint32_t slot = sl[u];
                            if (slot >= L.slots) return "dependency slot out of range";
                            const int64_t ow = c.owner[slot];
                            if (ow == -2) {
                                if (cf[u] != (Acc)0) return "padding entry with a coefficient";
                            } else {
                                if (ow < 0) return "a slot read before anything was written to it";
                                size_t t = 0;
                                while (t < deps.size() && (used[t] || deps[t] != (uint32_t)ow || (Acc)cvals[t] != cf[u]))
                                    ++t;
                                if (t == deps.size()) return "a slot does not hold a dependency of the row";
                                used[t] = 1;
                                if (!done[(uint32_t)ow]) return "a dependency read before it was finished";
                                const bool in_slab = (uint32_t)ow >= rb && (uint32_t)ow < rb + owned;
                                if (late) {
                                    if (!in_slab || rnd[(uint32_t)ow] >= r || rnd[(uint32_t)ow] + kStreamLate < r)
                                        return "a late entry not computed in the rounds just before";
                                } else if (in_slab && rnd[(uint32_t)ow] + kStreamLate + 1 > r) {
                                    return "an early entry computed in the rounds just before";
                                }
                            }
                            (late ? kx : ex).push_back(c.xs[slot]);
                            (late ? kc : ec).push_back(cf[u]);
                            read_slots[j].push_back(slot);
                            read_owner[j].push_back(ow);
                        }
                    }
                    for (size_t t = 0; t < deps.size(); ++t)
                        if (!used[t]) return "a dependency missing from the row's entries";
                    res[j] = row_result<Acc>(s.op, vin, dg, ex.data(), ec.data(), (uint32_t)ex.size(), kx.data(),
                                             kc.data(), (uint32_t)kx.size());
                }
                // the round's results, then the race check: a slower warp may still read the
                // round's slots after a faster one wrote its results
                for (uint32_t j = 0; j < v.nr; ++j) {
                    const uint8_t* f = v.base + v.rec.fld + 16 * j;
                    const uint32_t lo = ab == 4 ? rd32(f + 8) : rd32(v.base + v.rec.lo + 4 * j);
                    const uint32_t os = lo >> 16;
                    const uint32_t row = rows[j];
                    val[row] = res[j];
                    out[row] = (double)res[j];
                    done[row] = 1;
                    rnd[row] = r;
                    if (os != kNoSlot) {
                        if (os < NZ || os >= L.slots) return "result slot out of range";
                        c.xs[os] = res[j];
                        c.owner[os] = row;
                    }
                }
                for (uint32_t j = 0; j < v.nr; ++j)
                    for (size_t t = 0; t < read_slots[j].size(); ++t)
                        if (c.owner[read_slots[j][t]] != read_owner[j][t])
                            return "a result overwrites a slot the same round reads";
                ++c.next;
                ++finished;
                progress = true;
                // copies allowed now that one more round is done
                while (hbeg + c.copied < hend) {
                    const uint32_t x = hbeg + c.copied, row = L.halo_row[x];
                    const uint32_t slot = L.halo_sw[x] & 0xFFFFu, wait = L.halo_sw[x] >> 16;
                    if (c.next < wait || !done[row]) break;
                    if (slot < NZ || slot >= L.slots) return "halo slot out of range";
                    c.xs[slot] = val[row];
                    c.owner[slot] = row;
                    ++c.copied;
                }
            }
        }
        if (!progress) return "rounds wait on each other";
    }
    for (uint32_t r = 0; r < n; ++r)
        if (!done[r]) return "row never visited";
    return std::string();
}
}  // namespace

template <typename Low>
std::string stream_layout_replay(const Sweep<Low>& s, const StreamLayout& L, const double* in, double* out) {
    if (L.slot_bytes == 4) {
        if constexpr (std::is_same<Low, float>::value) return replay_impl<Low, float>(s, L, in, out);
        return "4-byte slots need float factor values";
    }
    return replay_impl<Low, double>(s, L, in, out);
}

// ---- explicit instantiations ------------------------------------------------
template int ict_factor<double>(const CsrHost&, double, CsrT<double>&, std::string*, RefactorPlan*);
template int ict_factor<float>(const CsrHost&, double, CsrT<float>&, std::string*, RefactorPlan*);
template int ildlt_factor<double>(const CsrHost&, double, CsrT<double>&, std::vector<double>&, std::string*,
                                  RefactorPlan*);
template int ildlt_factor<float>(const CsrHost&, double, CsrT<float>&, std::vector<double>&, std::string*,
                                 RefactorPlan*);
template int ilut_factor<double>(const CsrHost&, uint32_t, double, CsrT<double>&, CsrT<double>&,
                                 std::vector<double>&, std::string*);
template int ilut_factor<float>(const CsrHost&, uint32_t, double, CsrT<float>&, CsrT<float>&,
                                std::vector<float>&, std::string*);
template void transpose_csr<double>(uint32_t, const std::vector<uint32_t>&, const std::vector<uint32_t>&,
                                    const std::vector<double>&, std::vector<uint32_t>&, std::vector<uint32_t>&,
                                    std::vector<double>&);
template void transpose_csr<float>(uint32_t, const std::vector<uint32_t>&, const std::vector<uint32_t>&,
                                   const std::vector<float>&, std::vector<uint32_t>&, std::vector<uint32_t>&,
                                   std::vector<float>&);
template void slab_layout<double>(const Sweep<double>&, uint32_t, uint32_t, std::vector<uint32_t>&,
                                  Sweep<double>&);
template void slab_layout<float>(const Sweep<float>&, uint32_t, uint32_t, std::vector<uint32_t>&, Sweep<float>&);
template std::vector<uint32_t> slab_ranges<double>(const Sweep<double>&, uint32_t);
template std::vector<uint32_t> slab_ranges<float>(const Sweep<float>&, uint32_t);
template bool stream_layout<double>(const Sweep<double>&, const std::vector<uint32_t>&, uint32_t, uint32_t,
                                    StreamLayout&, std::string*, StreamOrder*, std::vector<uint32_t>*, uint32_t);
template bool stream_layout<float>(const Sweep<float>&, const std::vector<uint32_t>&, uint32_t, uint32_t,
                                   StreamLayout&, std::string*, StreamOrder*, std::vector<uint32_t>*, uint32_t);
template std::string stream_layout_replay<double>(const Sweep<double>&, const StreamLayout&, const double*,
                                                  double*);
template std::string stream_layout_replay<float>(const Sweep<float>&, const StreamLayout&, const double*, double*);
template void pair_sweep<double>(const Sweep<double>&, Sweep<double>&, PairMap&);
template void pair_sweep<float>(const Sweep<float>&, Sweep<float>&, PairMap&);
template void build_sweep<double>(uint32_t, const std::vector<uint32_t>&, const std::vector<uint32_t>&,
                                  const std::vector<double>&, const std::vector<double>*, int, bool, Sweep<double>&);
template void build_sweep<float>(uint32_t, const std::vector<uint32_t>&, const std::vector<uint32_t>&,
                                 const std::vector<float>&, const std::vector<double>*, int, bool, Sweep<float>&);

}  // namespace prism
