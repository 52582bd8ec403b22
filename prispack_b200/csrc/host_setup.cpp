// Host-side setup: model problems, bit-exact incomplete factorisations and the
// exact integer level schedules used by the device sweeps.
#include "host_setup.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

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
int left_looking(const CsrHost& A, double thr, CsrT<Low>& Lt, std::vector<double>* D, std::string* err) {
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

    for (uint32_t j = 0; j < n; ++j) {
        uint32_t cnt = 0;
        double colThr = 0.0;
        // lower part of column j of A (row j, symmetric storage)
        for (uint32_t p = A.rowptr[j]; p < A.rowptr[j + 1]; ++p) {
            const uint32_t i = A.col[p];
            const double a = A.val[p];
            if (i >= j) {
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
int ict_factor(const CsrHost& A, double threshold, CsrT<Low>& Lt, std::string* err) {
    return left_looking<Low, false>(A, threshold, Lt, nullptr, err);
}

template <typename Low>
int ildlt_factor(const CsrHost& A, double tol, CsrT<Low>& Lt, std::vector<double>& D, std::string* err) {
    return left_looking<Low, true>(A, tol, Lt, &D, err);
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

namespace {
template <typename Low>
int build_tri_t(int kind, const CsrHost& A, double tol, uint32_t lfill, HostFactor& F, Sweep<Low>& lo,
                Sweep<Low>& up, std::string* err) {
    const uint32_t n = A.n;
    if (kind == 1) {
        // IC: L^T rows hold the diagonal first.  Lower sweep = gather over L
        // (transpose of the strictly upper part), upper sweep = gather over L^T.
        CsrT<Low> Lt;
        int rc = ict_factor<Low>(A, tol, Lt, err);
        if (rc) return rc;
        ic_sweeps<Low>(Lt, lo, up);
        F.mnnz = Lt.nnz() * 2 + n;  // IncompleteCholesky.cpp:245
        widen_csr(Lt, F.f0);
        return 0;
    }
    if (kind == 3) {
        // ILDLT: unit L^T without diagonal, D separate; D^{-1} folded into the upper sweep.
        CsrT<Low> Lt;
        std::vector<double> D;
        int rc = ildlt_factor<Low>(A, tol, Lt, D, err);
        if (rc) return rc;
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

template <typename Low>
bool stream_layout(const Sweep<Low>& s, const std::vector<uint32_t>& start, uint32_t max_slots, StreamLayout& out,
                   std::string* why) {
    auto fail = [&](const std::string& m) {
        if (why) *why = m;
        return false;
    };
    const uint32_t n = s.n;
    if (n == 0 || start.size() < 2) return fail("empty sweep");
    const uint32_t num_ctas = (uint32_t)start.size() - 1;
    if (start[0] != 0 || start[num_ctas] != n) return fail("slabs do not cover the rows");
    for (uint32_t b = 0; b < num_ctas; ++b) {
        if (start[b + 1] <= start[b]) return fail("a slab without rows");
        if (start[b + 1] - start[b] > 0xFFFFu) return fail("slab larger than 65535 rows");
    }
    if (max_slots > kNoSlot) max_slots = kNoSlot;
    Sweep<Low> sl;
    std::vector<uint32_t> cpos;
    slab_layout_ranges<Low>(s, start, cpos, sl);
    const uint32_t vb = (uint32_t)sizeof(Low);
    const bool recip = s.op == SWEEP_DIV || s.op == SWEEP_PREDIV;
    out = StreamLayout();
    out.num_ctas = num_ctas;
    out.slab_start = start;
    out.cta_pos = cpos;
    out.cta_round.assign((size_t)num_ctas + 1, 0);
    out.in_slot.assign(n, 0);

    struct Round {
        uint32_t p0, p1, L;
        std::vector<uint32_t> xrow, xslot, xwait;
    };
    constexpr uint32_t kNone = 0xFFFFFFFFu;
    std::vector<uint32_t> round_of(n, kNone);   // by row: round of the slab being laid out
    std::vector<uint32_t> seen(n, kNone);       // by row: slab that last read it ...
    std::vector<int64_t> last_use(n, -1);       // ... and the last round of that slab reading it
    std::vector<uint32_t> slot_of(n, kNoSlot);  // by row: its value slot in the slab being laid out
    std::vector<uint32_t> slot_in(n, kNone);    // by row: slab that slot_of refers to
    for (uint32_t b = 0; b < num_ctas; ++b) {
        const uint32_t rb = start[b], re = start[b + 1];
        const uint32_t P0 = cpos[b], P1 = cpos[b + 1];
        std::vector<Round> R;
        // 1. rounds: consecutive positions, at most kRoundRows, no dependency inside a round.
        // A dependency has a lower level, hence an earlier position, so its round is known.
        for (uint32_t p = P0; p < P1;) {
            Round rd;
            rd.p0 = p;
            const uint32_t id = (uint32_t)R.size();
            while (p < P1 && p - rd.p0 < kRoundRows) {
                bool clash = false;
                for (uint32_t k = sl.rowptr[p]; k < sl.rowptr[p + 1] && !clash; ++k) {
                    const uint32_t d = sl.col[k];
                    clash = d >= rb && d < re && round_of[d] == id;
                }
                if (clash) break;
                round_of[sl.order[p]] = id;
                ++p;
            }
            rd.p1 = p;
            rd.L = 0;
            for (uint32_t q = rd.p0; q < rd.p1; ++q) rd.L = std::max(rd.L, sl.rowptr[q + 1] - sl.rowptr[q]);
            if (rd.L > 0xFFFFu) return fail("a row with more than 65535 entries");
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
        // slab row, its first reading round for a halo row) through its last reading round.  A
        // slot released after round r takes a row result of round r + 1 or later; a halo value
        // only from round r + 2 on, because the kernel copies round r + 2's halo in while round
        // r + 1 computes, when only rounds up to r are known to be done.  Oldest first.
        std::vector<uint32_t> free_q;
        size_t free_head = 0;
        std::vector<int64_t> slot_last{INT64_MAX};  // last reading round of the slot's value; slot 0 holds 0.0
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
            // halo rows first read in round r: copied in by a prefetcher
            for (uint32_t p = R[r].p0; p < R[r].p1; ++p)
                for (uint32_t k = sl.rowptr[p]; k < sl.rowptr[p + 1]; ++k) {
                    const uint32_t d = sl.col[k];
                    if ((d >= rb && d < re) || slot_in[d] == b) continue;
                    uint32_t slot, wait;
                    if (!take(last_use[d], slot, wait, (int64_t)r - 2))
                        return fail("more value slots than shared memory holds");
                    if (wait > (r > 0 ? r - 1 : 0)) return fail("a prefetch would wait on its own or a later round");
                    slot_of[d] = slot;
                    slot_in[d] = b;
                    R[r].xrow.push_back(d);
                    R[r].xslot.push_back(slot);
                    R[r].xwait.push_back(wait);
                }
            // rows of round r read later in the slab: their results go to a slot
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
        out.slots = std::max<uint32_t>(out.slots, (uint32_t)slot_last.size());
        out.cta_round[b + 1] = out.cta_round[b] + (uint32_t)R.size();
        out.max_rounds_per_cta = std::max<uint32_t>(out.max_rounds_per_cta, (uint32_t)R.size());
        // 4. records of this slab's rounds
        for (uint32_t r = 0; r < R.size(); ++r) {
            const Round& rd = R[r];
            const uint32_t nr = rd.p1 - rd.p0, X = (uint32_t)rd.xrow.size();
            const RoundRec rec = round_rec(nr, rd.L, X, vb);
            const uint64_t off = out.blob.size();
            if ((off + rec.bytes) / 8 > 0xFFFFFFFFull) return fail("blob beyond 32 GB");
            out.blob.resize(off + rec.bytes, 0);
            uint8_t* base = out.blob.data() + off;
            double* diag = reinterpret_cast<double*>(base + rec.diag);
            uint16_t* lrow = reinterpret_cast<uint16_t*>(base + rec.lrow);
            uint16_t* oslot = reinterpret_cast<uint16_t*>(base + rec.oslot);
            uint8_t* ent = base + rec.ent;
            uint32_t* xrow = reinterpret_cast<uint32_t*>(base + rec.xrow);
            uint16_t* xslot = reinterpret_cast<uint16_t*>(base + rec.xslot);
            uint16_t* xwait = reinterpret_cast<uint16_t*>(base + rec.xwait);
            for (uint32_t p = rd.p0; p < rd.p1; ++p) {
                const uint32_t j = p - rd.p0, row = sl.order[p];
                diag[j] = recip ? 1.0 / sl.diag[p] : sl.diag[p];  // divisions become products
                lrow[j] = (uint16_t)(row - rb);
                oslot[j] = (uint16_t)(slot_in[row] == b && seen[row] == b && last_use[row] > (int64_t)r
                                          ? slot_of[row] : kNoSlot);
                out.in_slot[row] = (uint32_t)((off + rec.in) / 8 + j);
                for (uint32_t k = sl.rowptr[p]; k < sl.rowptr[p + 1]; ++k) {
                    const uint32_t d = sl.col[k], e = (k - sl.rowptr[p]) * rec.m + j;
                    if (slot_in[d] != b || slot_of[d] == 0) return fail("a dependency without a value slot");
                    if (vb == 4) {  // {u32 slot, f32 value}
                        const uint32_t slot = slot_of[d];
                        std::memcpy(ent + (size_t)e * 8, &slot, 4);
                        std::memcpy(ent + (size_t)e * 8 + 4, &sl.val[k], 4);
                    } else {        // u16 slot; f64 value in the value section
                        const uint16_t slot = (uint16_t)slot_of[d];
                        std::memcpy(ent + (size_t)e * 2, &slot, 2);
                        std::memcpy(base + rec.val + (size_t)e * 8, &sl.val[k], 8);
                    }
                }
            }
            for (uint32_t x = 0; x < X; ++x) {
                xrow[x] = rd.xrow[x];
                xslot[x] = (uint16_t)rd.xslot[x];
                xwait[x] = (uint16_t)rd.xwait[x];
            }
            out.meta.push_back((uint32_t)(off / 16));
            out.meta.push_back(rec.bytes);
            out.meta.push_back(nr | (rd.L << 16));
            out.meta.push_back(X);
            out.max_round_bytes = std::max(out.max_round_bytes, rec.bytes);
        }
    }
    out.num_rounds = out.cta_round[num_ctas];
    return true;
}

template <typename Low>
std::string stream_layout_replay(const Sweep<Low>& s, const StreamLayout& L, const double* in, double* out) {
    const uint32_t n = s.n;
    const uint32_t vb = (uint32_t)sizeof(Low);
    const bool recip = s.op == SWEEP_DIV || s.op == SWEEP_PREDIV;
    std::vector<uint8_t> blob = L.blob;
    if (L.in_slot.size() != n) return "in_slot size";
    for (uint32_t r = 0; r < n; ++r) {
        if ((uint64_t)L.in_slot[r] * 8 + 8 > blob.size()) return "in_slot beyond the blob";
        std::memcpy(blob.data() + (uint64_t)L.in_slot[r] * 8, in + r, 8);
    }
    std::vector<uint32_t> pos_of(n);
    for (uint32_t p = 0; p < n; ++p) pos_of[s.order[p]] = p;
    std::vector<uint8_t> done(n, 0);
    struct Cta {
        uint32_t next = 0;
        std::vector<double> xs;
        std::vector<int64_t> owner;  // row whose value the slot holds (-1: none)
    };
    std::vector<Cta> ctas(L.num_ctas);
    for (Cta& c : ctas) {
        c.xs.assign(L.slots, 0.0);
        c.owner.assign(L.slots, -1);
    }
    uint32_t finished = 0;
    const uint32_t total = L.cta_round[L.num_ctas];
    while (finished < total) {
        bool progress = false;
        for (uint32_t b = 0; b < L.num_ctas; ++b) {
            Cta& c = ctas[b];
            const uint32_t rb = L.slab_start[b];
            if (rb >= n) return "a slab beyond the rows";
            const uint32_t owned = L.slab_start[b + 1] - rb;
            const uint32_t R = L.cta_round[b + 1] - L.cta_round[b];
            while (c.next < R) {
                const uint32_t r = c.next, gr = L.cta_round[b] + r;
                const uint64_t off = (uint64_t)L.meta[(size_t)gr * 4] * 16;
                const uint32_t bytes = L.meta[(size_t)gr * 4 + 1], nr = L.meta[(size_t)gr * 4 + 2] & 0xFFFFu,
                               Lr = L.meta[(size_t)gr * 4 + 2] >> 16, X = L.meta[(size_t)gr * 4 + 3];
                const RoundRec rec = round_rec(nr, Lr, X, vb);
                if (off % 16 || rec.bytes != bytes || off + bytes > blob.size() || bytes > L.max_round_bytes)
                    return "round record outside the blob";
                if (nr == 0 || nr > kRoundRows) return "round size";
                const uint8_t* base = blob.data() + off;
                const uint32_t* xrow = reinterpret_cast<const uint32_t*>(base + rec.xrow);
                const uint16_t* xslot = reinterpret_cast<const uint16_t*>(base + rec.xslot);
                const uint16_t* xwait = reinterpret_cast<const uint16_t*>(base + rec.xwait);
                bool ready = true;
                for (uint32_t x = 0; x < X && ready; ++x) {
                    if (xrow[x] >= n) return "halo row out of range";
                    if (xrow[x] >= rb && xrow[x] < rb + owned) return "halo row inside the slab";
                    ready = done[xrow[x]] != 0;
                }
                if (!ready) break;  // an upstream slab first
                for (uint32_t x = 0; x < X; ++x) {
                    if (xslot[x] >= L.slots || xslot[x] == 0) return "halo slot out of range";
                    // the kernel copies round r's halo in while round r - 1 computes
                    if (xwait[x] > (r > 0 ? r - 1 : 0)) return "a prefetch waits on its own or a later round";
                    c.xs[xslot[x]] = out[xrow[x]];
                    c.owner[xslot[x]] = xrow[x];
                }
                const double* vin = reinterpret_cast<const double*>(base + rec.in);
                const double* diag = reinterpret_cast<const double*>(base + rec.diag);
                const uint16_t* lrow = reinterpret_cast<const uint16_t*>(base + rec.lrow);
                const uint16_t* oslot = reinterpret_cast<const uint16_t*>(base + rec.oslot);
                const uint8_t* ent = base + rec.ent;
                auto ent_slot = [&](uint32_t e) -> uint64_t {
                    if (vb == 4) {
                        uint32_t w;
                        std::memcpy(&w, ent + (size_t)e * 8, 4);
                        return w;
                    }
                    uint16_t w;
                    std::memcpy(&w, ent + (size_t)e * 2, 2);
                    return w;
                };
                auto ent_val = [&](uint32_t e) {
                    Low v;
                    if (vb == 4) std::memcpy(&v, ent + (size_t)e * 8 + 4, 4);
                    else std::memcpy(&v, base + rec.val + (size_t)e * 8, 8);
                    return v;
                };
                // the rows of a round run at once: all of them read before any writes
                std::vector<double> res(nr);
                for (uint32_t j = 0; j < nr; ++j) {
                    if (lrow[j] >= owned) return "row outside its slab";
                    const uint32_t row = rb + lrow[j];
                    if (done[row]) return "row visited twice";
                    const uint32_t p = pos_of[row];
                    const uint32_t len = s.rowptr[p + 1] - s.rowptr[p];
                    if (len > Lr) return "row longer than its round's entry table";
                    if (diag[j] != (recip ? 1.0 / s.diag[p] : s.diag[p])) return "diagonal";
                    double acc = 0.0;
                    for (uint32_t t = 0; t < Lr; ++t) {
                        const uint32_t e = t * rec.m + j;
                        const uint64_t cs = ent_slot(e);
                        const Low cv = ent_val(e);
                        if (cs >= L.slots) return "dependency slot out of range";
                        if (t >= len) {  // padding: slot 0 (0.0) times 0
                            if (cs != 0 || cv != (Low)0) return "padding entry";
                            continue;
                        }
                        const uint32_t k = s.rowptr[p] + t;
                        if (cs == 0) return "a dependency in the zero slot";
                        if (c.owner[cs] != (int64_t)s.col[k]) return "a slot does not hold the dependency";
                        if (!done[s.col[k]]) return "a dependency read before it was finished";
                        if (cv != s.val[k]) return "coefficient";
                        acc += (double)cv * c.xs[cs];
                    }
                    if (s.op == SWEEP_DIV || s.op == SWEEP_MUL) res[j] = (vin[j] - acc) * diag[j];
                    else if (s.op == SWEEP_NONE) res[j] = vin[j] - acc;
                    else res[j] = vin[j] * diag[j] - acc;
                }
                for (uint32_t j = 0; j < nr; ++j) {
                    const uint32_t row = rb + lrow[j];
                    out[row] = res[j];
                    done[row] = 1;
                    if (oslot[j] != kNoSlot) {
                        if (oslot[j] >= L.slots || oslot[j] == 0) return "result slot out of range";
                        c.xs[oslot[j]] = res[j];
                        c.owner[oslot[j]] = row;
                    }
                }
                ++c.next;
                ++finished;
                progress = true;
            }
        }
        if (!progress) return "rounds wait on each other";
    }
    for (uint32_t r = 0; r < n; ++r)
        if (!done[r]) return "row never visited";
    return std::string();
}

// ---- explicit instantiations ------------------------------------------------
template int ict_factor<double>(const CsrHost&, double, CsrT<double>&, std::string*);
template int ict_factor<float>(const CsrHost&, double, CsrT<float>&, std::string*);
template int ildlt_factor<double>(const CsrHost&, double, CsrT<double>&, std::vector<double>&, std::string*);
template int ildlt_factor<float>(const CsrHost&, double, CsrT<float>&, std::vector<double>&, std::string*);
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
template bool stream_layout<double>(const Sweep<double>&, const std::vector<uint32_t>&, uint32_t, StreamLayout&,
                                    std::string*);
template bool stream_layout<float>(const Sweep<float>&, const std::vector<uint32_t>&, uint32_t, StreamLayout&,
                                   std::string*);
template std::string stream_layout_replay<double>(const Sweep<double>&, const StreamLayout&, const double*,
                                                  double*);
template std::string stream_layout_replay<float>(const Sweep<float>&, const StreamLayout&, const double*, double*);
template void build_sweep<double>(uint32_t, const std::vector<uint32_t>&, const std::vector<uint32_t>&,
                                  const std::vector<double>&, const std::vector<double>*, int, bool, Sweep<double>&);
template void build_sweep<float>(uint32_t, const std::vector<uint32_t>&, const std::vector<uint32_t>&,
                                 const std::vector<float>&, const std::vector<double>*, int, bool, Sweep<float>&);

}  // namespace prism
