// Host setup of AMSED / MSLR (reference: source/Preconditioner/AMSEDPrecondition.cpp).
// Compiled with -ffp-contract=off: the per-block factors are bit-exact with the
// reference's setup for the same partition; the Lanczos quantities agree to
// rounding (their tridiagonal eigen-decomposition is this file's own).
#include "amsed_setup.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <limits>
#include <numeric>
#include <random>
#include <thread>

extern "C" int64_t prism_graph_bisect(int32_t n, const int32_t* xadj, const int32_t* adjncy, int32_t* part);

namespace prism {

// ============================================================================
// Reverse Cuthill-McKee (vendored genrcm, restated).  Positions keep the
// original 1-based bookkeeping of the vendored code (perm[i-1] is position i)
// so that the control flow -- and hence the ordering -- is the same; node ids
// are 0-based here.
// ============================================================================
namespace {
struct Graph {
    const uint32_t* rp;
    const uint32_t* ci;
};

// level_set (rcm.cpp:2325-2460)
void rcm_level_set(const Graph& g, int root, std::vector<int>& mask, int& level_num, int* level_row, int* level) {
    mask[root] = 0;
    level[0] = root;
    level_num = 0;
    int lvlend = 0, iccsze = 1;
    for (;;) {
        const int lbegin = lvlend + 1;
        lvlend = iccsze;
        level_num = level_num + 1;
        level_row[level_num - 1] = lbegin;
        for (int i = lbegin; i <= lvlend; ++i) {
            const int node = level[i - 1];
            for (uint32_t j = g.rp[node]; j < g.rp[node + 1]; ++j) {
                const int nbr = (int)g.ci[j];
                if (mask[nbr] != 0) {
                    iccsze = iccsze + 1;
                    level[iccsze - 1] = nbr;
                    mask[nbr] = 0;
                }
            }
        }
        if (iccsze - lvlend <= 0) break;
    }
    level_row[level_num] = lvlend + 1;
    for (int i = 0; i < iccsze; ++i) mask[level[i]] = 1;
}

// root_find (rcm.cpp:3367-3558): pseudo-peripheral node of the component of `root`
void rcm_root_find(const Graph& g, int& root, std::vector<int>& mask, int* level_row, int* level) {
    int level_num;
    rcm_level_set(g, root, mask, level_num, level_row, level);
    const int iccsze = level_row[level_num] - 1;
    if (level_num == 1 || level_num == iccsze) return;
    for (;;) {
        int mindeg = iccsze;
        const int jstrt = level_row[level_num - 1];
        root = level[jstrt - 1];
        if (jstrt < iccsze) {
            for (int j = jstrt; j <= iccsze; ++j) {
                const int node = level[j - 1];
                int ndeg = 0;
                for (uint32_t k = g.rp[node]; k < g.rp[node + 1]; ++k)
                    if (0 < mask[g.ci[k]]) ndeg = ndeg + 1;
                if (ndeg < mindeg) {
                    root = node;
                    mindeg = ndeg;
                }
            }
        }
        int level_num2;
        rcm_level_set(g, root, mask, level_num2, level_row, level);
        if (level_num2 <= level_num) break;
        level_num = level_num2;
        if (iccsze <= level_num) break;
    }
}

// degree (rcm.cpp:860-997): component BFS order from root and masked degrees (self loop included)
void rcm_degree(const Graph& g, int root, const std::vector<int>& mask, std::vector<int>& deg, int& iccsze, int* ls,
                std::vector<uint8_t>& visited) {
    ls[0] = root;
    visited[root] = 1;
    int lvlend = 0;
    iccsze = 1;
    for (;;) {
        const int lbegin = lvlend + 1;
        lvlend = iccsze;
        for (int i = lbegin; i <= lvlend; ++i) {
            const int node = ls[i - 1];
            int ideg = 0;
            for (uint32_t j = g.rp[node]; j < g.rp[node + 1]; ++j) {
                const int nbr = (int)g.ci[j];
                if (mask[nbr] != 0) {
                    ideg = ideg + 1;
                    if (!visited[nbr]) {
                        visited[nbr] = 1;
                        iccsze = iccsze + 1;
                        ls[iccsze - 1] = nbr;
                    }
                }
            }
            deg[node] = ideg;
        }
        if (iccsze - lvlend == 0) break;
    }
    for (int i = 0; i < iccsze; ++i) visited[ls[i]] = 0;
}

// rcm (rcm.cpp:3137-3365): Cuthill-McKee from root, neighbours by increasing degree, reversed
void rcm_component(const Graph& g, int root, std::vector<int>& mask, int* perm, int& iccsze, std::vector<int>& deg,
                   std::vector<uint8_t>& visited) {
    rcm_degree(g, root, mask, deg, iccsze, perm, visited);
    mask[root] = 0;
    if (iccsze == 1) return;
    int lvlend = 0, lnbr = 1;
    while (lvlend < lnbr) {
        const int lbegin = lvlend + 1;
        lvlend = lnbr;
        for (int i = lbegin; i <= lvlend; ++i) {
            const int node = perm[i - 1];
            const int fnbr = lnbr + 1;
            for (uint32_t j = g.rp[node]; j < g.rp[node + 1]; ++j) {
                const int nbr = (int)g.ci[j];
                if (mask[nbr] != 0) {
                    lnbr = lnbr + 1;
                    mask[nbr] = 0;
                    perm[lnbr - 1] = nbr;
                }
            }
            if (lnbr <= fnbr) continue;
            // insertion sort of the new neighbours by increasing degree
            int k = fnbr;
            while (k < lnbr) {
                int l = k;
                k = k + 1;
                const int nbr = perm[k - 1];
                while (fnbr < l) {
                    const int lperm = perm[l - 1];
                    if (deg[lperm] <= deg[nbr]) break;
                    perm[l] = lperm;
                    l = l - 1;
                }
                perm[l] = nbr;
            }
        }
    }
    std::reverse(perm, perm + iccsze);
}
}  // namespace

void rcm_order(uint32_t n, const uint32_t* rowptr, const uint32_t* col, uint32_t* perm_out) {
    Graph g{rowptr, col};
    std::vector<int> mask(n, 1), level_row(n + 1), deg(n, 0), perm(n);
    std::vector<uint8_t> visited(n, 0);
    int num = 1;
    for (uint32_t i = 0; i < n; ++i) {
        if (mask[i] != 0) {
            int root = (int)i;
            rcm_root_find(g, root, mask, level_row.data(), perm.data() + num - 1);
            int iccsze = 0;
            rcm_component(g, root, mask, perm.data() + num - 1, iccsze, deg, visited);
            num = num + iccsze;
            if ((int)n < num) break;
        }
    }
    for (uint32_t i = 0; i < n; ++i) perm_out[i] = (uint32_t)perm[i];
}

// ============================================================================
// Sub-matrices
// ============================================================================
namespace {
// A(rows, cols) with columns renumbered by position in `cols`, each row's
// entries in the source row's order (CSRMatrix::getSubMatrix(rowPerm, colPerm),
// CSRMatrix.cpp:510-548), optionally sorted by the new column (formatStructure).
CsrHost sub_matrix(const CsrHost& A, const std::vector<uint32_t>& rows, const std::vector<uint32_t>& cols, bool sorted) {
    std::vector<uint32_t> table(A.n, 0xFFFFFFFFu);
    for (uint32_t i = 0; i < cols.size(); ++i) table[cols[i]] = i;
    CsrHost B;
    B.n = (uint32_t)rows.size();
    B.rowptr.assign(rows.size() + 1, 0);
    for (uint32_t i = 0; i < rows.size(); ++i) {
        const uint32_t r = rows[i];
        const size_t first = B.col.size();
        for (uint32_t k = A.rowptr[r]; k < A.rowptr[r + 1]; ++k) {
            const uint32_t c = table[A.col[k]];
            if (c == 0xFFFFFFFFu) continue;
            B.col.push_back(c);
            B.val.push_back(A.val[k]);
        }
        if (sorted) {
            // stable insertion sort by column (sortVectorPair, VectorTools.h:39-57)
            for (size_t a = first + 1; a < B.col.size(); ++a) {
                const uint32_t kc = B.col[a];
                const double kv = B.val[a];
                size_t b = a;
                while (b > first && B.col[b - 1] > kc) { B.col[b] = B.col[b - 1]; B.val[b] = B.val[b - 1]; --b; }
                B.col[b] = kc;
                B.val[b] = kv;
            }
        }
        B.rowptr[i + 1] = (uint32_t)B.col.size();
    }
    return B;
}

// rows [r0, r1) x cols [c0, c1) of a row-sorted CSR, columns shifted by c0
// (CSRMatrix::getSubMatrix by ranges, CSRMatrix.cpp:474-507)
CsrHost range_matrix(const CsrHost& A, uint32_t r0, uint32_t r1, uint32_t c0, uint32_t c1) {
    CsrHost B;
    B.n = r1 - r0;
    B.rowptr.assign((size_t)B.n + 1, 0);
    for (uint32_t r = r0; r < r1; ++r) {
        for (uint32_t k = A.rowptr[r]; k < A.rowptr[r + 1]; ++k) {
            const uint32_t c = A.col[k];
            if (c >= c0 && c < c1) {
                B.col.push_back(c - c0);
                B.val.push_back(A.val[k]);
            }
        }
        B.rowptr[r - r0 + 1] = (uint32_t)B.col.size();
    }
    return B;
}

// getConnectedComponents with ncomps = 0 (AMSEDPrecondition.cpp:427-556): BFS from the
// lowest unvisited node; each component's node list sorted ascending.
std::vector<std::vector<uint32_t>> components(const CsrHost& A) {
    const uint32_t n = A.n;
    std::vector<int32_t> marker(n, -1);
    std::vector<uint32_t> queue(n);
    std::vector<std::vector<uint32_t>> comps;
    int32_t current = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (marker[i] >= 0) continue;
        uint32_t qs = 0, qe = 1;
        queue[0] = i;
        marker[i] = current;
        while (qe > qs) {
            const uint32_t idx = queue[qs];
            for (uint32_t j = A.rowptr[idx]; j < A.rowptr[idx + 1]; ++j) {
                const uint32_t u = A.col[j];
                if (marker[u] < 0) {
                    queue[qe++] = u;
                    marker[u] = current;
                }
            }
            ++qs;
        }
        comps.emplace_back(queue.begin(), queue.begin() + qe);
        std::sort(comps.back().begin(), comps.back().end());
        ++current;
    }
    return comps;
}

// csrMatrixMetisKwayHID with num_dom = 2 (include/utils/ExternalTools/MetisTools.h:105-267):
// bisection, then the edge separator = every node with a neighbour in the other part.
// Returns err (1: a part without interior node); sets ndom and edgecut (separator size).
int hid_bisect(const CsrHost& C, uint32_t& ndom, std::vector<uint32_t>& sep, uint32_t& edgecut) {
    const uint32_t n = C.n;
    std::vector<int32_t> xadj(n + 1, 0), adjncy;
    adjncy.reserve(C.nnz());
    for (uint32_t i = 0; i < n; ++i) {
        for (uint32_t k = C.rowptr[i]; k < C.rowptr[i + 1]; ++k)
            if (C.col[k] != i) adjncy.push_back((int32_t)C.col[k]);
        xadj[i + 1] = (int32_t)adjncy.size();
    }
    std::vector<int32_t> part(n, 0);
    prism_graph_bisect((int32_t)n, xadj.data(), adjncy.data(), part.data());
    uint32_t sizes[2] = {0, 0};
    for (uint32_t i = 0; i < n; ++i) sizes[part[i]]++;
    ndom = (sizes[0] > 0) + (sizes[1] > 0);
    if (ndom < 2) {  // empty domain removed: everything in domain 0
        for (uint32_t i = 0; i < n; ++i) part[i] = 0;
    }
    sep.assign(n, 0);
    edgecut = 0;
    uint32_t sep_size[2] = {0, 0};
    for (uint32_t i = 0; i < n; ++i) {
        for (uint32_t k = C.rowptr[i]; k < C.rowptr[i + 1]; ++k) {
            if (part[C.col[k]] != part[i]) {
                sep[i] = 1;
                sep_size[part[i]]++;
                ++edgecut;
                break;
            }
        }
    }
    const uint32_t dsz[2] = {ndom < 2 ? n : sizes[0], sizes[1]};
    for (uint32_t d = 0; d < ndom; ++d)
        if (sep_size[d] == dsz[d]) return 1;
    return 0;
}

using Domains = std::vector<std::vector<uint32_t>>;

// setupPermutationNDRecursive (AMSEDPrecondition.cpp:302-423)
void nd_recursive(const CsrHost& A, uint32_t clvl, uint32_t& tlvl, std::vector<Domains>& level_str, uint32_t minsep) {
    if (tlvl < 2) {
        tlvl = 1;
        level_str.assign(1, Domains(1));
        level_str[0][0].resize(A.n);
        std::iota(level_str[0][0].begin(), level_str[0][0].end(), 0u);
        return;
    }
    if (clvl >= tlvl - 1) {
        tlvl = 1;
        level_str.assign(1, components(A));
        return;
    }
    const uint32_t dim = tlvl - clvl;
    level_str.assign(dim, Domains());
    Domains comps = components(A);
    std::vector<uint32_t> tlvls(comps.size(), 1);
    for (size_t i = 0; i < comps.size(); ++i) {
        const uint32_t nS = (uint32_t)comps[i].size();
        if (nS <= minsep || nS <= 2) {
            tlvls[i] = 1;
            level_str[0].push_back(comps[i]);
            continue;
        }
        CsrHost C = sub_matrix(A, comps[i], comps[i], false);
        uint32_t ndom = 2, edgecut = 0;
        std::vector<uint32_t> sep;
        if (hid_bisect(C, ndom, sep, edgecut) == 1) edgecut = nS;
        if (ndom < 2 || edgecut == nS) {
            tlvls[i] = 1;
            level_str[0].push_back(comps[i]);
            continue;
        }
        std::vector<uint32_t> keep;
        for (uint32_t j = 0; j < nS; ++j)
            if (sep[j] == 0) keep.push_back(j);
        CsrHost B = sub_matrix(C, keep, keep, false);
        tlvls[i] = tlvl;
        std::vector<Domains> sub;
        nd_recursive(B, clvl + 1, tlvls[i], sub, minsep);
        for (uint32_t j = 0; j < tlvls[i]; ++j) {
            for (auto& nodes : sub[j]) {
                for (auto& v : nodes) v = comps[i][keep[v]];
                level_str[j].push_back(nodes);
            }
        }
        std::vector<uint32_t> sepnodes;
        for (uint32_t j = 0; j < nS; ++j)
            if (sep[j] != 0) sepnodes.push_back(comps[i][j]);
        level_str[tlvls[i]].push_back(sepnodes);
        tlvls[i] += 1;
    }
    tlvl = *std::max_element(tlvls.begin(), tlvls.end());
    level_str.resize(tlvl);
}

// ---- host triangular applies in the reference's order (for the Lanczos process) ----
template <typename Low>
void ildlt_apply(const CsrT<Low>& Lt, const std::vector<double>& D, double* v) {
    const uint32_t n = Lt.n;
    for (uint32_t i = 0; i < n; ++i)  // IncompleteLDLT.cpp:216-233
        for (uint32_t k = Lt.rowptr[i]; k < Lt.rowptr[i + 1]; ++k) v[Lt.col[k]] -= (double)Lt.val[k] * v[i];
    for (uint32_t i = 0; i < n; ++i) v[i] /= D[i];  // :206-214
    for (uint32_t i = n; i-- > 0;)  // :188-204
        for (uint32_t k = Lt.rowptr[i]; k < Lt.rowptr[i + 1]; ++k) v[i] -= (double)Lt.val[k] * v[Lt.col[k]];
}

template <typename Low>
void ic_apply(const CsrT<Low>& Lt, double* v) {
    const uint32_t n = Lt.n;
    for (uint32_t i = 0; i < n; ++i) {  // IncompleteCholesky.cpp:249-271
        const double t = v[i] / (double)Lt.val[Lt.rowptr[i]];
        v[i] = t;
        for (uint32_t k = Lt.rowptr[i] + 1; k < Lt.rowptr[i + 1]; ++k) v[Lt.col[k]] -= (double)Lt.val[k] * t;
    }
    for (uint32_t i = n; i-- > 0;) {  // :274-295
        double t = v[i];
        for (uint32_t k = Lt.rowptr[i] + 1; k < Lt.rowptr[i + 1]; ++k) t -= (double)Lt.val[k] * v[Lt.col[k]];
        v[i] = t / (double)Lt.val[Lt.rowptr[i]];
    }
}

void spmv_host(const CsrHost& M, const double* x, double* y) {  // MatPVecWithRawPtr
    for (uint32_t i = 0; i < M.n; ++i) {
        double s = 0;
        for (uint32_t k = M.rowptr[i]; k < M.rowptr[i + 1]; ++k) s += x[M.col[k]] * M.val[k];
        y[i] = s;
    }
}

void spmv_t_add_host(const CsrHost& M, const double* x, double* y) {  // transMatPVec: y += M^T x
    for (uint32_t i = 0; i < M.n; ++i)
        for (uint32_t k = M.rowptr[i]; k < M.rowptr[i + 1]; ++k) y[M.col[k]] += M.val[k] * x[i];
}

double dot_host(size_t n, const double* a, const double* b) {
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

// Eigen-decomposition of the symmetric tridiagonal matrix (diagonal d[0..m),
// off-diagonal e[0..m-1)), with the contract of LAPACK dstevx, RANGE = 'A'
// (AMSEDPrecondition.cpp:975-1006): eigenvalues ascending in mu, unit
// eigenvectors as the columns of Y (column-major, m x m), the first component of
// largest magnitude of each made positive (the sign dstevx's inverse iteration,
// dstein, leaves).  Eigenvalues by implicit-shift QL.
//
// Eigenvectors: with inverse_iteration false, from the QL rotations accumulated
// (accurate to eps |T| in each component).  With inverse_iteration true, by
// inverse iteration on T - mu_j I, the method dstevx uses with a positive
// ABSTOL: an LU factorisation with partial pivoting (zero pivots replaced by
// eps |T|), four solves from a fixed start, each followed, inside a cluster
// (eigenvalues closer than 1e-3 |T|_1), by modified Gram-Schmidt against the
// cluster's earlier vectors.  Inverse iteration gives the small components of an
// eigenvector to high relative accuracy; the restarted Lanczos builds its Givens
// rotations from the last components of converged Ritz vectors, 1e-20 and below,
// and needs them.  The classic process only compares those components with
// 1e-15 / |beta_k|; there the accumulated rotations are kept.
void tridiag_eig(int m, const double* d_in, const double* e_in, double* mu, double* Y, bool inverse_iteration) {
    if (m <= 0) return;
    std::vector<double> d(d_in, d_in + m), e(m, 0.0), z;
    for (int i = 0; i + 1 < m; ++i) e[i] = e_in[i];
    if (!inverse_iteration) {
        z.assign((size_t)m * m, 0.0);
        for (int i = 0; i < m; ++i) z[(size_t)i * m + i] = 1.0;
    }
    for (int l = 0; l < m; ++l) {
        for (int iter = 0; iter < 60; ++iter) {
            int k = l;
            for (; k < m - 1; ++k) {
                const double dd = std::fabs(d[k]) + std::fabs(d[k + 1]);
                if (std::fabs(e[k]) <= 1e-16 * dd) break;
            }
            if (k == l) break;
            // Wilkinson-type shift from the leading 2x2 block
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::hypot(g, 1.0);
            g = d[k] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
            double s = 1.0, c = 1.0, p = 0.0;
            int i = k - 1;
            for (; i >= l; --i) {
                double f = s * e[i];
                const double b = c * e[i];
                r = std::hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {
                    d[i + 1] -= p;
                    e[k] = 0.0;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
                if (!inverse_iteration) {
                    for (int q = 0; q < m; ++q) {  // rotate columns i, i+1 of z
                        f = z[(size_t)(i + 1) * m + q];
                        z[(size_t)(i + 1) * m + q] = s * z[(size_t)i * m + q] + c * f;
                        z[(size_t)i * m + q] = c * z[(size_t)i * m + q] - s * f;
                    }
                }
            }
            if (r == 0.0 && i >= l) continue;
            d[l] -= p;
            e[l] = g;
            e[k] = 0.0;
        }
    }
    std::vector<int> idx(m);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return d[a] < d[b]; });
    for (int j = 0; j < m; ++j) mu[j] = d[idx[j]];
    auto store = [&](int j, const double* v) {  // with dstein's sign
        int big = 0;
        for (int q = 1; q < m; ++q)
            if (std::fabs(v[q]) > std::fabs(v[big])) big = q;
        const double sg = v[big] < 0 ? -1.0 : 1.0;
        for (int q = 0; q < m; ++q) Y[(size_t)j * m + q] = sg * v[q];
    };
    if (!inverse_iteration) {
        for (int j = 0; j < m; ++j) store(j, z.data() + (size_t)idx[j] * m);
        return;
    }

    const double eps = std::numeric_limits<double>::epsilon();
    double tnorm = 0.0;  // |T|_1
    for (int i = 0; i < m; ++i) {
        const double col = std::fabs(d_in[i]) + (i > 0 ? std::fabs(e_in[i - 1]) : 0.0) +
                           (i + 1 < m ? std::fabs(e_in[i]) : 0.0);
        tnorm = std::max(tnorm, col);
    }
    const double ortol = 1e-3 * tnorm, tiny = eps * std::max(tnorm, std::numeric_limits<double>::min());
    std::vector<double> dg(m), du(m), du2(m), ml(m), x(m);
    std::vector<char> swp(m);
    int cluster = 0;
    double prev = 0.0;
    for (int j = 0; j < m; ++j) {
        double lam = mu[j];
        if (j > 0) {
            if (mu[j] - mu[j - 1] > ortol) cluster = j;
            const double pert = 10.0 * std::fabs(eps * lam);  // separate equal shifts
            if (lam - prev < pert) lam = prev + pert;
        }
        prev = lam;
        // T - lam I = P L U, U with two superdiagonals
        for (int i = 0; i < m; ++i) {
            dg[i] = d_in[i] - lam;
            du[i] = i + 1 < m ? e_in[i] : 0.0;
            du2[i] = 0.0;
        }
        for (int i = 0; i + 1 < m; ++i) {
            const double sub = e_in[i];
            if (std::fabs(dg[i]) >= std::fabs(sub)) {
                swp[i] = 0;
                if (dg[i] == 0.0) dg[i] = tiny;
                ml[i] = sub / dg[i];
                dg[i + 1] -= ml[i] * du[i];
            } else {
                swp[i] = 1;
                ml[i] = dg[i] / sub;
                dg[i] = sub;
                const double t = dg[i + 1];
                dg[i + 1] = du[i] - ml[i] * t;
                if (i + 2 < m) {
                    du2[i] = du[i + 1];
                    du[i + 1] = -ml[i] * du[i + 1];
                }
                du[i] = t;
            }
        }
        for (int i = 0; i < m; ++i)
            if (std::fabs(dg[i]) < tiny) dg[i] = dg[i] < 0 ? -tiny : tiny;
        uint32_t lcg = 12345u + 7919u * (uint32_t)j;  // fixed start in [-1, 1)
        for (int i = 0; i < m; ++i) {
            lcg = lcg * 1664525u + 1013904223u;
            x[i] = (double)(lcg >> 8) / 8388608.0 - 1.0;
        }
        for (int it = 0; it < 4; ++it) {
            for (int i = 0; i + 1 < m; ++i) {
                if (swp[i]) {
                    const double t = x[i];
                    x[i] = x[i + 1];
                    x[i + 1] = t - ml[i] * x[i];
                } else {
                    x[i + 1] -= ml[i] * x[i];
                }
            }
            for (int i = m - 1; i >= 0; --i) {
                double v = x[i];
                if (i + 1 < m) v -= du[i] * x[i + 1];
                if (i + 2 < m) v -= du2[i] * x[i + 2];
                x[i] = v / dg[i];
            }
            for (int q = cluster; q < j; ++q) {
                const double* yq = Y + (size_t)q * m;
                double dot = 0.0;
                for (int i = 0; i < m; ++i) dot += yq[i] * x[i];
                for (int i = 0; i < m; ++i) x[i] -= dot * yq[i];
            }
            double nrm = 0.0, big = 0.0;
            for (int i = 0; i < m; ++i) big = std::max(big, std::fabs(x[i]));
            if (big == 0.0) {
                x[j] = 1.0;
                big = 1.0;
            }
            for (int i = 0; i < m; ++i) {
                x[i] /= big;
                nrm += x[i] * x[i];
            }
            nrm = std::sqrt(nrm);
            for (int i = 0; i < m; ++i) x[i] /= nrm;
        }
        store(j, x.data());
    }
}
}  // namespace

// ============================================================================
// Host applies of the partial preconditioner
// ============================================================================
// fn(i) for i in [0, count) on up to `threads` host threads (the items are independent:
// the results do not depend on the thread count)
template <typename F>
void host_parallel_for(uint32_t count, unsigned threads, F&& fn) {
    threads = std::min<unsigned>(threads, count);
    if (threads <= 1) {
        for (uint32_t i = 0; i < count; ++i) fn(i);
        return;
    }
    std::atomic<uint32_t> next{0};
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < threads; ++t)
        pool.emplace_back([&] {
            for (uint32_t i = next++; i < count; i = next++) fn(i);
        });
    for (auto& th : pool) th.join();
}
unsigned host_threads() { return std::max(1u, std::min(std::thread::hardware_concurrency(), 16u)); }

template <typename Low>
void amsed_block_solve_host(const AmsedSetup<Low>& S, int level, double* x) {
    const AmsedLevel<Low>& L = S.levels[level];
    const bool last = level == (int)S.nlev - 1;
    auto block = [&](uint32_t b) {
        double* seg = x + (L.dom_ptr[b] - L.dom_ptr[0]);
        if (last) {
            if (b == 0) ic_apply(L.Lt[0], seg);  // only block 0 carries a factor on the last level
        } else {
            ildlt_apply(L.Lt[b], L.D[b], seg);
        }
    };
    // the blocks are independent: large levels solve them on several host threads
    const uint32_t rows = L.dom_ptr[L.ncomps] - L.dom_ptr[0];
    host_parallel_for(L.ncomps, !last && rows >= 65536 ? host_threads() : 1u, block);
}

// levelCInvRecursiveSolve(level, x, 0) with x the C block of `level` (length len)
template <typename Low>
void amsed_c_solve_host(const AmsedSetup<Low>& S, int level, double* x, uint32_t len) {
    const int next = level + 1;
    if (level == (int)S.nlev - 2) {
        ic_apply(S.levels[S.nlev - 1].Lt[0], x);
        return;
    }
    const AmsedLevel<Low>& NL = S.levels[next];
    const uint32_t nb = S.lev_ptr[next + 1] - S.lev_ptr[next];
    const uint32_t nrem = S.n - S.lev_ptr[next + 1];
    (void)len;
    amsed_block_solve_host(S, next, x);
    std::vector<double> xc(nrem, 0.0);
    spmv_t_add_host(NL.E, x, xc.data());
    for (uint32_t i = 0; i < nrem; ++i) x[nb + i] -= xc[i];
    xc.assign(x + nb, x + nb + nrem);
    amsed_c_solve_host(S, next, x + nb, nrem);
    if (!NL.H.empty()) {
        const uint32_t r = (uint32_t)NL.H.size();
        std::vector<double> t(r, 0.0), t2(nrem, 0.0);
        for (uint32_t i = 0; i < r; ++i)
            for (uint32_t j = 0; j < nrem; ++j) t[i] += NL.W[(size_t)i * nrem + j] * xc[j];
        for (uint32_t i = 0; i < r; ++i) t[i] *= NL.H[i];
        for (uint32_t i = 0; i < r; ++i)
            for (uint32_t j = 0; j < nrem; ++j) t2[j] += NL.W[(size_t)i * nrem + j] * t[i];
        for (uint32_t j = 0; j < nrem; ++j) x[nb + j] += t2[j];
    }
    std::vector<double> tmp(nb);
    spmv_host(NL.E, x + nb, tmp.data());
    amsed_block_solve_host(S, next, tmp.data());
    for (uint32_t i = 0; i < nb; ++i) x[i] -= tmp[i];
}

// ============================================================================
// Setup
// ============================================================================
namespace {
// reorthogonalGeneralizedLanczos (AMSEDPrecondition.cpp:860-965) followed by the
// classic correction (classicLanczosForGeneralizedEigenvaluesProblem, :747-858).
template <typename Low>
void classic_lanczos(AmsedSetup<Low>& S, int level, const AmsedOptions& opt, unsigned seed) {
    AmsedLevel<Low>& L = S.levels[level];
    const uint32_t n_end = S.lev_ptr[level + 1];
    const uint32_t n_start = S.lev_ptr[level];
    const uint32_t n_local = n_end - n_start;
    const uint32_t nr = S.n - n_end;
    const int steps = opt.lanczos_steps;
    std::vector<double> D(steps, 0.0), E(steps, 0.0), V((size_t)nr * steps, 0.0);
    std::vector<double> v1(nr), u1(nr), z0(nr, 0.0), z1(nr, 0.0), v(nr), w(nr), tv(n_local);
    std::vector<double> rv((size_t)nr * steps, 0.0), rz((size_t)nr * steps, 0.0);
    {
        // generateArrayRandom1D (include/utils/TestTools/generateTools.hpp:79-102), seeded
        std::default_random_engine gen(seed);
        std::uniform_real_distribution<float> dist(-1.0, 1.0);
        for (uint32_t i = 0; i < nr; ++i) v1[i] = dist(gen);
    }
    spmv_host(L.C, v1.data(), u1.data());
    double ut = dot_host(nr, u1.data(), v1.data());
    ut = std::sqrt(ut);
    ut = 1.0 / ut;
    for (uint32_t i = 0; i < nr; ++i) v1[i] *= ut;
    spmv_host(L.C, v1.data(), z1.data());
    double beta = 0.0, alpha;
    int actual = 0;
    for (int i = 0; i < steps; ++i) {
        ++actual;
        if (beta != 0.0)
            for (uint32_t j = 0; j < nr; ++j) z0[j] *= beta;
        std::fill(v.begin(), v.end(), 0.0);
        spmv_host(L.E, v1.data(), tv.data());
        amsed_block_solve_host(S, level, tv.data());
        spmv_t_add_host(L.E, tv.data(), v.data());
        for (uint32_t j = 0; j < nr; ++j) v[j] = v[j] + -1 * z0[j];
        alpha = dot_host(nr, v.data(), v1.data());
        for (uint32_t j = 0; j < nr; ++j) v[j] = v[j] + (-1.0 * alpha) * z1[j];
        if (i > 1) {
            for (int k = 0; k < i - 1; ++k) {
                const double tp = dot_host(nr, v.data(), rv.data() + (size_t)k * nr);
                for (uint32_t j = 0; j < nr; ++j) v[j] -= rz[(size_t)k * nr + j] * tp;
            }
        }
        w = v;
        amsed_c_solve_host(S, level, w.data(), nr);
        const double tmp = dot_host(nr, w.data(), v.data());
        if (tmp < 0) break;
        beta = std::sqrt(tmp);
        if (beta <= 1e-15) break;
        D[i] = alpha;
        E[i] = beta;
        std::copy(v1.begin(), v1.end(), V.begin() + (size_t)i * nr);
        std::copy(v1.begin(), v1.end(), rv.begin() + (size_t)i * nr);
        std::copy(z1.begin(), z1.end(), rz.begin() + (size_t)i * nr);
        for (uint32_t j = 0; j < nr; ++j) {
            v1[j] = w[j] / beta;
            z0[j] = z1[j];
            z1[j] = v[j] / beta;
        }
    }
    S.lanczos_steps_done[level] = actual;
    std::vector<double> mu(actual), Y((size_t)actual * actual);
    tridiag_eig(actual, D.data(), E.data(), mu.data(), Y.data(), false);
    // converged Ritz pairs: |beta_k| |Y(last, i)| <= AMSED_EXIT_ZERO
    std::vector<int> conv;
    const double betak = E[actual - 1];
    for (int i = 0; i < actual; ++i)
        if (std::fabs(betak) * std::fabs(Y[(size_t)i * actual + actual - 1]) <= 1e-15) conv.push_back(i);
    L.rank = 0;
    L.H.clear();
    L.W.clear();
    if (conv.empty()) return;
    const int cc = (int)conv.size();
    int m = opt.lowrank_type == 0 ? std::min(cc, opt.low_rank) : cc;
    std::vector<int> chosen;
    if (opt.lowrank_type == 0) {
        for (int i = 0; i < m; ++i) chosen.push_back(conv[cc - i - 1]);
        for (int idx : chosen) L.H.push_back(mu[idx] / (1.0 - mu[idx]));
    } else {
        const double eps = opt.eig_bound, para = 1.0 - eps;
        for (int i = 0; i < m; ++i) {
            const int idx = conv[cc - i - 1];
            if (mu[idx] <= para) break;
            chosen.push_back(idx);
        }
        for (int idx : chosen) {
            const double lambda = 1.0 - mu[idx];
            L.H.push_back((eps - lambda) / lambda);
        }
    }
    const uint32_t r = (uint32_t)chosen.size();
    L.rank = r;
    L.rank_reported = r;
    L.W.assign((size_t)nr * r, 0.0);
    for (uint32_t i = 0; i < r; ++i) {
        double* wc = L.W.data() + (size_t)i * nr;
        const double* yc = Y.data() + (size_t)chosen[i] * actual;
        for (int c = 0; c < actual; ++c) {
            const double* vc = V.data() + (size_t)c * nr;
            for (uint32_t j = 0; j < nr; ++j) wc[j] += vc[j] * yc[c];
        }
    }
    const uint64_t lr = 2ull * r * nr + r;
    S.mnnz += lr;
    S.lowrank_nnz += lr;
}

// The low-rank terms of a level from its converged Ritz pairs (AMSEDPrecondition.cpp:1204-1267):
// the top m of mu (ascending), W = V Y over the `actual` Lanczos vectors.
template <typename Low>
void lowrank_from_ritz(AmsedSetup<Low>& S, AmsedLevel<Low>& L, const AmsedOptions& opt, uint32_t nr, int actual,
                       const std::vector<double>& mu, const std::vector<double>& Y, const std::vector<double>& V) {
    const int m = opt.lowrank_type == 0 ? std::min(actual, opt.low_rank) : actual;
    std::vector<int> chosen;
    L.H.clear();
    if (opt.lowrank_type == 0) {
        for (int i = 0; i < m; ++i) {
            const int idx = actual - i - 1;
            chosen.push_back(idx);
            L.H.push_back(mu[idx] / (1.0 - mu[idx]));
        }
    } else {
        const double eps = opt.eig_bound, para = 1.0 - eps;
        int count = 0;
        for (int i = 0; i < m; ++i) {
            if (mu[actual - i - 1] <= para || count >= opt.lanczos_steps) break;
            ++count;
        }
        for (int i = 0; i < count; ++i) {
            const int idx = actual - i - 1;
            chosen.push_back(idx);
            const double lambda = 1.0 - mu[idx];
            L.H.push_back((eps - lambda) / lambda);
        }
    }
    const uint32_t r = (uint32_t)chosen.size();
    L.rank = r;
    L.rank_reported = r;
    L.W.assign((size_t)nr * r, 0.0);
    for (uint32_t i = 0; i < r; ++i) {
        double* wc = L.W.data() + (size_t)i * nr;
        const double* yc = Y.data() + (size_t)chosen[i] * actual;
        for (int c = 0; c < actual; ++c) {
            const double* vc = V.data() + (size_t)c * nr;
            for (uint32_t j = 0; j < nr; ++j) wc[j] += vc[j] * yc[c];
        }
    }
    const uint64_t lr = 2ull * r * nr + r;
    S.mnnz += lr;
    S.lowrank_nnz += lr;
}

// expandReorthogonalLanczos (AMSEDPrecondition.cpp:1275-1351): steps from..to-1 of the
// generalized Lanczos process with full reorthogonalization, V and Z column-major (nr).
template <typename Low>
void expand_lanczos(AmsedSetup<Low>& S, int level, std::vector<double>& D, std::vector<double>& E,
                    std::vector<double>& V, std::vector<double>& Z, int from, int to, int& actual) {
    const AmsedLevel<Low>& L = S.levels[level];
    const uint32_t n_local = S.lev_ptr[level + 1] - S.lev_ptr[level];
    const uint32_t nr = S.n - S.lev_ptr[level + 1];
    std::vector<double> u(nr), w(nr), ut(n_local);
    actual = from;
    size_t vs = (size_t)from * nr;  // V(:, i)
    for (int i = from; i < to; ++i) {
        if (E[i - 1] <= 1e-15) return;  // AMSED_EXIT_ZERO
        ++actual;
        spmv_host(L.E, V.data() + vs, ut.data());
        amsed_block_solve_host(S, level, ut.data());
        std::fill(u.begin(), u.end(), 0.0);
        spmv_t_add_host(L.E, ut.data(), u.data());
        for (uint32_t j = 0; j < nr; ++j) u[j] = u[j] + (-1.0 * E[i - 1]) * Z[vs - nr + j];
        D[i] = dot_host(nr, u.data(), V.data() + vs);
        for (uint32_t j = 0; j < nr; ++j) u[j] = u[j] + (-1.0 * D[i]) * Z[vs + j];
        size_t ro = 0;
        for (int q = 0; q <= i; ++q) {  // full reorthogonalization: u -= Z(:, 1:i) (V(:, 1:i)' u)
            const double coef = dot_host(nr, V.data() + ro, u.data());
            for (uint32_t j = 0; j < nr; ++j) u[j] = u[j] + (-1.0 * coef) * Z[ro + j];
            ro += nr;
        }
        w = u;
        amsed_c_solve_host(S, level, w.data(), nr);
        E[i] = dot_host(nr, w.data(), u.data());
        if (E[i] < 0) {  // inexact B and C solves: stop
            E[i] = 1e-15;
            break;
        }
        E[i] = std::sqrt(E[i]);
        if (E[i] <= 1e-15) break;
        const double inv = 1.0 / E[i];
        for (uint32_t j = 0; j < nr; ++j) {
            V[vs + nr + j] = w[j] * inv;
            Z[vs + nr + j] = u[j] * inv;
        }
        vs += nr;
    }
}

// implicitRestartKrylovSchurLanczosForGeneralizedEigenvaluesProblem
// (AMSEDPrecondition.cpp:1010-1274): 2r Lanczos steps, then up to three restarts, each
// expanding to 4r steps, keeping the 2r largest Ritz pairs and bringing their
// tridiagonal form back with Givens rotations (convertDiagonal2TriDiagonal, :1381-1468;
// the rotations are applied as the reference applies them, each one to the rotated
// columns' values before any rotation, transposedGivensApplied2Columns, :1470-1490).
template <typename Low>
void restart_lanczos(AmsedSetup<Low>& S, int level, const AmsedOptions& opt, unsigned seed) {
    AmsedLevel<Low>& L = S.levels[level];
    const uint32_t n_local = S.lev_ptr[level + 1] - S.lev_ptr[level];
    const uint32_t nr = S.n - S.lev_ptr[level + 1];
    const int ms = opt.low_rank * 2, ks = opt.low_rank * 4, restarts = 3, maxs = opt.low_rank * 5;
    L.rank = 0;
    L.H.clear();
    L.W.clear();
    if (L.E.nnz() == 0) return;
    std::vector<double> D(maxs, 0.0), E(maxs, 0.0), V((size_t)nr * maxs, 0.0), auxV((size_t)nr * maxs, 0.0),
        Z((size_t)nr * maxs, 0.0), auxZ((size_t)nr * maxs, 0.0), Y((size_t)maxs * maxs, 0.0), mu(maxs, 0.0);
    std::vector<double> u(nr, 0.0), w(nr), ut(n_local), lastY(ms);
    {
        // generateArrayRandom1D, seeded as in the classic process
        std::default_random_engine gen(seed);
        std::uniform_real_distribution<float> dist(-1.0, 1.0);
        for (uint32_t i = 0; i < nr; ++i) V[i] = dist(gen);
    }
    {  // v1 = v / sqrt(v' C v)  (CSRMatrix::getMatrixNorm)
        double sum = 0.0;
        for (uint32_t r = 0; r < nr; ++r) {
            double cs = 0.0;
            for (uint32_t k = L.C.rowptr[r]; k < L.C.rowptr[r + 1]; ++k) cs += L.C.val[k] * V[L.C.col[k]];
            sum += V[r] * cs;
        }
        const double scale = 1.0 / std::sqrt(sum);
        for (uint32_t i = 0; i < nr; ++i) V[i] *= scale;
    }
    spmv_host(L.C, V.data(), Z.data());  // z1 = C v1
    spmv_host(L.E, V.data(), ut.data());
    amsed_block_solve_host(S, level, ut.data());
    spmv_t_add_host(L.E, ut.data(), u.data());
    D[0] = dot_host(nr, u.data(), V.data());
    for (uint32_t j = 0; j < nr; ++j) u[j] = u[j] + (-1.0 * D[0]) * Z[j];
    const double co = dot_host(nr, u.data(), V.data());
    for (uint32_t j = 0; j < nr; ++j) u[j] = u[j] + (-1.0 * co) * Z[j];
    w = u;
    amsed_c_solve_host(S, level, w.data(), nr);
    E[0] = std::sqrt(dot_host(nr, w.data(), u.data()));
    {
        const double inv = 1.0 / E[0];
        for (uint32_t j = 0; j < nr; ++j) {
            V[nr + j] = w[j] * inv;
            Z[nr + j] = u[j] * inv;
        }
    }
    int actual = 0;
    expand_lanczos(S, level, D, E, V, Z, 1, ms, actual);
    for (int rs = 0; rs < restarts; ++rs) {
        if (actual < ms) {  // ended early: no restart
            tridiag_eig(actual, D.data(), E.data(), mu.data(), Y.data(), true);
            break;
        }
        expand_lanczos(S, level, D, E, V, Z, ms, ks, actual);
        const int last = actual - 1;
        const double betak = E[last];
        tridiag_eig(actual, D.data(), E.data(), mu.data(), Y.data(), true);
        if (std::fabs(betak) * std::fabs(Y[(size_t)last * actual + last]) <= 1e-30 || rs == restarts - 1) break;
        // eigenpairs in descending order
        for (int e = 0; e < actual / 2; ++e) {
            const int p = actual - 1 - e;
            std::swap(mu[e], mu[p]);
            for (int q = 0; q < actual; ++q) std::swap(Y[(size_t)e * actual + q], Y[(size_t)p * actual + q]);
        }
        // auxV = V(:, 1:k) Y(:, 1:m), auxZ likewise
        if (rs > 0) {
            std::fill(auxV.begin(), auxV.end(), 0.0);
            std::fill(auxZ.begin(), auxZ.end(), 0.0);
        }
        for (int i = 0; i < ms; ++i) {
            double* av = auxV.data() + (size_t)i * nr;
            double* az = auxZ.data() + (size_t)i * nr;
            const double* yc = Y.data() + (size_t)i * actual;
            for (int c = 0; c < actual; ++c) {
                const size_t b = (size_t)c * nr;
                const double yv = yc[c];
                for (uint32_t r = 0; r < nr; ++r) {
                    av[r] += V[b + r] * yv;
                    az[r] += Z[b + r] * yv;
                }
            }
        }
        for (int st = 0; st < ms; ++st) lastY[st] = Y[(size_t)st * actual + last];
        // convertDiagonal2TriDiagonal: D = mu(1:m), E = 0, then Givens rotations; each one
        // reads columns of auxV / auxZ and writes the same columns of V / Z
        auto rotate = [&](double c, double s, int c1, int c2) {
            const size_t p1 = (size_t)c1 * nr, p2 = (size_t)c2 * nr;
            for (uint32_t r = 0; r < nr; ++r) {
                V[p1 + r] = auxV[p1 + r] * c + auxV[p2 + r] * s;
                Z[p1 + r] = auxZ[p1 + r] * c + auxZ[p2 + r] * s;
                V[p2 + r] = -1.0 * auxV[p1 + r] * s + auxV[p2 + r] * c;
                Z[p2 + r] = -1.0 * auxZ[p1 + r] * s + auxZ[p2 + r] * c;
            }
        };
        std::copy(mu.begin(), mu.begin() + ms, D.begin());
        std::fill(E.begin(), E.begin() + (ms - 1), 0.0);
        for (int i = 0; i < ms - 1; ++i) {
            const double zi = lastY[i], zi1 = lastY[i + 1];
            const double delta = std::sqrt(zi * zi + zi1 * zi1);
            double c = zi1 * 1.0 / delta, s = -1.0 * zi / delta;
            lastY[i + 1] = delta;
            lastY[i] = 0;
            double sc = c * c, ss = s * s, cs = c * s;
            const double ai = D[i], bi = E[i], ai1 = D[i + 1], tr = 2 * cs * bi;
            D[i] = sc * ai + tr + ss * ai1;
            E[i] = -1.0 * cs * ai + (sc - ss) * bi + cs * ai1;
            D[i + 1] = ss * ai - tr + sc * ai1;
            rotate(c, s, i, i + 1);
            if (i > 0) {
                double gamma = -1.0 * s * E[i - 1];
                E[i - 1] *= c;
                for (int r = i; r >= 1; --r) {
                    const double arm = D[r - 1], brm = E[r - 1], br = E[r], ar = D[r];
                    const double sigma = std::sqrt(gamma * gamma + br * br);
                    c = br * 1.0 / sigma;
                    s = -1.0 * gamma / sigma;
                    sc = c * c;
                    ss = s * s;
                    cs = c * s;
                    const double t2 = 2 * cs * brm;
                    D[r - 1] = sc * arm + t2 + ss * ar;
                    E[r - 1] = -1.0 * cs * arm + (sc - ss) * brm + cs * ar;
                    D[r] = ss * arm - t2 + sc * ar;
                    E[r] = sigma;
                    if (r > 1) {
                        gamma = -1.0 * s * E[r - 2];
                        E[r - 2] *= c;
                    }
                    rotate(c, s, r - 1, r);
                }
            }
        }
        E[ms - 1] = lastY[ms - 1] * betak;
        // v_{k+1} and z_{k+1} become columns m + 1
        std::copy(V.begin() + (size_t)actual * nr, V.begin() + (size_t)(actual + 1) * nr, V.begin() + (size_t)ms * nr);
        std::copy(Z.begin() + (size_t)actual * nr, Z.begin() + (size_t)(actual + 1) * nr, Z.begin() + (size_t)ms * nr);
    }
    S.lanczos_steps_done[level] = actual;
    lowrank_from_ritz(S, L, opt, nr, actual, mu, Y, V);
}
}  // namespace

template <typename Low>
int amsed_setup(const CsrHost& A, const AmsedOptions& opt, AmsedSetup<Low>& S, std::string* err) {
    if (opt.family != 4 && opt.family != 5) {
        if (err) *err = "family must be 5 (AMSED) or 4 (GMSLR)";
        return SETUP_BAD_INPUT;
    }
    const bool gmslr = opt.family == 4;
    if (!gmslr && opt.lanczos_type != 0 && opt.lanczos_type != 1) {
        if (err) *err = "lanczos_type must be 0 (UseClassicLanczos) or 1 (UseRestartLanczos)";
        return SETUP_BAD_INPUT;
    }
    if (opt.reorder != 0 && opt.reorder != 2) {
        if (err) *err = "local reordering must be MatrixReorderNo (0) or MatrixReorderRCM (2)";
        return SETUP_BAD_INPUT;
    }
    if (opt.levels < 1 || opt.lanczos_steps < 1) {
        if (err) *err = "levels and lanczos_steps must be >= 1";
        return SETUP_BAD_INPUT;
    }
    const uint32_t n = A.n;
    S = AmsedSetup<Low>();
    S.n = n;
    // ---- HID ordering (setupPermutationND, AMSEDPrecondition.cpp:80-110) ----
    uint32_t tlvl = (uint32_t)opt.levels;
    std::vector<Domains> level_str;
    nd_recursive(A, 0, tlvl, level_str, opt.minsep);
    S.nlev = tlvl;
    std::vector<int32_t> map_v(n);
    std::vector<uint32_t> mapptr(tlvl + 1, 0);
    int32_t domi = 0;
    for (uint32_t i = 0; i < tlvl; ++i) {
        for (auto& nodes : level_str[i]) {
            for (uint32_t v : nodes) map_v[v] = domi;
            ++domi;
        }
        mapptr[i + 1] = (uint32_t)domi;
    }
    // ---- level structure (buildLevelStructure, :112-300) ----
    const uint32_t ndom = mapptr[tlvl];
    std::vector<uint32_t> domsize(ndom, 0), domptr(ndom + 1, 0);
    for (uint32_t i = 0; i < n; ++i) domsize[map_v[i]]++;
    for (uint32_t d = 0; d < ndom; ++d) domptr[d + 1] = domptr[d] + domsize[d];
    S.pperm.assign(n, 0);
    {
        std::vector<uint32_t> fill(domptr.begin(), domptr.end() - 1);
        for (uint32_t i = 0; i < n; ++i) S.pperm[fill[map_v[i]]++] = i;
    }
    S.levels.assign(tlvl, AmsedLevel<Low>());
    S.lev_ptr.assign(tlvl + 1, 0);
    S.lev_ptr[tlvl] = n;
    S.lanczos_steps_done.assign(tlvl, 0);
    for (uint32_t level = 0; level < tlvl; ++level) {
        AmsedLevel<Low>& L = S.levels[level];
        const uint32_t maps = mapptr[level], mape = mapptr[level + 1];
        L.ncomps = mape - maps;
        S.lev_ptr[level] = domptr[maps];
        L.dom_ptr.assign(domptr.begin() + maps, domptr.begin() + mape + 1);
        if (opt.reorder == 2) {
            for (uint32_t b = 0; b < L.ncomps; ++b) {
                const uint32_t st = L.dom_ptr[b], ni = L.dom_ptr[b + 1] - L.dom_ptr[b];
                std::vector<uint32_t> copy(S.pperm.begin() + st, S.pperm.begin() + st + ni);
                CsrHost sub = sub_matrix(A, copy, copy, false);
                std::vector<uint32_t> sp(ni);
                rcm_order(ni, sub.rowptr.data(), sub.col.data(), sp.data());
                for (uint32_t i = 0; i < ni; ++i) S.pperm[st + i] = copy[sp[i]];
            }
        }
    }
    // A(pperm, pperm) with every row sorted (getSubMatrix + formatStructure)
    const CsrHost Apq = sub_matrix(A, S.pperm, S.pperm, true);
    for (uint32_t level = 0; level < tlvl; ++level) {
        AmsedLevel<Low>& L = S.levels[level];
        L.B.resize(L.ncomps);
        for (uint32_t b = 0; b < L.ncomps; ++b)
            L.B[b] = range_matrix(Apq, L.dom_ptr[b], L.dom_ptr[b + 1], L.dom_ptr[b], L.dom_ptr[b + 1]);
        if (level + 1 < tlvl) {
            const uint32_t n_start = S.lev_ptr[level], n_end = S.lev_ptr[level + 1];
            L.E = range_matrix(Apq, n_start, n_end, n_end, n);
            if (gmslr) L.F = range_matrix(Apq, n_end, n, n_start, n_end);
            else L.C = range_matrix(Apq, n_end, n, n_end, n);
        }
    }
    if (gmslr) {
        // GMSLR setupMSLR (GMSLRDPrecondition.cpp:649-733): ILUT(GMSLR_LFILL = 20, tol) on the last
        // level's block 0 and on every block of the other levels.  Its low-rank step
        // (reorthogonalSecondArnoldi + computeArnoldiEigenValuesAndEigenVectors, :849-1036)
        // calls LAPACKE_dhseqr with COMPZ = 'V' on a zero-initialised Z, which returns Q*Z = 0:
        // W is identically zero and the correction W H W^T vanishes.  The Arnoldi process is
        // therefore not run; the rank the reference reports (min(lanczosSteps, lowRankSize))
        // and its non-zero accounting (rank * n_remain + rank) are kept.
        const uint32_t lfill = 20;
        for (int level = (int)tlvl - 1; level >= 0; --level) {
            AmsedLevel<Low>& L = S.levels[level];
            const uint32_t nblk = level == (int)tlvl - 1 ? 1 : L.ncomps;
            L.Lt.resize(nblk);
            L.U.resize(nblk);
            L.Dinv.resize(nblk);
            std::vector<int> rcs(nblk, 0);
            std::vector<std::string> errs(nblk);
            host_parallel_for(nblk, host_threads(), [&](uint32_t b) {
                rcs[b] = ilut_factor<Low>(L.B[b], lfill, opt.factor_tol, L.Lt[b], L.U[b], L.Dinv[b],
                                          err ? &errs[b] : nullptr);
            });
            for (uint32_t b = 0; b < nblk; ++b) {
                if (rcs[b]) {
                    if (err) *err = errs[b];
                    return rcs[b];
                }
                const uint64_t m = L.Lt[b].nnz() + L.U[b].nnz() + L.B[b].n;
                S.mnnz += m;
                S.incomp_nnz += m;
            }
            if (level + 1 < (int)tlvl) {
                const uint32_t k = (uint32_t)std::min(opt.lanczos_steps, opt.low_rank);
                const uint32_t nr = n - S.lev_ptr[level + 1];
                L.rank = 0;
                L.rank_reported = k;
                const uint64_t lr = (uint64_t)k * nr + k;
                S.mnnz += lr;
                S.lowrank_nnz += lr;
            }
        }
        return SETUP_OK;
    }
    // ---- MSLR (setupMSLR, :652-743): IC on the last level, then per level ILDLT + Lanczos ----
    {
        AmsedLevel<Low>& last = S.levels[tlvl - 1];
        last.Lt.resize(1);
        int rc = ict_factor<Low>(last.B[0], opt.factor_tol, last.Lt[0], err);
        if (rc) return rc;
        const uint64_t m = last.Lt[0].nnz() * 2 + last.B[0].n;
        S.mnnz += m;
        S.incomp_nnz += m;
    }
    unsigned call = 0;
    for (int level = (int)tlvl - 2; level >= 0; --level) {
        AmsedLevel<Low>& L = S.levels[level];
        L.Lt.resize(L.ncomps);
        L.D.resize(L.ncomps);
        // the blocks' factorisations are independent: several host threads, results and the
        // first failing block (in block order) as one thread would give them
        std::vector<int> rcs(L.ncomps, 0);
        std::vector<std::string> errs(L.ncomps);
        host_parallel_for(L.ncomps, host_threads(), [&](uint32_t b) {
            rcs[b] = ildlt_factor<Low>(L.B[b], opt.factor_tol, L.Lt[b], L.D[b], err ? &errs[b] : nullptr);
        });
        for (uint32_t b = 0; b < L.ncomps; ++b) {
            if (rcs[b]) {
                if (err) *err = errs[b];
                return rcs[b];
            }
            const uint64_t m = L.Lt[b].nnz() * 2 + L.B[b].n;
            S.mnnz += m;
            S.incomp_nnz += m;
        }
        if (opt.lanczos_type == 1) restart_lanczos(S, level, opt, (unsigned)(opt.seed + call));
        else classic_lanczos(S, level, opt, (unsigned)(opt.seed + call));
        ++call;
    }
    return SETUP_OK;
}

template int amsed_setup<double>(const CsrHost&, const AmsedOptions&, AmsedSetup<double>&, std::string*);
template int amsed_setup<float>(const CsrHost&, const AmsedOptions&, AmsedSetup<float>&, std::string*);
template void amsed_block_solve_host<double>(const AmsedSetup<double>&, int, double*);
template void amsed_block_solve_host<float>(const AmsedSetup<float>&, int, double*);
template void amsed_c_solve_host<double>(const AmsedSetup<double>&, int, double*, uint32_t);
template void amsed_c_solve_host<float>(const AmsedSetup<float>&, int, double*, uint32_t);

}  // namespace prism
