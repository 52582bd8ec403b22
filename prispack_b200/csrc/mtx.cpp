// Matrix Market ingestion: HOST::ReadMtxTools::loadMatrix / loadRightHand
// (source/utils/TestTools/ReadMtxTools.cpp:50-453 of the reference), restated.
//
// What the reference reader does, and this one too:
//   * the banner "%%MatrixMarket matrix <coordinate|array> <real|complex|
//     pattern|integer> <general|symmetric|hermitian|skew-symmetric>" (words
//     after the banner compared case-insensitively) must be present; comment
//     lines start with '%'; the first other line holds "rows cols [nnz]";
//   * a sparse matrix must be "coordinate" with real (or complex: the real
//     part is the matrix, the imaginary part a second one) values; pattern and
//     integer files are refused (the reference throws);
//   * entries with |value| <= 10 * DBL_EPSILON are not stored
//     (IS_DOUBLE_NEAR_ZERO, config/config.h:19), indices are shifted by the
//     index base (1 for Matrix Market files);
//   * "symmetric" files are expanded to the full matrix (each off-diagonal
//     entry mirrored), "skew-symmetric" ones mirrored with the opposite sign;
//     "hermitian" files are taken as stored (the reference mirrors neither
//     part of those);
//   * COO -> CSR as transCOO2CSR (include/MatrixClass/MatrixTools.h:16-62):
//     entries grouped by row in file order, then each row ordered by column
//     with a stable sort (duplicates stay, in file order);
//   * a right-hand side is an "array" file of rows x cols values in column
//     order.
#include <algorithm>
#include <cctype>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "host_setup.hpp"

namespace prism {

namespace {
std::string lower(std::string s) {
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

struct Header {
    bool coordinate = true;
    std::string field, symmetry;
    uint64_t rows = 0, cols = 0, nnz = 0;
};

// Reads the banner, comments and size line; leaves `in` at the first entry line.
bool read_header(std::istream& in, Header& h, bool want_coordinate, std::string* err) {
    std::string line;
    bool banner = false;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] != '%') break;
        std::istringstream is(line);
        std::string tag, obj, fmt, field, sym;
        is >> tag;
        if (tag != "%%MatrixMarket") continue;
        banner = true;
        is >> obj >> fmt >> field >> sym;
        obj = lower(obj), fmt = lower(fmt), field = lower(field), sym = lower(sym);
        if (obj != "matrix") return *err = "not a Matrix Market matrix file", false;
        if (fmt != "coordinate" && fmt != "array") return *err = "unknown storage '" + fmt + "'", false;
        if (field != "real" && field != "complex" && field != "pattern" && field != "integer")
            return *err = "unknown value type '" + field + "'", false;
        if (sym != "general" && sym != "symmetric" && sym != "hermitian" && sym != "skew-symmetric")
            return *err = "unknown symmetry '" + sym + "'", false;
        h.coordinate = fmt == "coordinate";
        h.field = field;
        h.symmetry = sym;
    }
    if (!banner) return *err = "no %%MatrixMarket banner", false;
    if (want_coordinate != h.coordinate)
        return *err = want_coordinate ? "a sparse matrix must be stored as coordinate"
                                      : "a right-hand side must be stored as array",
               false;
    std::istringstream is(line);
    if (!(is >> h.rows >> h.cols)) return *err = "missing size line", false;
    if (h.coordinate && !(is >> h.nnz)) return *err = "missing number of entries", false;
    return true;
}
}  // namespace

int read_mtx(const std::string& path, uint32_t base, int part, uint32_t& rows, uint32_t& cols,
             std::vector<uint32_t>& rowptr, std::vector<uint32_t>& col, std::vector<double>& val, std::string* err) {
    std::ifstream in(path, std::ios::binary);
    if (!in) return *err = "cannot open " + path, SETUP_BAD_INPUT;
    Header h;
    if (!read_header(in, h, true, err)) return SETUP_BAD_INPUT;
    if (h.field != "real" && h.field != "complex")
        return *err = "value type '" + h.field + "' is not supported (real or complex only)", SETUP_BAD_INPUT;
    if (h.rows > 0xFFFFFFFFull || h.cols > 0xFFFFFFFFull) return *err = "more than 2^32 rows", SETUP_BAD_INPUT;
    rows = (uint32_t)h.rows;
    cols = (uint32_t)h.cols;
    const bool cplx = h.field == "complex";
    if (part == 1 && !cplx) return *err = "no imaginary part in a real file", SETUP_BAD_INPUT;
    const bool sym = h.symmetry == "symmetric", skew = h.symmetry == "skew-symmetric";
    const double zero = 10.0 * DBL_EPSILON;  // IS_DOUBLE_NEAR_ZERO
    // COO in file order (mirrored entries right after their source, as the reference pushes them)
    std::vector<uint32_t> ci, cj;
    std::vector<double> cv;
    ci.reserve(h.nnz * (sym || skew ? 2 : 1));
    cj.reserve(ci.capacity());
    cv.reserve(ci.capacity());
    std::string line;
    uint64_t lines = 0;
    auto push = [&](std::vector<uint32_t>& r, std::vector<uint32_t>& c, std::vector<double>& v, uint32_t i, uint32_t j,
                    double x) {
        r.push_back(i);
        c.push_back(j);
        v.push_back(x);
        if (i != j && sym) {
            r.push_back(j);
            c.push_back(i);
            v.push_back(x);
        } else if (i != j && skew) {
            r.push_back(j);
            c.push_back(i);
            v.push_back(-1.0 * x);
        }
    };
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '%') continue;
        const char* p = line.c_str();
        char* e = nullptr;
        const unsigned long long i = std::strtoull(p, &e, 10);
        if (e == p) continue;  // a blank line with spaces
        p = e;
        const unsigned long long j = std::strtoull(p, &e, 10);
        if (e == p) return *err = "malformed entry line: " + line, SETUP_BAD_INPUT;
        p = e;
        const double re = std::strtod(p, &e);
        if (e == p) return *err = "malformed entry line: " + line, SETUP_BAD_INPUT;
        p = e;
        double im = 0.0;
        if (cplx) {
            im = std::strtod(p, &e);
            if (e == p) return *err = "malformed complex entry: " + line, SETUP_BAD_INPUT;
        }
        if (i < base || j < base || i - base >= h.rows || j - base >= h.cols)
            return *err = "entry index out of range: " + line, SETUP_BAD_INPUT;
        const uint32_t r = (uint32_t)(i - base), c = (uint32_t)(j - base);
        const double x = part == 1 ? im : re;  // the part asked for, each with its own pattern
        if (!(std::fabs(x) <= zero)) push(ci, cj, cv, r, c, x);
        ++lines;
    }
    if (lines != h.nnz) return *err = "the file lists " + std::to_string(lines) + " entries, its size line " +
                                      std::to_string(h.nnz), SETUP_BAD_INPUT;
    // transCOO2CSR: rows in file order, then a stable sort by column inside each row
    auto to_csr = [&](const std::vector<uint32_t>& r, const std::vector<uint32_t>& c, const std::vector<double>& v,
                      std::vector<uint32_t>& rp, std::vector<uint32_t>& cc, std::vector<double>& vv) {
        const size_t nnz = r.size();
        if (nnz > 0xFFFFFFFFull) return false;
        rp.assign((size_t)rows + 1, 0);
        for (size_t k = 0; k < nnz; ++k) rp[r[k] + 1]++;
        for (uint32_t q = 0; q < rows; ++q) rp[q + 1] += rp[q];
        std::vector<uint32_t> fill(rp.begin(), rp.end() - 1);
        cc.resize(nnz);
        vv.resize(nnz);
        for (size_t k = 0; k < nnz; ++k) {
            cc[fill[r[k]]] = c[k];
            vv[fill[r[k]]] = v[k];
            fill[r[k]]++;
        }
        std::vector<uint32_t> idx;
        for (uint32_t q = 0; q < rows; ++q) {
            const uint32_t b = rp[q], e = rp[q + 1];
            idx.resize(e - b);
            std::iota(idx.begin(), idx.end(), b);
            std::stable_sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) { return cc[x] < cc[y]; });
            std::vector<uint32_t> c2(e - b);
            std::vector<double> v2(e - b);
            for (uint32_t t = 0; t < e - b; ++t) {
                c2[t] = cc[idx[t]];
                v2[t] = vv[idx[t]];
            }
            std::copy(c2.begin(), c2.end(), cc.begin() + b);
            std::copy(v2.begin(), v2.end(), vv.begin() + b);
        }
        return true;
    };
    if (!to_csr(ci, cj, cv, rowptr, col, val)) return *err = "more than 2^32 stored entries", SETUP_BAD_INPUT;
    return SETUP_OK;
}

int read_mtx_dense(const std::string& path, uint32_t& rows, uint32_t& cols, std::vector<double>& values,
                   std::string* err) {
    std::ifstream in(path, std::ios::binary);
    if (!in) return *err = "cannot open " + path, SETUP_BAD_INPUT;
    Header h;
    if (!read_header(in, h, false, err)) return SETUP_BAD_INPUT;
    if (h.field != "real") return *err = "value type '" + h.field + "' is not supported (real only)", SETUP_BAD_INPUT;
    if (h.rows * h.cols > 0xFFFFFFFFull) return *err = "more than 2^32 values", SETUP_BAD_INPUT;
    rows = (uint32_t)h.rows;
    cols = (uint32_t)h.cols;
    values.assign((size_t)rows * cols, 0.0);
    for (size_t k = 0; k < values.size(); ++k)
        if (!(in >> values[k])) return *err = "the file holds fewer values than rows x cols", SETUP_BAD_INPUT;
    return SETUP_OK;
}

}  // namespace prism
