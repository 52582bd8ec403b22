// The reference's own solver with the device preconditioner plugged in.
//
// Built by `make -C oracle integration REF=<reference tree>` against the
// reference's headers and its compiled sources (oracle/_ref/parity objects),
// linked with libprism_solve.so; run on a machine with a B200:
//
//   oracle/_ref/device_cg_driver [nx ny nz]        (default 48 48 48)
//
// For 3D Poisson (generateLaplacianCSR, the reference's generator) and a
// seeded right-hand side it runs, and prints as one JSON line:
//   ic.reference   HOST::CG<double> FlexibleCG + HOST::IncompleteCholesky<double,double>(1e-3)
//   ic.device      the same HOST::CG<double> with DevicePrecondition (IC 1e-3, FP64 factors)
//   ic.solver      DeviceSolver (the whole FCG on the device), same preconditioner
//   refactor.reference / refactor.device   A scaled by 1.5 on the same pattern: a new
//                  IncompleteCholesky setup against DevicePrecondition::refactor()
//   amsed.reference / amsed.device   the same with AMSEDPrecondition<double,double>
//                  (3 levels, 32 Lanczos steps, rank 16, MSLR, natural local order)
// with iteration counts, true relative residuals and the relative difference
// of each solution from the reference's.
#include "config/headers.h"
#include <omp.h>

#include <cmath>
#include <cstdio>
#include <algorithm>
#include <random>
#include <vector>
#include <string>

#include "MatrixClass/CSRMatrix.h"
#include "MatrixClass/ModelProblem.h"
#include "Preconditioner/AMSEDPrecondition.h"
#include "Preconditioner/BasePreconditon.h"
#include "Preconditioner/IncompleteCholesky.h"
#include "Solver/CG.h"
#include "VectorClass/AutoAllocateVector.h"

#include "DevicePrecondition.hpp"
#include "DeviceSolver.hpp"

using namespace HOST;

extern "C" void ref_set_seed(unsigned seed);  // the Lanczos start vector's seed (oracle shim)

namespace {
using Vec = AutoAllocateVector<FLOAT64>;

double rel_residual(const CSRMatrix<FLOAT64>& A, const HostVector<FLOAT64>& b, const HostVector<FLOAT64>& x) {
    const UINT32 n = A.getRowNum();
    double rr = 0.0, bb = 0.0;
    for (UINT32 i = 0; i < n; ++i) {
        double s = 0.0;
        for (UINT32 k = A.getRowOffsetPtr(0)[i]; k < A.getRowOffsetPtr(0)[i + 1]; ++k)
            s += A.getCSRValuesPtr(0)[k] * x[A.getColIndicesPtr(0)[k]];
        rr += (b[i] - s) * (b[i] - s);
        bb += b[i] * b[i];
    }
    return std::sqrt(rr / bb);
}

double rel_diff(const HostVector<FLOAT64>& x, const HostVector<FLOAT64>& y) {
    double d = 0.0, m = 0.0;
    for (UINT32 i = 0; i < x.getLength(); ++i) {
        d += (x[i] - y[i]) * (x[i] - y[i]);
        m += y[i] * y[i];
    }
    return std::sqrt(d / m);
}

std::string run_cg(const char* name, const std::shared_ptr<CSRMatrix<FLOAT64>>& A,
                   const std::shared_ptr<BasePrecondition<FLOAT64>>& M, const HostVector<FLOAT64>& b,
                   HostVector<FLOAT64>& x, const HostVector<FLOAT64>* xref) {
    const UINT32 n = A->getRowNum();
    for (UINT32 i = 0; i < n; ++i) x[i] = 0.0;
    CG<FLOAT64> cg(n, M, FlexibleCG, 1e-10, 1000);
    cg.solve(*A, b, x);
    char buf[256];
    std::snprintf(buf, sizeof buf, "\"%s\": {\"iters\": %d, \"converged\": %d, \"true_rel_residual\": %.3e, \"diff\": %.3e}",
                  name, cg.getNumIter(), cg.getConvergence() ? 1 : 0, rel_residual(*A, b, x),
                  xref ? rel_diff(x, *xref) : 0.0);
    return buf;
}
}  // namespace

int main(int argc, char** argv) {
    const int nx = argc > 3 ? std::atoi(argv[1]) : 48, ny = argc > 3 ? std::atoi(argv[2]) : 48,
              nz = argc > 3 ? std::atoi(argv[3]) : 48;
    auto A = std::make_shared<CSRMatrix<FLOAT64>>();
    generateLaplacianCSR(*A, nx, ny, nz, 0.0, 0.0, 0.0, 0.0);
    const UINT32 n = A->getRowNum();
    Vec b(n, memoryBase), xr(n, memoryBase), xd(n, memoryBase), xs(n, memoryBase);
    std::mt19937_64 gen(2024);
    std::normal_distribution<double> nd(0.0, 1.0);
    for (UINT32 i = 0; i < n; ++i) b[i] = nd(gen);
    std::string out = "{\"n\": " + std::to_string(n);
    try {
        // ---- IC(1e-3)
        auto ic = std::make_shared<IncompleteCholesky<FLOAT64, FLOAT64>>(A, 1e-3);
        out += ", " + run_cg("ic.reference", A, ic, *b, *xr, nullptr);
        auto dev = std::make_shared<DevicePrecondition<FLOAT64>>(A, 0);
        dev->useIC(1e-3, PRISM_FP64);
        out += ", " + run_cg("ic.device", A, dev, *b, *xd, &*xr);
        out += ", \"ic.mnnz\": [" + std::to_string(ic->getPreconditionNonZeroCount()) + ", " +
               std::to_string(dev->getPreconditionNonZeroCount()) + "]";
        for (UINT32 i = 0; i < n; ++i) (*xs)[i] = 0.0;
        DeviceSolver<FLOAT64> solver(dev, PRISM_SOLVER_FCG, 1e-10, 1000);
        solver.solve(*A, *b, *xs);
        char buf[256];
        std::snprintf(buf, sizeof buf, ", \"ic.solver\": {\"iters\": %d, \"converged\": %d, \"true_rel_residual\": "
                      "%.3e, \"diff\": %.3e}", solver.getNumIter(), solver.getConvergence() ? 1 : 0,
                      rel_residual(*A, *b, *xs), rel_diff(*xs, *xr));
        out += buf;
        // the four MInvSolve overloads on one vector: whole, in place at an offset, out of place
        Vec v(n, memoryBase), w(n, memoryBase), big(2 * n, memoryBase), big2(3 * n, memoryBase);
        for (UINT32 i = 0; i < n; ++i) (*v)[i] = (*big)[n + i] = (*b)[i];
        dev->MInvSolve(*v, *w);
        dev->MInvSolve(*v);
        dev->MInvSolve(*big, n);
        dev->MInvSolve(*b, 0, *big2, 2 * n);
        double d1 = 0.0, d2 = 0.0, d3 = 0.0;
        for (UINT32 i = 0; i < n; ++i) {
            d1 = std::max(d1, std::fabs((*v)[i] - (*w)[i]));
            d2 = std::max(d2, std::fabs((*big)[n + i] - (*w)[i]));
            d3 = std::max(d3, std::fabs((*big2)[2 * n + i] - (*w)[i]));
        }
        std::snprintf(buf, sizeof buf, ", \"overloads_max_diff\": [%.3e, %.3e, %.3e]", d1, d2, d3);
        out += buf;
        // ---- new values on the same pattern (A scaled by 1.5, so IC(1e-3) keeps its pattern):
        // a new reference setup against DevicePrecondition::refactor on the device
        {
            const UINT32 nnz = A->getNNZnum(0, n - 1);
            FLOAT64* av = A->getCSRValuesPtr(0);
            std::vector<FLOAT64> saved(av, av + nnz);
            for (UINT32 k = 0; k < nnz; ++k) av[k] *= 1.5;
            Vec xr2(n, memoryBase), xd2(n, memoryBase);
            auto ic2 = std::make_shared<IncompleteCholesky<FLOAT64, FLOAT64>>(A, 1e-3);
            out += ", " + run_cg("refactor.reference", A, ic2, *b, *xr2, nullptr);
            dev->refactor();
            out += ", " + run_cg("refactor.device", A, dev, *b, *xd2, &*xr2);
            out += ", \"refactor.mnnz\": [" + std::to_string(ic2->getPreconditionNonZeroCount()) + ", " +
                   std::to_string(dev->getPreconditionNonZeroCount()) + "]";
            std::copy(saved.begin(), saved.end(), av);
        }
        // ---- AMSED / MSLR
        ref_set_seed(20241116u);
        auto am = std::make_shared<AMSEDPrecondition<FLOAT64, FLOAT64>>(A, 3, 32, 16, 0.8, MatrixReorderNo,
                                                                        AMSEDBasic, UseClassicLanczos);
        out += ", " + run_cg("amsed.reference", A, am, *b, *xr, nullptr);
        auto adev = std::make_shared<DevicePrecondition<FLOAT64>>(A, 0);
        prism_amsed_opts o;
        prism_amsed_default_opts(&o);
        o.levels = 3;
        o.lanczos_steps = 32;
        o.low_rank = 16;
        o.eig_bound = 0.8;
        o.lowrank_type = 0;
        o.reorder = 0;
        adev->useAMSED(o, PRISM_FP64);
        out += ", " + run_cg("amsed.device", A, adev, *b, *xd, &*xr);
        out += ", \"ok\": 1}";
    } catch (const std::exception& e) {
        out += std::string(", \"error\": \"") + e.what() + "\"}";
        std::printf("%s\n", out.c_str());
        return 1;
    }
    std::printf("%s\n", out.c_str());
    return 0;
}
