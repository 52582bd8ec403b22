// DeviceSolver: a PrisPack BaseSolver<double> (include/Solver/BaseSolver.h:16)
// whose whole Krylov iteration -- FCG as CG<double>::solve (CG.cpp:34-83) or
// FGMRES as GMRES<double>::solve (GMRES.cpp:122-221) -- runs on the device
// with the DevicePrecondition's factors, through prism_solve.
//
// solve(matA, b, x) copies b and the initial guess x to the device, iterates
// there (one synchronisation per iteration for the convergence test) and
// copies x back; matA must be the matrix the DevicePrecondition was built on.
// getNumIter / getError / getConvergence mean what the reference's do
// (include/Solver/CG.h:44-54).
#ifndef PRISM_DEVICE_SOLVER_HPP
#define PRISM_DEVICE_SOLVER_HPP

#include "DevicePrecondition.hpp"

template <typename T>
class DeviceSolver : public BaseSolver<T> {
  public:
    // kind: PRISM_SOLVER_FCG, PRISM_SOLVER_CG, PRISM_SOLVER_FGMRES or PRISM_SOLVER_GMRES;
    // restart: GMRES restart length (0: none)
    DeviceSolver(const std::shared_ptr<DevicePrecondition<T>>& M, int32_t kind, double tol, UINT32 maxIter,
                 UINT32 restart = 0)
        : M_(M) {
        opts_.solver = kind;
        opts_.tol = tol;
        opts_.max_iter = maxIter;
        opts_.restart = restart;
        opts_.x_ref = nullptr;
        opts_.launch_mode = PRISM_LAUNCH_AUTO;
    }

    void solve(const HOST::CSRMatrix<T>& matA, const HostVector<T>& b, HostVector<T>& x) override {
        THROW_EXCEPTION(matA.getRowNum() != b.getLength() || x.getLength() != b.getLength(),
                        THROW_INVALID_ARGUMENT("DeviceSolver: sizes differ"))
        M_->setup();
        const int32_t rc = prism_solve(M_->handle(), &opts_, b.getRawValPtr(), x.getRawValPtr(), &stats_);
        THROW_EXCEPTION(rc != PRISM_OK, THROW_RANGE_ERROR(std::string("prism: ") + prism_last_error()))
    }

    INT32 getNumIter() const { return stats_.num_iter; }
    FLOAT64 getError() const { return stats_.final_error; }
    bool getConvergence() const { return stats_.converged != 0; }
    // no reference counterpart: ||b - A x|| / ||b|| recomputed in FP64 at exit
    FLOAT64 getTrueRelativeResidual() const { return stats_.true_rel_residual; }

  private:
    std::shared_ptr<DevicePrecondition<T>> M_;
    prism_solve_opts opts_{};
    prism_solve_stats stats_{};
};

#endif  // PRISM_DEVICE_SOLVER_HPP
