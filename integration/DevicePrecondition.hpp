// DevicePrecondition: a PrisPack BasePrecondition<double> whose M^{-1} runs on
// a B200 through the C ABI of include/prism_solve.h.
//
// Drop-in for the reference's preconditioner objects
// (include/Preconditioner/BasePreconditon.h:34-145): it implements setup()
// and all four MInvSolve overloads, so HOST::CG / HOST::GMRES, or any other
// caller holding a std::shared_ptr<BasePrecondition<double>>, use it
// unchanged.  The host setup (factorisation, HID ordering, Lanczos) runs in
// the library, bit-exact with the reference's setup(), and the factors stay
// resident on the device; each MInvSolve copies its vector to the device,
// applies M^{-1} there and copies the result back.  Device-resident callers
// use prism_apply_device / prism_solve_device on their own pointers instead
// (DeviceSolver.hpp).
//
// Include after the reference's headers (it uses BaseVector, HOST::CSRMatrix,
// THROW_EXCEPTION); link -lprism_solve.
#ifndef PRISM_DEVICE_PRECONDITION_HPP
#define PRISM_DEVICE_PRECONDITION_HPP

#include <functional>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "../include/prism_solve.h"

template <typename T>
class DevicePrecondition : public BasePrecondition<T> {
    static_assert(std::is_same<T, double>::value, "the device apply takes double vectors");

  public:
    // The operator is copied to `device` once; A must stay the matrix the solver works with.
    explicit DevicePrecondition(const std::shared_ptr<HOST::CSRMatrix<T>>& A, int32_t device = 0) : A_(A) {
        const UINT32 n = A->getRowNum();
        check(prism_create(n, A->getRowOffsetPtr(0), A->getColIndicesPtr(0), A->getCSRValuesPtr(0), device, &h_));
        this->m_ArowNum = n;
        this->m_AcolNum = n;
        this->m_Annz = A->getNNZnum(0, n - 1);
    }
    ~DevicePrecondition() override {
        if (h_) prism_destroy(h_);
    }
    DevicePrecondition(const DevicePrecondition&) = delete;
    DevicePrecondition& operator=(const DevicePrecondition&) = delete;

    // Which preconditioner, as the reference's constructors take them.  precision:
    // PRISM_FP64 (<double,double>), PRISM_FP32 (<float,double>) or PRISM_FP32_APPLY
    // (float values and float arithmetic inside the triangular sweeps).
    void useIC(double threshold, prism_precision p = PRISM_FP64) {
        kind_ = [=](prism_handle h) { return prism_set_precond_ic(h, threshold, p); };
        this->m_precondType = PreconditionIC;
    }
    void useILDLT(double tol, prism_precision p = PRISM_FP64) {
        kind_ = [=](prism_handle h) { return prism_set_precond_ildlt(h, tol, p); };
        this->m_precondType = PreconditionILDLT;
    }
    void useILUT(UINT32 lfill, double tol, prism_precision p = PRISM_FP64) {
        kind_ = [=](prism_handle h) { return prism_set_precond_ilut(h, lfill, tol, p); };
        this->m_precondType = PreconditionILUT;
    }
    void useAMSED(const prism_amsed_opts& o, prism_precision p = PRISM_FP64) {
        kind_ = [=](prism_handle h) { return prism_set_precond_amsed(h, &o, p); };
        this->m_precondType = PreconditionAMSED;
    }
    void useGMSLR(const prism_amsed_opts& o, prism_precision p = PRISM_FP64) {
        kind_ = [=](prism_handle h) { return prism_set_precond_gmslr(h, &o, p); };
        this->m_precondType = PreconditionGMSLR;
    }

    // BasePrecondition::setup (the reference's solvers call it first; a no-op once ready)
    void setup() override {
        if (this->m_isReady == PRECONDITION_READY) return;
        THROW_EXCEPTION(!kind_, THROW_LOGIC_ERROR("DevicePrecondition: choose a preconditioner (useIC, useAMSED, ...) first"))
        check(kind_(h_));
        uint64_t mnnz = 0;
        check(prism_precond_nnz(h_, &mnnz));
        this->m_Mnnz = (UINT32)mnnz;
        this->m_isReady = PRECONDITION_READY;
    }

    // vec = M^{-1} vec
    void MInvSolve(BaseVector<T>& vec) override { apply(vec.getRawValPtr(), vec.getRawValPtr(), vec.getLength(), 0, 0); }

    // vec[resStartIdx : resStartIdx + n] = M^{-1} vec[resStartIdx : resStartIdx + n]
    void MInvSolve(BaseVector<T>& vec, UINT32 resStartIdx) override {
        apply(vec.getRawValPtr(), vec.getRawValPtr(), vec.getLength(), resStartIdx, resStartIdx);
    }

    // vecOUT = M^{-1} vecIN; vecOUT is resized to n
    void MInvSolve(BaseVector<T>& vecIN, BaseVector<T>& vecOUT) override {
        if (vecOUT.getLength() != this->m_ArowNum) vecOUT.resize(this->m_ArowNum, RESERVE_NO_DATA);
        apply(vecIN.getRawValPtr(), vecOUT.getRawValPtr(), vecIN.getLength(), 0, 0, vecOUT.getLength());
    }

    // vecOUT[outStartIdx : outStartIdx + n] = M^{-1} vecIN[inStartIdx : inStartIdx + n]
    void MInvSolve(BaseVector<T>& vecIN, UINT32 inStartIdx, BaseVector<T>& vecOUT, UINT32 outStartIdx) override {
        apply(vecIN.getRawValPtr(), vecOUT.getRawValPtr(), vecIN.getLength(), inStartIdx, outStartIdx,
              vecOUT.getLength());
    }

    // A's values changed on the same pattern (a new time step, a new coefficient
    // field): copy them to the device and recompute the IC / ILDLT factor there on
    // its own pattern (prism_refactor), instead of a new host setup.  The reference
    // has no counterpart: it builds a new preconditioner object.
    void refactor() {
        setup();
        check(prism_update_values(h_, A_->getCSRValuesPtr(0)));
        check(prism_refactor(h_));
    }

    prism_handle handle() const { return h_; }

  private:
    static void check(int32_t rc) {
        THROW_EXCEPTION(rc != PRISM_OK, THROW_RANGE_ERROR(std::string("prism: ") + prism_last_error()))
    }
    void apply(const T* in, T* out, UINT32 in_len, UINT32 in_off, UINT32 out_off, UINT32 out_len = 0) {
        setup();
        const UINT32 n = this->m_ArowNum;
        if (!out_len) out_len = in_len;
        THROW_EXCEPTION(in_off + n > in_len || out_off + n > out_len,
                        THROW_OUT_OF_RANGE("DevicePrecondition: segment out of range"))
        check(prism_apply(h_, in + in_off, out + out_off));
    }

    std::shared_ptr<HOST::CSRMatrix<T>> A_;
    prism_handle h_ = nullptr;
    std::function<int32_t(prism_handle)> kind_;
};

#endif  // PRISM_DEVICE_PRECONDITION_HPP
