/* LAPACKE declarations for the reference checker build -- TEST INFRASTRUCTURE
 * ONLY.  The reference calls LAPACKE_dstevx / sstevx / dlamch / slamch
 * (AMSEDPrecondition.cpp:975-1006) and dhseqr (GMSLRDPrecondition.cpp:1011).
 * LAPACK is not part of its sources; the checker links the OpenBLAS shipped
 * with scipy in this image, whose LAPACKE symbols carry a `scipy_` prefix. */
#ifndef PRISM_REF_LAPACKE_SHIM_H
#define PRISM_REF_LAPACKE_SHIM_H
typedef int lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
#ifdef __cplusplus
extern "C" {
#endif
lapack_int scipy_LAPACKE_dstevx(int layout, char jobz, char range, lapack_int n, double* d, double* e, double vl,
                                double vu, lapack_int il, lapack_int iu, double abstol, lapack_int* m, double* w,
                                double* z, lapack_int ldz, lapack_int* ifail);
lapack_int scipy_LAPACKE_sstevx(int layout, char jobz, char range, lapack_int n, float* d, float* e, float vl,
                                float vu, lapack_int il, lapack_int iu, float abstol, lapack_int* m, float* w,
                                float* z, lapack_int ldz, lapack_int* ifail);
double scipy_LAPACKE_dlamch(char cmach);
float scipy_LAPACKE_slamch(char cmach);
lapack_int scipy_LAPACKE_dhseqr(int layout, char job, char compz, lapack_int n, lapack_int ilo, lapack_int ihi,
                                double* h, lapack_int ldh, double* wr, double* wi, double* z, lapack_int ldz);
lapack_int scipy_LAPACKE_shseqr(int layout, char job, char compz, lapack_int n, lapack_int ilo, lapack_int ihi,
                                float* h, lapack_int ldh, float* wr, float* wi, float* z, lapack_int ldz);
#ifdef __cplusplus
}
#endif
#define LAPACKE_dstevx scipy_LAPACKE_dstevx
#define LAPACKE_sstevx scipy_LAPACKE_sstevx
#define LAPACKE_dlamch scipy_LAPACKE_dlamch
#define LAPACKE_slamch scipy_LAPACKE_slamch
#define LAPACKE_dhseqr scipy_LAPACKE_dhseqr
#define LAPACKE_shseqr scipy_LAPACKE_shseqr
#endif
