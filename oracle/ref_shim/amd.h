/* Stand-in for SuiteSparse AMD in the reference checker build -- TEST
 * INFRASTRUCTURE ONLY.  AMD is not part of the reference's sources; the
 * checker uses the vendored RCM ordering (MatrixReorderRCM) only, so amd_order
 * reports failure if it is ever reached. */
#ifndef PRISM_REF_AMD_SHIM_H
#define PRISM_REF_AMD_SHIM_H
#define AMD_OK 0
#define AMD_OK_BUT_JUMBLED 1
#define AMD_INVALID -2
static inline int amd_order(int n, const int* Ap, const int* Ai, int* P, double* Control, double* Info) {
    (void)n; (void)Ap; (void)Ai; (void)P; (void)Control; (void)Info;
    return AMD_INVALID;
}
#endif
