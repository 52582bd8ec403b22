/* Stand-in for METIS in the reference checker build -- TEST INFRASTRUCTURE ONLY.
 * METIS is not part of the reference's sources.  The reference calls
 * METIS_PartGraphRecursive / METIS_PartGraphKway for 2-way partitions when it
 * builds its HID ordering (include/utils/ExternalTools/MetisTools.h:173-180);
 * here both entry points forward to the deterministic bisection that the
 * product's AMSED setup uses (prispack_b200/csrc/partition.cpp, compiled into
 * the checker build), so reference and product consume the same partition. */
#ifndef PRISM_REF_METIS_SHIM_H
#define PRISM_REF_METIS_SHIM_H
#include <stdint.h>
typedef int32_t idx_t;
typedef float real_t;
#define METIS_OK 1
#define METIS_ERROR -4
#ifdef __cplusplus
extern "C" {
#endif
int64_t prism_graph_bisect(int32_t n, const int32_t* xadj, const int32_t* adjncy, int32_t* part);
#ifdef __cplusplus
}
#endif
static inline int prism_metis_two_way(idx_t* nvtxs, idx_t* xadj, idx_t* adjncy, idx_t* nparts, idx_t* edgecut,
                                      idx_t* part) {
    if (*nparts != 2) return METIS_ERROR;
    *edgecut = (idx_t)prism_graph_bisect(*nvtxs, xadj, adjncy, part);
    return METIS_OK;
}
static inline int METIS_PartGraphRecursive(idx_t* nvtxs, idx_t* ncon, idx_t* xadj, idx_t* adjncy, idx_t* vwgt,
                                           idx_t* vsize, idx_t* adjwgt, idx_t* nparts, real_t* tpwgts,
                                           real_t* ubvec, idx_t* options, idx_t* edgecut, idx_t* part) {
    (void)ncon; (void)vwgt; (void)vsize; (void)adjwgt; (void)tpwgts; (void)ubvec; (void)options;
    return prism_metis_two_way(nvtxs, xadj, adjncy, nparts, edgecut, part);
}
static inline int METIS_PartGraphKway(idx_t* nvtxs, idx_t* ncon, idx_t* xadj, idx_t* adjncy, idx_t* vwgt,
                                      idx_t* vsize, idx_t* adjwgt, idx_t* nparts, real_t* tpwgts, real_t* ubvec,
                                      idx_t* options, idx_t* edgecut, idx_t* part) {
    (void)ncon; (void)vwgt; (void)vsize; (void)adjwgt; (void)tpwgts; (void)ubvec; (void)options;
    return prism_metis_two_way(nvtxs, xadj, adjncy, nparts, edgecut, part);
}
#endif
