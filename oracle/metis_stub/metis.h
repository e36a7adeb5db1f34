/* Minimal stand-in for metis.h so that the reference grid reader compiles for the oracle.
 * Test infrastructure only.  The reference calls METIS only when nPartitions > 1
 * (read_and_process_grid.cpp:1101-1134); the oracle always asks for one partition, so every
 * entry point here reports an error instead of partitioning. */
#pragma once
#include <stdint.h>
typedef int32_t idx_t;
enum { METIS_OK = 1, METIS_ERROR = -4 };
enum {
    METIS_OPTION_NSEPS = 0, METIS_OPTION_NITER, METIS_OPTION_UFACTOR,
    METIS_OPTION_COMPRESS, METIS_OPTION_CCORDER, METIS_NOPTIONS = 40
};
static inline int METIS_SetDefaultOptions(idx_t* opt) {
    for (int i = 0; i < METIS_NOPTIONS; i++) opt[i] = -1;
    return METIS_OK;
}
static inline int METIS_PartGraphKway(idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*,
                                      idx_t*, float*, float*, idx_t*, idx_t*, idx_t*) {
    return METIS_ERROR;
}
static inline int METIS_NodeND(idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*) {
    return METIS_ERROR;
}
