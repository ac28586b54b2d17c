/* ParMETIS stand-in (CPU oracle build only).  With HEMELB_USE_PARMETIS off (the
 * reference's default, src/CMakeLists.txt:30) the decomposition never calls
 * ParMETIS, but OptimisedDecomposition::CallParmetis is still compiled, so the
 * one entry point it names is declared; the stub refuses to partition.  The
 * index types follow ParMETIS 4's defaults (64-bit idx_t here, 32-bit real_t). */
#ifndef HB_REF_SHIM_PARMETIS_H
#define HB_REF_SHIM_PARMETIS_H
#include <stdint.h>
#include "mpi.h"
#define PARMETIS_MAJOR_VERSION 4
#define METIS_OK 1
#define METIS_ERROR (-4)
typedef int64_t idx_t;
typedef float real_t;
#ifdef __cplusplus
extern "C" {
#endif
int ParMETIS_V3_PartKway(idx_t* vtxdist, idx_t* xadj, idx_t* adjncy, idx_t* vwgt, idx_t* adjwgt,
                         idx_t* wgtflag, idx_t* numflag, idx_t* ncon, idx_t* nparts, real_t* tpwgts,
                         real_t* ubvec, idx_t* options, idx_t* edgecut, idx_t* part, MPI_Comm* comm);
#ifdef __cplusplus
}
#endif
#endif
