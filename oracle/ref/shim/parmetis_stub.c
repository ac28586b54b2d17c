/* ParMETIS entry point for the single-rank oracle build: never reached with
 * HEMELB_USE_PARMETIS off; refuses loudly if it ever is. */
#include <stdio.h>
#include "parmetis.h"
int ParMETIS_V3_PartKway(idx_t* vtxdist, idx_t* xadj, idx_t* adjncy, idx_t* vwgt, idx_t* adjwgt,
                         idx_t* wgtflag, idx_t* numflag, idx_t* ncon, idx_t* nparts, real_t* tpwgts,
                         real_t* ubvec, idx_t* options, idx_t* edgecut, idx_t* part, MPI_Comm* comm) {
  (void)vtxdist; (void)xadj; (void)adjncy; (void)vwgt; (void)adjwgt; (void)wgtflag; (void)numflag;
  (void)ncon; (void)nparts; (void)tpwgts; (void)ubvec; (void)options; (void)edgecut; (void)part;
  (void)comm;
  fprintf(stderr, "single-rank oracle: ParMETIS partitioning is not available\n");
  return METIS_ERROR;
}
