/* Declarations standing in for METIS 5's metis.h, enough for the reference's
 * partition.hpp / partition.cu / problem.hpp to compile.  The serial and OMP
 * loops never call METIS; the definitions in stubs.cpp abort if reached. */
#ifndef FOT_STUB_METIS_H
#define FOT_STUB_METIS_H
#include <stdint.h>
typedef int32_t idx_t;
typedef float real_t;
#define METIS_NOPTIONS 40
#define METIS_OK 1
#define METIS_OPTION_OBJTYPE 1
#define METIS_OBJTYPE_VOL 1
#ifdef __cplusplus
extern "C" {
#endif
int METIS_SetDefaultOptions(idx_t *options);
int METIS_PartGraphKway(idx_t *nvtxs, idx_t *ncon, idx_t *xadj, idx_t *adjncy,
                        idx_t *vwgt, idx_t *vsize, idx_t *adjwgt, idx_t *nparts,
                        real_t *tpwgts, real_t *ubvec, idx_t *options,
                        idx_t *edgecut, idx_t *part);
#ifdef __cplusplus
}
#endif
#endif
