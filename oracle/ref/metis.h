/* Declarations of the public METIS 5 API, written for building the reference
 * partitioner against the METIS that ships inside the CUDA toolkit
 * (libmetis_static.a).  The widths (64-bit idx_t, 32-bit real_t) and the
 * option indices (SEED = 8, NUMBERING = 17, 40 option slots) were established
 * by running that library on CPU: varying options[8] changes the partition
 * while options[9] does not, and options[17] = 1 accepts 1-based input.
 * That layout is the METIS 5.1 one. */
#ifndef GPART_REF_METIS_H
#define GPART_REF_METIS_H
#include <stdint.h>
typedef int64_t idx_t;
typedef float real_t;
#define METIS_VER_MAJOR 0
#define METIS_VER_MINOR 0
#define METIS_VER_SUBMINOR 0
#define METIS_NOPTIONS 40
enum { METIS_OK = 1, METIS_ERROR_INPUT = -2, METIS_ERROR_MEMORY = -3, METIS_ERROR = -4 };
enum { METIS_OPTION_SEED = 8, METIS_OPTION_NUMBERING = 17 };
#ifdef __cplusplus
extern "C" {
#endif
int METIS_SetDefaultOptions(idx_t* options);
int METIS_PartGraphKway(idx_t* nvtxs, idx_t* ncon, idx_t* xadj, idx_t* adjncy,
                        idx_t* vwgt, idx_t* vsize, idx_t* adjwgt, idx_t* nparts,
                        real_t* tpwgts, real_t* ubvec, idx_t* options,
                        idx_t* objval, idx_t* part);
#ifdef __cplusplus
}
#endif
#endif
