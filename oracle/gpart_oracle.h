/*
 * CPU oracle of the Acc-GPart multilevel k-way partitioner — TEST
 * INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load liboracle.so; the product never does.
 *
 * Parity status: coarsening, contraction and the METIS step are pinned against
 * the reference's own CUDA build (tests/golden/*.json, produced by
 * tests/golden/make_golden.py on a B200).  Refinement is the reference's LP,
 * priority filter, exact update and capacity exchange restated serially, with
 * the repair step in the deterministic (bucket, vertex id) order that the
 * GPU path also uses (the reference ranks repair donors by atomic arrival).
 */
#ifndef GPART_ORACLE_H
#define GPART_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_csr {
    int64_t n, m;
    const int32_t* offsets;
    const int32_t* neighbors;
    const uint32_t* vertex_weights; /* NULL: unit */
    const uint32_t* edge_weights;   /* NULL: unit */
} orc_csr;

#define ORC_FLAG_NO_SEED_MATCHING 0x4u
#define ORC_FLAG_COARSEN_ONLY 0x10u

/* Returns 0 on success, otherwise a gp_status-compatible code; the message is
 * available from orc_last_error().  The hierarchy, the METIS labels and the
 * per-level refinement results stay available through the accessors until
 * the next call on the same thread. */
int orc_partition(const orc_csr* graph, int32_t k, double epsilon, uint32_t seed,
                  uint32_t flags, int32_t* labels_out, uint64_t* cut_out);
const char* orc_last_error(void);
int orc_level_count(void);
int orc_level_size(int32_t level, int64_t* n, int64_t* m);
int orc_level_copy(int32_t level, int32_t* offsets, int32_t* neighbors,
                   uint32_t* edge_weights, uint32_t* vertex_weights, int32_t* map,
                   uint64_t* metadata);
int orc_initial_labels(int32_t* labels, int64_t capacity);
/* Refined labels of every level (level order as in the hierarchy). */
int orc_level_labels(int32_t level, int32_t* labels);
/* Cut after refinement of a level, and whether that level was refined. */
int orc_level_result(int32_t level, uint64_t* cut, int32_t* refined);

#ifdef __cplusplus
}
#endif
#endif
