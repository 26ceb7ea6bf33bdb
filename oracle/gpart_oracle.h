/*
 * CPU oracle of the Acc-GPart multilevel k-way partitioner — TEST
 * INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load liboracle.so; the product never does.
 *
 * Parity status: coarsening, contraction and the METIS step are pinned against
 * the reference's own CUDA build (tests/golden/*.json, produced by
 * tests/golden/make_golden.py on a B200).  Refinement is the reference's LP,
 * priority filter, exact update and capacity exchange restated serially, with
 * the repair step in the deterministic (bucket, repair hash, id) order that
 * the GPU path also uses (the reference ranks repair donors by atomic
 * arrival).  Single-level refinement without repair batches is pinned against
 * the reference's refine_partition (tests/golden/refine_cases.json).
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
/* RefineStats of include/refine.hpp:28-53 (the fields describing moves). */
typedef struct orc_refine_stats {
    int32_t rounds, admission_iterations, checkpoint_updates, reserved;
    uint64_t proposals, accepted, initial_cut, final_cut, final_max_part_weight, capacity;
    uint64_t lp_cut_gain, lp_cut_loss, rebalance_cut_gain, rebalance_cut_loss;
    uint64_t group_cut_gain, group_accepted;
} orc_refine_stats;

/* refine_partition (include/refine.hpp:84-88): one level of refinement of
 * `labels` (in/out) with the given round and exchange budgets. */
int orc_refine(const orc_csr* graph, int32_t k, double epsilon, int32_t max_rounds,
               int32_t exchange_rounds, int32_t* labels, orc_refine_stats* stats);

/* Refined labels of every level (level order as in the hierarchy). */
int orc_level_labels(int32_t level, int32_t* labels);
/* Cut after refinement of a level, and whether that level was refined. */
int orc_level_result(int32_t level, uint64_t* cut, int32_t* refined);

#ifdef __cplusplus
}
#endif
#endif
