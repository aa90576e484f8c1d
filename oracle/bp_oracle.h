/*
 * bp_oracle.h -- CPU restatement of the reference's belief-propagation
 * arithmetic.  TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA
 * kernels.  Nothing in the product links it; only tests/, the smoke check and
 * the bench's CPU-baseline leg load it.
 *
 * It restates, in this project's own code, the schedules of the reference's
 * src/graph/graph.c on the reference's own host layout (node beliefs at a
 * MAX_STATES stride, joint tables at MAX_STATES^2, messages at MAX_STATES, all
 * indexed by edge id), so its float build can be compared bit for bit with the
 * reference compiled from source.  The double build runs the same schedule in
 * fp64 and is used to state every configuration's error against fp64.
 *
 * Where the reference reads uninitialised memory (graphs whose nodes have
 * different state counts: graph.c:462, :481-483, :851-857; message slots at or
 * beyond an edge's x_dim that init_edge never zeroes, graph.c:99-105), this
 * restatement reads zeros.  That is the convention of the CUDA engine too.
 */
#ifndef BP_ORACLE_H_
#define BP_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BPO_MS 10 /* MAX_STATES of the reference (constants.h:11) */

typedef struct {
    uint32_t V, E;
    const uint32_t *num_states; /* [V] */
    const uint32_t *edge_src;   /* [E] */
    const uint32_t *edge_dst;   /* [E] */
    const float *joint;         /* [E][10][10]: row i < S_src, column j < S_dst */
    const uint32_t *in_ptr;     /* [V+1] dest-CSR row starts (last = E) */
    const uint32_t *in_edges;   /* [E]   edge ids, per node in insertion order */
    const uint32_t *out_ptr;    /* [V+1] src-CSR */
    const uint32_t *out_edges;  /* [E] */
} bpo_graph;

typedef struct {
    uint32_t executed;   /* iterations actually run */
    int swapped_odd;     /* 1 when the caller's previous/current arrays swapped an odd number of times */
    double delta;        /* last delta (the reference's `delta`) */
    double prev_delta;   /* the reference's `previous_delta` at return */
} bpo_loopy_info;

/* stable counting sort of edges by key (graph.c:249-313 order) */
void bpo_build_csr(uint32_t V, uint32_t E, const uint32_t *key, uint32_t *ptr, uint32_t *order);

/* level lists of the tree schedule (graph.c:753-827), O(V+E).  Returns 0, or
 * -1 when some node is unreachable from the in-degree<=2 seed set (where the
 * reference loops forever). */
int bpo_levels(const bpo_graph *g, uint32_t *levels, uint32_t *num_levels);

#define BPO_DECLARE(R, SFX)                                                              \
    void bpo_init_messages_##SFX(const bpo_graph *g, const R *b, R *m_prev);             \
    uint32_t bpo_loopy_##SFX(const bpo_graph *g, R *b, R *m_prev, R *m_cur, R tol,      \
                             uint32_t max_it, uint32_t check_every, int verbose,        \
                             bpo_loopy_info *info);                                     \
    uint32_t bpo_loopy_edge_##SFX(const bpo_graph *g, R *b, R *m_prev, R *m_cur, R tol, \
                                  uint32_t max_it, int acc, int verbose,                \
                                  bpo_loopy_info *info);                                \
    void bpo_tree_start_##SFX(const bpo_graph *g, const uint32_t *levels,                \
                              uint32_t num_levels, char *visited, const R *b, R *m);     \
    void bpo_tree_level_##SFX(const bpo_graph *g, const uint32_t *levels,                \
                              uint32_t num_levels, uint32_t level, char *visited, R *m); \
    void bpo_tree_marginalize_##SFX(const bpo_graph *g, R *b, const R *m);               \
    void bpo_tree_##SFX(const bpo_graph *g, const uint32_t *levels, uint32_t num_levels, \
                        R *b, R *m);

BPO_DECLARE(float, f32)
BPO_DECLARE(double, f64)

#ifdef __cplusplus
}
#endif

#endif
