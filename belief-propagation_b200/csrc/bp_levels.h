/* bp_levels.h -- host helpers of the tree schedule (levels.c) */
#ifndef BP_LEVELS_H_
#define BP_LEVELS_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* init_levels_to_nodes (graph.c:806-827) from CSR arrays: in_ptr [V+1],
 * out_ptr [V+1], out_dst [E] (destination of each out-edge, src order).
 * Returns 0, -1 when a node is unreachable from the seed set (the reference
 * loops forever there), -2 on allocation failure. */
int bp_levels_from_csr(uint32_t V, const uint32_t *in_ptr, const uint32_t *out_ptr, const uint32_t *out_dst,
                       uint32_t *levels, uint32_t *num_levels);

/* waves of every level; wave_nodes [V]; *wave_off_out (malloc'd) has
 * total_waves + 1 entries; level_wave_begin [num_levels + 1]. Returns 0, -1
 * on malformed levels, -2 on allocation failure. */
int bp_tree_waves(uint32_t V, const uint32_t *levels, uint32_t num_levels, const uint32_t *in_ptr,
                  const uint32_t *in_src, uint32_t *node_level, uint32_t *node_lidx, uint32_t *wave_nodes,
                  uint32_t **wave_off_out, uint32_t *level_wave_begin, uint32_t *total_waves);

#ifdef __cplusplus
}
#endif

#endif
