/*
 * bp_oracle.c -- CPU restatement of the reference's BP schedules.
 * TEST INFRASTRUCTURE ONLY: the checker the CUDA engine is compared against.
 * Built by oracle/Makefile into oracle/_ref/libbp_oracle.so (not linked by
 * the product).  Must be compiled without FMA contraction
 * (-ffp-contract=off) so the float build keeps the reference's rounding.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bp_oracle.h"

/* stable counting sort: per key in insertion order, keys ascending.  This is
 * the order set_up_src_nodes_to_edges / set_up_dest_nodes_to_edges produce
 * from their per-node buckets (graph.c:249-313). */
void bpo_build_csr(uint32_t V, uint32_t E, const uint32_t *key, uint32_t *ptr, uint32_t *order)
{
    memset(ptr, 0, sizeof(uint32_t) * ((size_t)V + 1));
    for (uint32_t e = 0; e < E; ++e)
        ptr[key[e] + 1]++;
    for (uint32_t v = 0; v < V; ++v)
        ptr[v + 1] += ptr[v];
    uint32_t *fill = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)V + 1));
    memcpy(fill, ptr, sizeof(uint32_t) * ((size_t)V + 1));
    for (uint32_t e = 0; e < E; ++e)
        order[fill[key[e]]++] = e;
    free(fill);
}

/* init_levels_to_nodes, graph.c:753-827.  The reference finds "already
 * listed" by scanning the whole list (graph.c:792-797); a flag per node gives
 * the same list in O(V+E). */
int bpo_levels(const bpo_graph *g, uint32_t *levels, uint32_t *num_levels)
{
    uint32_t V = g->V;
    char *visited = (char *)calloc(V ? V : 1, 1);
    char *listed = (char *)calloc(V ? V : 1, 1);
    uint32_t end = V;
    levels[0] = V;
    for (uint32_t v = 0; v < V; ++v) {
        if (g->in_ptr[v + 1] - g->in_ptr[v] <= 2) {
            levels[end++] = v;
            listed[v] = 1;
        }
    }
    uint32_t scan_from = V;
    int rc = 0;
    while (end < 2 * V) {
        uint32_t copy_end = end;
        for (uint32_t k = scan_from; k < copy_end; ++k) {
            uint32_t u = levels[k];
            if (visited[u])
                continue;
            visited[u] = 1;
            for (uint32_t q = g->out_ptr[u]; q < g->out_ptr[u + 1]; ++q) {
                uint32_t w = g->edge_dst[g->out_edges[q]];
                if (!listed[w]) {
                    listed[w] = 1;
                    levels[end++] = w;
                }
            }
        }
        scan_from = copy_end;
        *num_levels += 1;
        levels[*num_levels] = copy_end;
        if (end == copy_end && end < 2 * V) {
            rc = -1; /* no progress: the reference would loop forever */
            break;
        }
    }
    *num_levels += 1;
    free(visited);
    free(listed);
    return rc;
}

#define R float
#define SFX f32
#include "bp_oracle_impl.inc"
#undef R
#undef SFX

#define R double
#define SFX f64
#include "bp_oracle_impl.inc"
#undef R
#undef SFX
