/*
 * levels.c -- level lists and intra-level waves of the tree schedule.
 *
 * bp_levels_from_csr restates init_levels_to_nodes (graph.c:806-827):
 * level 0 lists, in ascending id, every node with in-degree <= 2
 * (fill_in_leaf_nodes_in_index with max_count 2, graph.c:753-772); each later
 * level lists, in visiting order, the out-neighbours of the previous level
 * that are not listed yet (visit_node, graph.c:774-804).  The reference finds
 * "listed yet" by scanning the whole list, O(V^2); a flag per node gives the
 * identical list in O(V + E).  Offsets go to levels[0..num_levels), nodes to
 * levels[V..2V), and num_levels continues from the caller's value as in the
 * reference (which never resets it).
 *
 * bp_tree_waves splits each level into waves for the GPU.  Inside a level the
 * reference processes nodes one after another and node u sends to w only if
 * w has not been processed yet (graph.c:508-521), so a later node of the same
 * level can read a message an earlier one just wrote.  Node k of a level is
 * put one wave after the latest earlier node of its level that has an edge
 * into it; nodes of one wave never depend on each other, so a wave is one
 * kernel launch.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "bp_levels.h"

int bp_levels_from_csr(uint32_t V, const uint32_t *in_ptr, const uint32_t *out_ptr, const uint32_t *out_dst,
                       uint32_t *levels, uint32_t *num_levels)
{
    char *visited = (char *)calloc(V ? V : 1, 1);
    char *listed = (char *)calloc(V ? V : 1, 1);
    if (!visited || !listed) {
        free(visited);
        free(listed);
        return -2;
    }
    uint32_t end = V;
    levels[0] = V;
    for (uint32_t v = 0; v < V; ++v) {
        if (in_ptr[v + 1] - in_ptr[v] <= 2) {
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
            for (uint32_t q = out_ptr[u]; q < out_ptr[u + 1]; ++q) {
                uint32_t w = out_dst[q];
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
            rc = -1;
            break;
        }
    }
    *num_levels += 1;
    free(visited);
    free(listed);
    return rc;
}

int bp_tree_waves(uint32_t V, const uint32_t *levels, uint32_t num_levels, const uint32_t *in_ptr,
                  const uint32_t *in_src, uint32_t *node_level, uint32_t *node_lidx, uint32_t *wave_nodes,
                  uint32_t **wave_off_out, uint32_t *level_wave_begin, uint32_t *total_waves)
{
    uint32_t *wave = (uint32_t *)malloc(sizeof(uint32_t) * (V ? V : 1));
    if (!wave)
        return -2;
    for (uint32_t v = 0; v < V; ++v)
        node_level[v] = 0xffffffffu;
    for (uint32_t l = 0; l < num_levels; ++l) {
        uint32_t lo = levels[l], hi = (l + 1 == num_levels) ? 2 * V : levels[l + 1];
        if (lo < V || hi > 2 * V || lo > hi) {
            free(wave);
            return -1;
        }
        for (uint32_t k = lo; k < hi; ++k) {
            uint32_t u = levels[k];
            if (u >= V) {
                free(wave);
                return -1;
            }
            node_level[u] = l;
            node_lidx[u] = k - lo;
        }
    }
    /* waves per level */
    uint32_t cap = 64, nw = 0;
    uint32_t *off = (uint32_t *)malloc(sizeof(uint32_t) * cap);
    uint32_t filled = 0;
    for (uint32_t l = 0; l < num_levels; ++l) {
        uint32_t lo = levels[l], hi = (l + 1 == num_levels) ? 2 * V : levels[l + 1];
        uint32_t maxw = 0;
        for (uint32_t k = lo; k < hi; ++k) {
            uint32_t u = levels[k], w = 0;
            for (uint32_t p = in_ptr[u]; p < in_ptr[u + 1]; ++p) {
                uint32_t s = in_src[p];
                if (node_level[s] == l && node_lidx[s] < k - lo && wave[s] + 1 > w)
                    w = wave[s] + 1;
            }
            wave[u] = w;
            if (w > maxw)
                maxw = w;
        }
        level_wave_begin[l] = nw;
        uint32_t nwl = (hi > lo) ? maxw + 1 : 0;
        if (nw + nwl + 1 > cap) {
            while (nw + nwl + 1 > cap)
                cap *= 2;
            off = (uint32_t *)realloc(off, sizeof(uint32_t) * cap);
        }
        /* counting sort of the level's nodes by wave, stable */
        uint32_t *cnt = (uint32_t *)calloc(nwl + 1, sizeof(uint32_t));
        for (uint32_t k = lo; k < hi; ++k)
            cnt[wave[levels[k]] + 1]++;
        for (uint32_t w = 0; w < nwl; ++w)
            cnt[w + 1] += cnt[w];
        for (uint32_t w = 0; w < nwl; ++w)
            off[nw + w] = filled + cnt[w];
        for (uint32_t k = lo; k < hi; ++k) {
            uint32_t u = levels[k];
            wave_nodes[filled + cnt[wave[u]]++] = u;
        }
        filled += hi - lo;
        nw += nwl;
        free(cnt);
    }
    level_wave_begin[num_levels] = nw;
    off[nw] = filled;
    *wave_off_out = off;
    *total_waves = nw;
    free(wave);
    return 0;
}
