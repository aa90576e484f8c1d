/*
 * ref_shim.c -- TEST INFRASTRUCTURE ONLY.  Compiled together with the
 * reference's unmodified src/graph/graph.c (and, for the BIF build, its
 * vendored parser) into oracle/_ref/, so tests can drive the reference's own
 * C engine on the same inputs as the CUDA engine.
 *
 * Graph construction follows the reference's API (create_graph,
 * graph_add_node, graph_set_node_state, graph_add_edge, set_up_*) when every
 * node has at most MAX_DEGREE in- and out-edges.  Larger graphs are filled
 * into struct graph directly (init_edge per edge, CSR arrays from a stable
 * counting sort -- the order set_up_*_nodes_to_edges produce,
 * graph.c:249-313), skipping only the hsearch bookkeeping that caps the
 * degree at MAX_DEGREE (graph.c:184, :201).  The message and belief arrays
 * are zeroed after create_graph so the slots the reference leaves
 * uninitialised (graph.c:33, :99-105) read as zeros.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

#include "graph.h"

static void counting_sort(uint32_t V, uint32_t E, const uint32_t *key, unsigned int *ptr,
                          unsigned int *order, uint32_t *max_deg)
{
    uint32_t *cnt = (uint32_t *)calloc((size_t)V + 1, sizeof(uint32_t));
    for (uint32_t e = 0; e < E; ++e)
        cnt[key[e] + 1]++;
    uint32_t md = 0;
    for (uint32_t v = 0; v < V; ++v) {
        if (cnt[v + 1] > md)
            md = cnt[v + 1];
        cnt[v + 1] += cnt[v];
    }
    for (uint32_t v = 0; v < V; ++v)
        ptr[v] = cnt[v];
    for (uint32_t e = 0; e < E; ++e)
        order[cnt[key[e]]++] = e;
    if (max_deg)
        *max_deg = md;
    free(cnt);
}

static uint32_t max_degree_of(uint32_t V, uint32_t E, const uint32_t *key)
{
    uint32_t *cnt = (uint32_t *)calloc((size_t)V + 1, sizeof(uint32_t));
    uint32_t md = 0;
    for (uint32_t e = 0; e < E; ++e)
        if (++cnt[key[e]] > md)
            md = cnt[key[e]];
    free(cnt);
    return md;
}

/* beliefs: [V][MAX_STATES]; observed: [V] (0/1) or NULL; joint: [E][10][10] */
Graph_t refshim_build(uint32_t V, uint32_t E, const uint32_t *num_states, const float *beliefs,
                      const uint8_t *observed, const uint32_t *src, const uint32_t *dst,
                      const float *joint, int force_direct)
{
    char name[CHAR_BUFFER_SIZE];
    Graph_t g = create_graph(V, E);
    memset(g->edges_messages, 0, sizeof(float) * MAX_STATES * (size_t)E);
    memset(g->last_edges_messages, 0, sizeof(float) * MAX_STATES * (size_t)E);
    memset(g->node_states, 0, sizeof(float) * MAX_STATES * (size_t)V);
    for (uint32_t v = 0; v < V; ++v) {
        snprintf(name, sizeof(name), "n%u", v);
        graph_add_node(g, num_states[v], name);
        node_set_state(g, v, num_states[v], (float *)(beliefs + (size_t)MAX_STATES * v));
        if (observed && observed[v])
            g->observed_nodes[v] = 1;
    }
    int direct = force_direct || E == 0 || max_degree_of(V, E, src) >= MAX_DEGREE ||
                 max_degree_of(V, E, dst) >= MAX_DEGREE;
    if (!direct) {
        for (uint32_t e = 0; e < E; ++e)
            graph_add_edge(g, src[e], dst[e], num_states[src[e]], num_states[dst[e]],
                           (float *)(joint + (size_t)MAX_STATES * MAX_STATES * e));
        set_up_src_nodes_to_edges(g);
        set_up_dest_nodes_to_edges(g);
    } else {
        for (uint32_t e = 0; e < E; ++e)
            init_edge(g, e, src[e], dst[e], num_states[src[e]], num_states[dst[e]],
                      (float *)(joint + (size_t)MAX_STATES * MAX_STATES * e));
        g->current_num_edges = E;
        uint32_t md = 0;
        counting_sort(V, E, src, g->src_nodes_to_edges_node_list, g->src_nodes_to_edges_edge_list, &md);
        counting_sort(V, E, dst, g->dest_nodes_to_edges_node_list, g->dest_nodes_to_edges_edge_list, NULL);
        g->max_degree = md;
    }
    return g;
}

int refshim_used_direct_fill(Graph_t g) { return g->edge_tables_created == 0; }

void refshim_get_beliefs(Graph_t g, float *out)
{
    memcpy(out, g->node_states, sizeof(float) * MAX_STATES * (size_t)g->current_num_vertices);
}

void refshim_set_beliefs(Graph_t g, const float *in)
{
    memcpy(g->node_states, in, sizeof(float) * MAX_STATES * (size_t)g->current_num_vertices);
}

/* which: 0 = edges_messages, 1 = last_edges_messages, 2 = *previous_edge_messages,
 * 3 = *current_edge_messages */
void refshim_get_messages(Graph_t g, int which, float *out)
{
    const float *src = which == 0 ? g->edges_messages
                     : which == 1 ? g->last_edges_messages
                     : which == 2 ? *g->previous_edge_messages
                                  : *g->current_edge_messages;
    memcpy(out, src, sizeof(float) * MAX_STATES * (size_t)g->current_num_edges);
}

void refshim_set_messages(Graph_t g, int which, const float *in)
{
    float *dst = which == 0 ? g->edges_messages
               : which == 1 ? g->last_edges_messages
               : which == 2 ? *g->previous_edge_messages
                            : *g->current_edge_messages;
    memcpy(dst, in, sizeof(float) * MAX_STATES * (size_t)g->current_num_edges);
}

int refshim_previous_is_edges_messages(Graph_t g) { return *g->previous_edge_messages == g->edges_messages; }

unsigned int refshim_num_levels(Graph_t g) { return g->num_levels; }

void refshim_get_levels(Graph_t g, unsigned int *out)
{
    memcpy(out, g->levels_to_nodes, sizeof(unsigned int) * 2 * (size_t)g->current_num_vertices);
}

void refshim_get_csr(Graph_t g, unsigned int *src_ptr, unsigned int *src_edges, unsigned int *dst_ptr,
                     unsigned int *dst_edges)
{
    memcpy(src_ptr, g->src_nodes_to_edges_node_list, sizeof(unsigned int) * g->current_num_vertices);
    memcpy(dst_ptr, g->dest_nodes_to_edges_node_list, sizeof(unsigned int) * g->current_num_vertices);
    memcpy(src_edges, g->src_nodes_to_edges_edge_list, sizeof(unsigned int) * g->current_num_edges);
    memcpy(dst_edges, g->dest_nodes_to_edges_edge_list, sizeof(unsigned int) * g->current_num_edges);
}

/* graph dump for fixtures: sizes, then arrays in the reference's layout */
void refshim_sizes(Graph_t g, unsigned int *V, unsigned int *E) { *V = g->current_num_vertices; *E = g->current_num_edges; }

void refshim_dump(Graph_t g, unsigned int *num_states, float *beliefs, unsigned char *observed,
                  unsigned int *src, unsigned int *dst, float *joint)
{
    unsigned int V = g->current_num_vertices, E = g->current_num_edges;
    memcpy(num_states, g->node_num_vars, sizeof(unsigned int) * V);
    memcpy(beliefs, g->node_states, sizeof(float) * MAX_STATES * (size_t)V);
    for (unsigned int v = 0; v < V; ++v)
        observed[v] = (unsigned char)g->observed_nodes[v];
    memcpy(src, g->edges_src_index, sizeof(unsigned int) * E);
    memcpy(dst, g->edges_dest_index, sizeof(unsigned int) * E);
    for (unsigned int e = 0; e < E; ++e) {
        unsigned int x = g->edges_x_dim[e], y = g->edges_y_dim[e];
        float *out = joint + (size_t)MAX_STATES * MAX_STATES * e;
        memset(out, 0, sizeof(float) * MAX_STATES * MAX_STATES);
        for (unsigned int i = 0; i < x; ++i)
            for (unsigned int j = 0; j < y; ++j)
                out[MAX_STATES * i + j] = g->edges_joint_probabilities[(size_t)MAX_STATES * MAX_STATES * e + MAX_STATES * i + j];
    }
}

/* the drivers' tree sequence (c_benchmark/main.c:224-236) on the reference */
void refshim_tree(Graph_t g)
{
    unsigned int i;
    init_levels_to_nodes(g);
    propagate_using_levels_start(g);
    for (i = 1; i < g->num_levels - 1; ++i)
        propagate_using_levels(g, i);
    reset_visited(g);
    for (i = g->num_levels - 1; i > 0; --i)
        propagate_using_levels(g, i);
    marginalize(g);
}
